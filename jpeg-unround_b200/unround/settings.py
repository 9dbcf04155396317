"""The settings of a reconstruction: the method, the model, and the solvers' options.

The same dataclasses, fields and defaults as the reference package's settings
(python/src/unround/settings.py:22-148 of JPEG-Unround), each field an option of the
command line (docs/cli.md:182-243) under the name unround.native.options gives it; the
library checks their ranges. A value of None takes the library's default.
"""

from dataclasses import dataclass, field
from typing import Literal

__all__ = ["TGV", "TV", "Centres", "DataTerm", "Method", "PdhgOptions", "Settings", "SubgradientOptions"]

type Method = Literal["mmse", "tv", "tgv", "subgradient"]
type Centres = Literal["mmse", "midpoint"]


@dataclass(frozen=True, slots=True)
class DataTerm:
    """The data term G of a component (docs/math.md 4.1): mu or its rule, the weights, the
    centres, the slack and its cost, and the flat blocks' weight."""

    mu: float | None = None
    mu_scale: float = 9.0
    mu_power: float = 0.9
    mu_chroma: float = 0.3
    slack: float = 0.0
    dc_weight: float = 1.0
    centres: Centres = "midpoint"
    power: float = 2.0
    slack_cost: float = 0.0
    flat_weight: float = 0.1
    flat_levels: int = 0
    flat_dc: int | None = 1


@dataclass(frozen=True, slots=True)
class TV:
    """Total variation's weight (docs/math.md 4.2) and how it takes several channels (4.4)."""

    alpha: float = 1.0
    channel_weights: tuple[float, ...] | None = None
    coupled: bool = True


@dataclass(frozen=True, slots=True)
class TGV:
    """TGV's weights (docs/math.md 4.3): alpha1 of ||grad x - w||, alpha0 of ||E w||."""

    alpha1: float = 1.0
    alpha0: float = 2.0
    channel_weights: tuple[float, ...] | None = None
    coupled: bool = True


@dataclass(frozen=True, slots=True)
class PdhgOptions:
    """The primal-dual method (docs/math.md 5, 6.4-6.6): the most iterations, the stops, the
    steps (their ratio, product and L^2), the relaxation, the records, the free samples' radius."""

    iterations: int | None = None
    tolerance: float | None = None
    relative_tolerance: float = 0.0
    partial_tolerance: float = 0.0
    step_ratio: float | None = None
    relaxation: float | None = None
    step_product: float = 0.99
    norm_squared: float | None = None
    scale_with_weight: bool = True
    record_every: int = 10
    partial_radius: float | None = None
    free_radius: float = 255.0
    threads: int = 0


@dataclass(frozen=True, slots=True)
class SubgradientOptions:
    """The subgradient method of jpeg2png's kind (docs/math.md 7)."""

    iterations: int = 50
    record_every: int = 1
    step: float = 0.5
    decay: float = 0.5
    momentum: bool = True


@dataclass(frozen=True, slots=True)
class Settings:
    """The method ("mmse", "tv", "tgv" or "subgradient"), the data terms (one, or one for each
    component), the models' weights and the solvers' options."""

    method: Method = "tgv"
    data: DataTerm | tuple[DataTerm, ...] = field(default_factory=DataTerm)
    tv: TV = field(default_factory=TV)
    tgv: TGV = field(default_factory=TGV)
    pdhg: PdhgOptions = field(default_factory=PdhgOptions)
    subgradient: SubgradientOptions = field(default_factory=SubgradientOptions)
