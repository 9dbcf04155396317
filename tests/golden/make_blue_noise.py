"""Writes tests/golden/blue_noise_ranks.npy: the reference's blue-noise matrix of the ordered
dither (64 x 64 ranks, row by row), made by running the reference's own generator
(scripts/blue_noise.py of JPEG-Unround, its matrix()) where the reference checkout lies. The
tests compare the library's own void-and-cluster ranks with it, and read only the .npy.

Run: python tests/golden/make_blue_noise.py <path to the reference checkout>
(or with the environment variable UNROUND_REFERENCE naming it)
"""

from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main() -> None:
    named = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("UNROUND_REFERENCE")
    if not named:
        raise SystemExit("name the reference checkout: make_blue_noise.py <path>, or UNROUND_REFERENCE=<path>")
    reference = Path(named)
    # Its annotations name its own class before the class is made (evaluated lazily by newer
    # Pythons): run its source with postponed annotations.
    path = reference / "scripts" / "blue_noise.py"
    module = types.ModuleType("reference_blue_noise")
    module.__file__ = str(path)
    sys.modules[module.__name__] = module
    source = "from __future__ import annotations\n" + path.read_text(encoding="utf-8")
    exec(compile(source, str(path), "exec"), module.__dict__)  # noqa: S102 -- the reference's generator
    ranks = np.asarray(module.matrix(), dtype=np.uint16).reshape(64, 64)
    assert sorted(ranks.ravel().tolist()) == list(range(4096))
    np.save(HERE / "blue_noise_ranks.npy", ranks)
    print("wrote", HERE / "blue_noise_ranks.npy")


if __name__ == "__main__":
    main()
