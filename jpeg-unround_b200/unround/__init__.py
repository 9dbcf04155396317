"""JPEG reconstruction within the quantization intervals, on a B200.

The drop-in for the reference package unround (python/src/unround of JPEG-Unround): the same
modules and names -- settings, native (solve, options, Decoded, UnroundError ...), jpegio
(Image, Component) -- over the same C interface (include/unround.h), whose library here runs
the TV/TGV primal-dual solve as CUDA kernels on the GPU. Files are read on the host by this
build's own JPEG and PNG readers (jpegio.read, native.decode), whose coefficients and levels
go to the same solve; levels and tables given as arrays (jpegio.image_of) go to native.solve.
synthetic makes seeded test pictures and their levels; native.solve_batch solves many pictures
at once; unrolled differentiates an unrolled TGV solve with torch; strips solves one picture in
row strips across ranks.
"""

from unround import jpegio, native, settings
from unround.jpegio import read
from unround.native import Decoded, Record, UnroundError, UnroundWarning, decode, project, solve, to_rgb, to_ycbcr
from unround.settings import TGV, TV, DataTerm, PdhgOptions, Settings, SubgradientOptions

__all__ = [
    "TGV",
    "TV",
    "DataTerm",
    "Decoded",
    "PdhgOptions",
    "Record",
    "Settings",
    "SubgradientOptions",
    "UnroundError",
    "UnroundWarning",
    "decode",
    "jpegio",
    "native",
    "project",
    "read",
    "settings",
    "solve",
    "to_rgb",
    "to_ycbcr",
]
__version__ = "0.1.0"
