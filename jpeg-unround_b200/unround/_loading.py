"""Where the package's shared library is: the path in an environment variable, or unround/_native.

The same lookup as the reference package's (python/src/unround/_loading.py of JPEG-Unround):
UNROUND_LIBRARY names the C-interface library; otherwise the one in unround/_native, where
jpeg-unround_b200/build.py writes this build's libunround_capi.so.
"""

import os
import sys
from pathlib import Path
from typing import Final

__all__ = ["C_LAYER", "RUST", "bundled", "configured", "file_name"]

C_LAYER: Final = "unround_jpegio"
"""The reference's C layer over libjpeg-turbo and libpng, which this build does not carry."""

RUST: Final = "unround_capi"
"""The C interface (unround.h): the reference's Rust library, or this build's B200 one."""

_AFFIXES: Final = {"win32": ("", ".dll"), "darwin": ("lib", ".dylib")}


def file_name(stem: str) -> str:
    """The file name of the shared library of the stem on this system."""
    prefix, suffix = _AFFIXES.get(sys.platform, ("lib", ".so"))
    return f"{prefix}{stem}{suffix}"


def configured(variable: str) -> Path | None:
    """The path in the environment variable, where it is set."""
    value = os.environ.get(variable)
    return Path(value) if value else None


def bundled(stem: str) -> Path | None:
    """The package's own library of the stem, where it is built."""
    path = Path(__file__).parent / "_native" / file_name(stem)
    return path if path.is_file() else None
