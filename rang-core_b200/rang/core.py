"""Access to the compiled extension (the reference's `rang.core` role for
the gridder: `extension()` and `library_path()`)."""

import importlib
from pathlib import Path

_EXT = None


def extension():
    """The extension module `rang._core`. There is no fallback: a missing or
    unbuilt extension raises ImportError (build it with
    `python rang-core_b200/build.py`)."""
    global _EXT
    if _EXT is None:
        _EXT = importlib.import_module("rang._core")
    return _EXT


def library_path():
    """The CUDA library the gridder runs in."""
    return str(Path(__file__).with_name("librang_wgrid_b200.so"))
