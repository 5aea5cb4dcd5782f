"""lima_b200 — B200-native force and integration path for LIMA-style MD.

The product is liblima_b200.so (C-ABI in include/lima_b200.h, CUDA for sm_100a,
sources in lima_b200/csrc/).  ``lima_b200.engine`` is its Python binding and
``lima_b200.systems`` generates seeded synthetic inputs.
"""
from .engine import Engine, LimaError, default_params, load_library  # noqa: F401

__all__ = ["Engine", "LimaError", "default_params", "load_library"]
