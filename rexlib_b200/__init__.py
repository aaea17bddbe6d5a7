"""rexlib_b200: a B200 (sm_100a) backend for rexlib's em reconstruction path.

``rexlib_b200.em`` mirrors rexlib's ``em`` functional API over the C-ABI of
``librexlib_b200.so`` (declared in ``include/rexlib_b200.h``). The library is
built in-tree by :func:`build`; importing a function that needs it raises if
it is missing, since no host fallback exists.
"""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))

__all__ = ["build", "em", "library_path"]


def library_path() -> str:
    return os.path.join(HERE, "_lib", "librexlib_b200.so")


def build(jobs: int | None = None) -> str:
    """Compile every CUDA source for sm_100a into rexlib_b200/_lib."""
    jobs = jobs or max(1, os.cpu_count() or 1)
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", os.path.join(HERE, "csrc")], check=True)
    return library_path()


def __getattr__(name):
    if name == "em":
        import importlib

        return importlib.import_module(".em", __name__)
    raise AttributeError(name)
