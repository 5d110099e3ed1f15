"""Import TensorLBM itself from its unmodified install in ``baseline/_ref``.

The reference arm of bench.py and the drop-in tests use this.  TensorLBM's
package ``__init__`` (and a few runners) import matplotlib, and its HDF5 export
imports h5py; neither is installed in this image and no compute path calls
them, so those names resolve to inert stub modules before the import.  Nothing
of the reference is changed.
"""

from __future__ import annotations

import pathlib
import sys
import types

REF_DIR = pathlib.Path(__file__).resolve().parent / "_ref"


class _Stub(types.ModuleType):
    """A module whose every attribute is another stub and which can be called."""

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        if name == "subplots":                   # fig, ax = plt.subplots(...)
            return lambda *a, **k: (_Stub("figure"), _Stub("axes"))
        sub = _Stub(f"{self.__name__}.{name}")
        sys.modules[sub.__name__] = sub
        return sub

    def __call__(self, *a, **k):
        return self

    def __iter__(self):
        return iter(())


def available() -> bool:
    return (REF_DIR / "tensorlbm" / "__init__.py").is_file()


def import_reference():
    """Return the ``tensorlbm`` package from ``baseline/_ref``."""
    if not available():
        raise FileNotFoundError(f"{REF_DIR} holds no tensorlbm install")
    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.colors", "h5py"):
        try:
            __import__(name)
        except ImportError:
            sys.modules[name] = _Stub(name)
    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    import tensorlbm

    if not str(pathlib.Path(tensorlbm.__file__).resolve()).startswith(str(REF_DIR.resolve())):
        raise ImportError(f"tensorlbm resolved to {tensorlbm.__file__}, not the install in {REF_DIR}")
    return tensorlbm
