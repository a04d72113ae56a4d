"""Import shim for the reference package (quantem 0.1.8).

The reference's ptychography modules import plotting / IO / hyper-parameter
packages at module import time (matplotlib, zarr, h5py, optuna, skimage, ...)
that are absent from this image, although the ptychography iteration never
calls them.  ``import_reference(path)`` installs permissive stand-in modules
for exactly those names, patches ``importlib.metadata.version("quantem")`` and
puts ``path`` (a directory holding the ``quantem`` package: the reference's
``src`` or the ``baseline/_ref`` install) first on ``sys.path``.

Users: the golden-fixture generators under ``tests/golden/`` and the timing of
the reference's own PyTorch iteration in ``bench.py``.  Nothing in the product
package imports it.
"""
from __future__ import annotations

import importlib
import importlib.metadata
import sys
import types

_STUB_ROOTS = (
    "matplotlib", "mpl_toolkits", "colorspacious", "cmasher", "skimage", "optuna",
    "zarr", "h5py", "hdf5plugin", "rsciio", "torchinfo", "torchmetrics", "tensorboard",
)


class _Anything:
    """Object that absorbs attribute access, calls, indexing and subclassing."""

    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Anything()

    def __getattr__(self, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        return _Anything()

    def __getitem__(self, k):
        return _Anything()

    def __setitem__(self, k, v):
        pass

    def __iter__(self):
        return iter(())

    def __mro_entries__(self, bases):
        return (_AnythingClass,)

    def _absorb(self, *a, **k):
        return self

    __mul__ = __rmul__ = __imul__ = __add__ = __radd__ = __iadd__ = _absorb
    __sub__ = __rsub__ = __isub__ = __truediv__ = __rtruediv__ = __itruediv__ = _absorb
    __neg__ = __pow__ = __or__ = __ror__ = _absorb

    def __len__(self):
        return 0

    def __bool__(self):
        return False


class _AnythingMeta(type):
    def __getattr__(cls, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        return _Anything()


class _AnythingClass(metaclass=_AnythingMeta):
    def __init__(self, *a, **k):
        pass

    def __call__(self, *a, **k):
        return _Anything()

    def __getattr__(self, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        return _Anything()


class _StubModule(types.ModuleType):
    def __init__(self, name):
        super().__init__(name)
        self.__path__ = []  # behave like a package so submodule imports resolve

    def __getattr__(self, name):
        if name.startswith("__") and name.endswith("__"):
            raise AttributeError(name)
        full = f"{self.__name__}.{name}"
        if full in sys.modules:
            return sys.modules[full]
        # Capitalised names are used as base classes (e.g. colors.Normalize).
        if name[:1].isupper():
            cls = _AnythingMeta(name, (_AnythingClass,), {})
            setattr(self, name, cls)
            return cls
        # lower-case names may be submodules (``from matplotlib import colors``)
        # or functions; a callable stub module serves both uses.
        sub = _StubModule(full)
        sys.modules[full] = sub
        setattr(self, name, sub)
        return sub

    def __call__(self, *a, **k):
        return _Anything()

    def __getitem__(self, k):
        return _Anything()


class _StubFinder:
    """Meta-path finder that materialises any submodule of a stubbed root."""

    def find_spec(self, fullname, path, target=None):
        root = fullname.split(".")[0]
        if root not in _STUB_ROOTS:
            return None
        from importlib.machinery import ModuleSpec

        return ModuleSpec(fullname, self, is_package=True)

    def create_module(self, spec):
        return _StubModule(spec.name)

    def exec_module(self, module):
        pass


def import_reference(src_path: str):
    """Import the reference ``quantem`` package from ``src_path`` with stubs."""
    for name in list(sys.modules):
        if name.split(".")[0] in _STUB_ROOTS and not isinstance(sys.modules[name], _StubModule):
            # a real installation would win; nothing to stub
            pass
    if not any(isinstance(f, _StubFinder) for f in sys.meta_path):
        sys.meta_path.insert(0, _StubFinder())
    _orig_version = importlib.metadata.version

    def _version(dist):
        if dist == "quantem":
            return "0.1.8"
        return _orig_version(dist)

    importlib.metadata.version = _version
    # torch.utils.tensorboard refuses to import without the tensorboard package;
    # the reference's logger imports its SummaryWriter at module level only.
    for name in ("torch.utils.tensorboard", "torch.utils.tensorboard.writer"):
        sys.modules.setdefault(name, _StubModule(name))
    if src_path not in sys.path:
        sys.path.insert(0, src_path)
    return importlib.import_module("quantem")
