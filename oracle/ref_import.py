"""Import the reference dpnegf hot path in a container without its heavy deps.

TEST INFRASTRUCTURE ONLY.  Used by ``tests/golden/make_golden.py`` to run the
reference's own functions and write golden fixtures.  Nothing in the product
package imports this module, and it needs the reference source tree on disk
(it is absent on machines that only run the GPU tests).

The reference package ``__init__`` calls ``importlib.metadata.version("dpnegf")``
(dpnegf/__init__.py:4), which fails when dpnegf is not pip-installed, and the
hot-path modules import ``ase``, ``xitorch``, ``matplotlib``, ``h5py``, ``dptb``
and ``pyinstrument`` at module level even though the functions used here never
touch them.  We therefore (1) register ``dpnegf``, ``dpnegf.negf`` and
``dpnegf.utils`` as bare namespace packages pointing at the source tree, and
(2) install a meta-path finder that serves inert stub modules for the absent
third-party packages.
"""
import importlib.abc
import importlib.machinery
import os
import sys
import types
from unittest import mock

# Where the reference source tree lies: no default; pass it, or set DPNEGF_REF_ROOT.
ENV_REF_ROOT = "DPNEGF_REF_ROOT"
_STUBBED = ("ase", "xitorch", "matplotlib", "h5py", "dptb", "pyinstrument")


class _StubModule(types.ModuleType):
    def __init__(self, name):
        super().__init__(name)
        self.__path__ = []  # behaves as a package so submodule imports resolve

    def __getattr__(self, item):
        if item.startswith("__"):
            raise AttributeError(item)
        val = mock.MagicMock(name=f"{self.__name__}.{item}")
        setattr(self, item, val)
        return val


class _StubLoader(importlib.abc.Loader):
    def create_module(self, spec):
        return _StubModule(spec.name)

    def exec_module(self, module):
        return None


class _StubFinder(importlib.abc.MetaPathFinder):
    def find_spec(self, fullname, path=None, target=None):
        root = fullname.split(".")[0]
        if root in _STUBBED:
            return importlib.machinery.ModuleSpec(fullname, _StubLoader(), is_package=True)
        return None


def ref_root_from_env():
    """The reference source root named by ``DPNEGF_REF_ROOT``, or None."""
    return os.environ.get(ENV_REF_ROOT) or None


def install(ref_root: str):
    """Make ``import dpnegf.negf.<module>`` resolve to the reference sources at ``ref_root``."""
    if not ref_root:
        raise ValueError(f"the reference source root is required (argument, or {ENV_REF_ROOT})")
    pkg_root = os.path.join(ref_root, "dpnegf")
    if not os.path.isdir(pkg_root):
        raise FileNotFoundError(f"reference source tree not found at {pkg_root}")
    if not any(isinstance(f, _StubFinder) for f in sys.meta_path):
        sys.meta_path.insert(0, _StubFinder())
    for name, sub in (("dpnegf", ""), ("dpnegf.negf", "negf"), ("dpnegf.utils", "utils")):
        if name in sys.modules:
            continue
        mod = types.ModuleType(name)
        mod.__path__ = [os.path.join(pkg_root, sub) if sub else pkg_root]
        sys.modules[name] = mod
    return True


def load(module: str, ref_root: str):
    """``load("recursive_green_cal")`` -> the reference module object."""
    install(ref_root)
    return importlib.import_module(f"dpnegf.negf.{module}")
