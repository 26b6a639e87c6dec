"""Loaders for the reference's own CPU code. TEST INFRASTRUCTURE ONLY.

Two uses:

1. ``load(name)`` returns one of the reference's Cython kernel modules (``em``,
   ``tools``, ``sqp``, ``bvls``, ``br_qn``, ``snp_reader``, ``clumppling``) compiled
   by ``oracle/Makefile`` into ``oracle/_ref/``. These travel with the repository
   snapshot and serve as the timed CPU baseline (the reference's ``adamStep``,
   ``adamixture/model/em_adam.py:12-54``, is ``em.P_step`` + ``em.Q_step`` +
   ``em.adamUpdateP/Q``).

2. ``import_reference()`` imports the reference's Python package itself from its
   read-only source tree (only where that tree exists, i.e. when fixtures are
   regenerated). Its compiled submodules are served from ``oracle/_ref/``;
   modules it needs that are not installed here (``matplotlib``,
   ``configargparse``, the build-generated ``_version``) are stubbed.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import sysconfig
import types
from pathlib import Path

REF_DIR = Path(__file__).resolve().parent / "_ref"
# The reference project tree: ADX_REFERENCE_TREE when set, else a sibling directory named
# "reference" beside this repository's root.
REFERENCE_TREE = Path(os.environ.get("ADX_REFERENCE_TREE",
                                     Path(__file__).resolve().parent.parent.parent / "reference"))
MODULES = ("em", "tools", "sqp", "bvls", "br_qn", "snp_reader", "clumppling")

_loaded: dict[str, types.ModuleType] = {}


def available() -> bool:
    """True when every compiled reference module is present in ``oracle/_ref/``."""
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    return all((REF_DIR / f"{m}{ext}").exists() for m in MODULES)


def load(name: str, fullname: str | None = None) -> types.ModuleType:
    """Load the compiled reference module ``name`` from ``oracle/_ref/``.

    ``fullname`` registers it under a package path (its last component must equal
    ``name`` because the module's init symbol is ``PyInit_<name>``).
    """
    key = fullname or f"adx_ref_{name}"
    if key in _loaded:
        return _loaded[key]
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    path = REF_DIR / f"{name}{ext}"
    if not path.exists():
        raise FileNotFoundError(
            f"{path} is missing: build it with `make -C oracle` in a tree that has the reference sources"
        )
    spec_name = fullname or name
    spec = importlib.util.spec_from_file_location(spec_name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    _loaded[key] = mod
    if fullname:
        sys.modules[fullname] = mod
    return mod


def _stub(name: str, **attrs) -> None:
    if name in sys.modules:
        return
    mod = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(mod, k, v)
    sys.modules[name] = mod


def import_reference():
    """Import the reference Python package ``adamixture`` from its source tree.

    Sets ``TORCHDYNAMO_DISABLE=1`` so its ``torch.compile`` wrappers run eagerly on
    the CPU (the reference GPU path then runs as float64 torch code on the host).
    Returns the top-level package.
    """
    if not (REFERENCE_TREE / "adamixture").is_dir():
        raise FileNotFoundError(f"reference tree not found at {REFERENCE_TREE}")
    os.environ.setdefault("TORCHDYNAMO_DISABLE", "1")
    _stub("adamixture._version", __version__="0", __version_tuple__=(0,))

    import torch  # noqa: F401  (import before the stubs exist)

    class _Anything(types.ModuleType):
        def __getattr__(self, item):  # plotting is never called by the fixtures
            if item.startswith("__"):
                raise AttributeError(item)
            return lambda *a, **k: None

    for name in ("matplotlib", "matplotlib.pyplot", "matplotlib.colors",
                 "matplotlib.patches", "matplotlib.ticker", "configargparse"):
        if name not in sys.modules:
            sys.modules[name] = _Anything(name)
    for m in MODULES:
        load(m, fullname=f"adamixture.src.utils_c.cython.{m}")
    if str(REFERENCE_TREE) not in sys.path:
        sys.path.insert(0, str(REFERENCE_TREE))
    import adamixture  # noqa: E402

    return adamixture
