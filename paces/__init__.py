"""`paces`: the reference's package name for paces_b200.

Driver scripts written for rkevk/paces import `paces.config`, `paces.core.*`,
`paces.models.holstein` and `paces.aux`; this package maps those module paths onto the
paces_b200 modules (the same module objects, so singletons such as
`paces.config.devices` are shared).
"""

import importlib
import sys

import paces_b200 as _impl

__all__ = ["aux", "core", "models", "config"]
__version__ = _impl.__version__

_SUBMODULES = (
    "config", "config.dbg_verbosity_levels", "config._dev_conf",
    "core", "core.hamiltonian", "core.observables", "core.time_evolution",
    "models", "models.holstein",
    "aux", "aux.helpers", "aux.cupy_search",
)
for _name in _SUBMODULES:
    sys.modules[f"{__name__}.{_name}"] = importlib.import_module(f"paces_b200.{_name}")

config = _impl.config
core = _impl.core
models = _impl.models
aux = _impl.aux
