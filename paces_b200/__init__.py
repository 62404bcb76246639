"""paces_b200: the adaptive-basis time step of paces (Parallelized Application of
Co-Evolving Subspaces) on B200.

The hot path -- truncation, enlargement, sort/unique, Hamiltonian assembly, the Taylor
series of exp(-i dt H) and the observables -- runs in libpaces_b200.so (sm_100a CUDA,
C ABI in include/paces_b200.h).  The subpackages mirror the reference's module layout
(config, core, models, aux) so that driver scripts written for it run unchanged; the
top-level package `paces` re-exports this one under the reference's name.
"""

__all__ = ["aux", "core", "models", "config"]
__version__ = "1.2.0"

from . import config, core, models, aux  # noqa: E402,F401
