"""Core framework classes (paces/core/__init__.py)."""

from . import hamiltonian, observables, time_evolution  # noqa: F401
