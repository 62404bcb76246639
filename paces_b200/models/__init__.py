"""Models (paces/models/__init__.py): the single-exciton Holstein chain."""

__all__ = ["holstein"]

from . import holstein  # noqa: F401
