"""Global configuration: the device singleton and the debug verbosity levels
(paces/config/__init__.py)."""

from .dbg_verbosity_levels import *  # noqa: F401,F403
from ._dev_conf import DeviceConfig

# Unconfigured until the driver calls devices.configure() (paces/config/__init__.py:9).
devices = DeviceConfig()
