"""B200 implementation of OpenQG's per-timestep quasi-geostrophic core."""
from .params import Basin, OqgParams, ocean_double_gyre, atmos_channel  # noqa: F401
