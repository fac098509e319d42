"""miniqmc_b200: B200-native VMC walker hot path of QMCPACK/miniqmc."""
from . import capi  # noqa: F401
