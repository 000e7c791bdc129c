"""B200 (sm_100a) ePlace global-placement engine: the density / Poisson / gather / WA /
Nesterov iteration of superPlace, device-resident behind a C ABI (include/spgpu.h)."""
from . import abi
from .placedb import PlaceDB, make_db

__all__ = ["abi", "PlaceDB", "make_db"]
