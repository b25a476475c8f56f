"""parcel_b -- host-side Python mirror of PARCEL-legacy's Krylov solver API on top of the
B200 library libparcelb.so (C-ABI declared in include/parcel_b.h)."""
from . import problems  # noqa: F401
from ._lib import load, last_error, last_stats, new_input  # noqa: F401
from .api import (parcel_dbicgstab, parcel_dcagmres, parcel_dcg, parcel_dgmres,  # noqa: F401
                  solve)
