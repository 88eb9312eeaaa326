"""ymgpu -- host mirror of the reference's lattice gauge API over libymgpu.

The reference (QSOLKCB/YANG-MILLS) exposes its hot path as Rust module
functions (``su3_ensemble``, ``su2_ensemble``, ``su3_lattice``, ...).  This
package keeps those module and function names and calls the B200 engine
through its C ABI (``include/ymgpu.h``).  There is no CPU fallback: importing
a compute entry point without the built ``libymgpu.so`` raises.
"""
from ._lib import LIB_PATH, lib
from .ensemble import Ensemble, F32_TWO_ROW, F64, ORDERED, SU2, SU3, UNIFORM
from .errors import YmError
from . import glueball, learned, path_holonomy, su2_ensemble, su3_ensemble, su3_lattice
from .learned import ProposalModel
from .lattice import Lattice4
from .su3_lattice import Su3Lattice4


def release_pooled_memory(device: int = 0) -> None:
    """Give the device memory that destroyed handles left in the device's
    memory pool back to the driver (ym_device_release_pooled_memory)."""
    from .errors import check
    check(lib().ym_device_release_pooled_memory(int(device)), "release_pooled_memory")


__all__ = ["Ensemble", "Lattice4", "Su3Lattice4", "path_holonomy", "YmError", "lib", "LIB_PATH", "su2_ensemble",
           "su3_ensemble", "su3_lattice", "glueball", "SU2", "SU3", "F64", "F32_TWO_ROW", "ORDERED",
           "UNIFORM", "learned", "ProposalModel", "release_pooled_memory"]
