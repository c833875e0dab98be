"""B200-native implicit edge-based finite-volume hot path (Euler3D-compatible).

The compute path is the CUDA library ``_lib/libcfd_b200.so`` (sm_100a), bound
through its C ABI (``include/cfd_b200.h``).  Importing the package loads the
library and fails loudly if it is missing.
"""
from . import _capi as capi  # noqa: F401  (loads the library)
from .mesh import Mesh, box_mesh, from_cells, perturbed_freestream, to_conservative, to_rup  # noqa: F401
from .solver import Euler3DGPU, default_params  # noqa: F401

__all__ = ["capi", "Mesh", "box_mesh", "from_cells", "perturbed_freestream", "to_rup", "to_conservative", "Euler3DGPU", "default_params"]
