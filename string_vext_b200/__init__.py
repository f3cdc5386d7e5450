"""vext_b200: B200 (sm_100a) engine for the exact two-identical-site
Lennard-Jones guest energy in a full triclinic periodic cell -- Vext fields
over (grid center x director) and String-path poses with their analytic
adjoint.  Compute lives in ``lib/libvext_b200.so`` (C ABI:
include/vext_b200.h); this package holds the host-side mirror of the
reference's Python interface (``calculate_vext``, ``parse_string_input``,
``regular_pose_grid``, ``cell_matrix``).  The reference's own CSR driver
(``NativeReusePotential``) binds the library's ``evaluate_reused_neighbors``
unchanged, so it needs no counterpart here.
"""

__version__ = "0.1.0"

from .cell import cell_matrix  # noqa: F401
from .input import parse_string_input  # noqa: F401
from .orientation import regular_pose_grid  # noqa: F401
