"""B200-native exterior Burton-Miller direct-system solver (drop-in for the
``burton_miller_assembly`` path of BEAT Engine's exterior solve)."""
from .mesh import (BoundaryMesh, arc_points, equator_meridian_directions, fibonacci_sphere,  # noqa: F401
                   load_gmsh22_with_tags, oscillating_sphere, reference_sphere, write_gmsh22)
from .phasor import (NEGATIVE_TIME_PHASOR, POSITIVE_TIME_PHASOR, burton_miller_coupling,  # noqa: F401
                     neumann_scale, outgoing_wavenumber, propagation_sign)

__version__ = "0.1.0"


def library_path() -> str:
    from ._lib import LIB_PATH
    return LIB_PATH
