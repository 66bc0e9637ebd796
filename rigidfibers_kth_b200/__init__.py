"""B200-native rigid-fiber slender-body solver.

The method of ericwolter/rigidfibers_kth (Legendre force expansion, analytic
or Gauss-quadrature pair integrals, dense assembly, restarted GMRES, velocity
recovery, multistep advection) behind the reference's step API, computed by
hand-written sm_100a CUDA kernels in librigidfibers.so (C ABI:
include/rigidfibers.h).
"""
from ._lib import (  # noqa: F401
    PC_CLUSTER,
    PC_LEARNED,
    PC_NONE,
    PREC_FP32,
    PREC_FP64,
    PREC_MIXED_BF16,
    PREC_MIXED_FP32,
    VEL_RECOMPUTE,
    VEL_REUSE,
    RfError,
    build,
    lib,
)
from .simulation import (  # noqa: F401
    Configuration,
    FiberParams,
    Simulation,
    generate_layout,
    min_segment_distance,
    parse_configuration_files,
    parse_layout_file,
    parse_parameter_file,
    shard_range,
    shard_unique_id,
    write_layout_file,
)
