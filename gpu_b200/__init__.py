"""B200-native cone-beam CT reconstruction engine (Siddon FP, matched gather
BP, SART + FISTA + FGP-TV, FDK) behind the C ABI of ``include/ctrecon.h``.

Importing the package loads the in-tree ``libctrecon.so`` and raises
ImportError when it has not been built: there is no CPU fallback.
"""
from .ctrecon import (  # noqa: F401
    BF16, BP_ACCUMULATE, BP_FOV_MASK, EXPORTED, F16, F32, F64, GEOM_ENTRY_F64, GEOM_FAN_SLICES, GEOM_FAST_SUMS,
    GEOM_PARALLEL, GEOM_TBCT, LIB_PATH,
    SART_REFERENCE_BP, SART_STOCHASTIC_ROUND, SART_TILED, VOLUME_TILED, Batch, CtrError, Geometry, GeometryDesc, Solver, SolverParams,
    check_matched_joint_operator, convert, dtype_code, fgp_denoise_gpux7_exact, forward_3d_ray_driven_siddon,
    l2_norm, l2_norm_gpu, last_error, load_library, make_desc, reconstruction_3d_ray_driven_cbct,
    reconstruction_fdk, set_default_devices, set_default_geometry, tv_norm_gpu,
)

load_library()
