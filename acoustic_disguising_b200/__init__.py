"""B200-native FDTD + Kirchhoff-Helmholtz hot path of AcousticDisguising.

The compute lives in libadfdtd.so (CUDA for sm_100a, C-ABI in
include/adfdtd.h); this package is its Python mirror of the reference API.
"""
from ._lib import AdfError, build, lib, last_error, LIB_PATH  # noqa: F401
from .api import (  # noqa: F401
    Context, default_context, Domain, coord, coords, t, fibonacci_sphere, impulsive_wavelet,
    ricker_wavelet, fib_sphere_area, cpml_profiles, cpml_profiles_static, static_cpml_max_npml,
    split_profiles, Cpml, shape_params,
    build_update_mask, Transceiver, TransceiverGrid, transceivers_to_grid, p_src, p_rec, vn_src,
    vn_rec, run_fdtd, run_fdtd_kh, GfMap, PVFromPin, PFromPin, PVFromPV, injection_coefficients, kh_pressure, kh_velocity, kh_test_fault, gf_postprocess, gf_unit_factors, fp32_fma_peak, fp64_fma_peak, GfRequest,
    gf_solve_batch, impulsive_gfs, autotune, Server, pinned_zeros,
)

__all__ = [n for n in dir() if not n.startswith("_")]
