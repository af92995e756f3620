"""ctypes binding of libadfdtd.so (the C-ABI declared in include/adfdtd.h).

The library is built in-tree by `build()` (nvcc, sm_100a) into
acoustic_disguising_b200/_lib/libadfdtd.so.  There is no fallback: if the
shared library is missing or no B200 is visible, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libadfdtd.so")
CSRC = os.path.join(HERE, "csrc")

ADF_OK = 0
ERRORS = {-1: "ADF_E_ARG", -2: "ADF_E_NOMEM", -3: "ADF_E_BUDGET", -4: "ADF_E_CANCELLED",
          -5: "ADF_E_DEVICE", -6: "ADF_E_TIMEOUT", -7: "ADF_E_STATE", -8: "ADF_E_NOTFOUND"}
ARITH = {"promote": 0, "fp32": 1}
SHAPES = {"none": 0, "sphere": 1, "cube": 2, "cross": 3, "ellipsoid": 4}


class AdfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def build(jobs: int = 8) -> str:
    """Compile libadfdtd.so for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", CSRC], check=True)
    return LIB_PATH


class Domain(C.Structure):
    """`struct Domain` (src/simulation.jl:25-44); field names as in Julia."""

    _fields_ = [
        ("tmax", C.c_double), ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("nx", C.c_int64), ("ny", C.c_int64), ("nz", C.c_int64),
        ("c0", C.c_double), ("r0", C.c_double), ("cf", C.c_double),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("fact_m0", C.c_double), ("fact_m1", C.c_double),
        ("dt", C.c_double), ("nt", C.c_int64), ("z0", C.c_double),
    ]

    def __repr__(self):
        return (f"Domain(nx={self.nx}, ny={self.ny}, nz={self.nz}, dx={self.dx:.6g}, "
                f"dt={self.dt:.6g}, nt={self.nt})")


class TxGridC(C.Structure):
    _fields_ = [
        ("ntx", C.c_int64), ("nt", C.c_int64),
        ("idx", C.c_void_p * 4), ("w", C.c_void_p * 4),
        ("src", C.c_void_p * 4), ("rec", C.c_void_p * 4),
        ("dir", C.c_void_p), ("vn_src", C.c_void_p), ("vn_rec", C.c_void_p),
    ]


class CpmlC(C.Structure):
    _fields_ = [("npml", C.c_int64), ("mv", C.c_void_p * 3), ("mp", C.c_void_p * 3),
                ("coef", C.c_void_p)]


class GfRequestC(C.Structure):
    _fields_ = [
        ("dom", Domain), ("npml", C.c_int64), ("pml_rcoef", C.c_double), ("pml_fc", C.c_double),
        ("shape", C.c_int), ("shape_params", C.c_double * 6),
        ("src_point", C.c_double * 3), ("src_dir", C.c_double * 4),
        ("src_tf", C.c_void_p), ("n_rec", C.c_int64),
        ("rec_points", C.c_void_p), ("rec_normals", C.c_void_p),
        ("flags", C.c_int), ("out_p", C.c_void_p), ("out_vn", C.c_void_p),
    ]


class KhDescC(C.Structure):
    _fields_ = [
        ("ns", C.c_int64), ("nr", C.c_int64), ("nt", C.c_int64),
        ("dt", C.c_double), ("sigma", C.c_double), ("c0", C.c_double), ("rho", C.c_double),
        ("aq", C.c_double), ("af", C.c_double), ("window_sigmas", C.c_double),
        ("s_pts", C.c_void_p), ("s_nrm", C.c_void_p), ("r_pts", C.c_void_p),
        ("r_nrm", C.c_void_p),
    ]


class GfMapC(C.Structure):
    _fields_ = [("kind", C.c_int), ("nt_gf", C.c_int64), ("n1", C.c_int64), ("n2", C.c_int64),
                ("t", C.c_void_p * 4), ("i_src", C.c_void_p), ("n_src", C.c_int64),
                ("i_rec", C.c_void_p), ("n_rec", C.c_int64), ("z0", C.c_double),
                ("discard", C.c_int), ("contraction", C.c_int)]


GF_KINDS = {"PVFromPin": 0, "PFromPin": 1, "PVFromPV": 2}
GF_CONTRACTIONS = {"fp64": 0, "tf32x3": 1}  # ADF_GF_CONTRACT_*


STEP_CB = C.CFUNCTYPE(C.c_int, C.c_int64, C.c_void_p)

# (name, restype, argtypes) for every entry point of include/adfdtd.h
SIGNATURES = [
    ("adf_version", C.c_int, []),
    ("adf_last_error", C.c_int, [C.c_char_p, C.c_size_t]),
    ("adf_ctx_create", C.c_int, [C.c_int, C.c_size_t, C.POINTER(C.c_void_p)]),
    ("adf_ctx_destroy", C.c_int, [C.c_void_p]),
    ("adf_domain_make", C.c_int, [C.c_double] * 4 + [C.c_int64] * 3 + [C.c_double] * 3
     + [C.POINTER(Domain)]),
    ("adf_coords", C.c_int, [C.POINTER(Domain), C.c_int, C.c_int, C.c_void_p]),
    ("adf_time_axis", C.c_int, [C.POINTER(Domain), C.c_void_p]),
    ("adf_cpml_profiles", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_void_p, C.c_void_p]),
    ("adf_cpml_profiles_static", C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_double, C.c_void_p,
                                           C.c_void_p]),
    ("adf_build_mask", C.c_int, [C.c_void_p, C.POINTER(Domain), C.c_int, C.c_void_p,
                                 C.c_void_p]),
    ("adf_pack_transceivers", C.c_int, [C.POINTER(Domain), C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(TxGridC)]),
    ("adf_run_fdtd", C.c_int, [C.c_void_p, C.POINTER(Domain), C.c_void_p, C.POINTER(TxGridC),
                               C.POINTER(CpmlC), C.c_void_p, C.c_int64, C.c_int64, C.c_int,
                               STEP_CB, C.c_void_p]),
    ("adf_run_fdtd_gf", C.c_int, [C.c_void_p, C.POINTER(Domain), C.c_void_p,
                                  C.POINTER(TxGridC), C.POINTER(CpmlC), C.c_void_p, C.c_int64,
                                  C.c_int64, C.c_int, C.POINTER(GfMapC), STEP_CB, C.c_void_p]),
    ("adf_read_field", C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    ("adf_last_timing", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("adf_set_kernel_timing", C.c_int, [C.c_void_p, C.c_int]),
    ("adf_last_io_bytes", C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("adf_kernel_timing", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64),
                                    C.c_int]),
    ("adf_host_pin", C.c_int, [C.c_void_p, C.c_size_t]),
    ("adf_host_unpin", C.c_int, [C.c_void_p]),
    ("adf_gf_solve_batch", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(GfRequestC), C.c_int]),
    ("adf_autotune", C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                               C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                               C.POINTER(C.c_double)]),
    ("adf_server_start", C.c_int, [C.c_void_p, C.c_size_t, C.c_int, C.POINTER(C.c_void_p)]),
    ("adf_server_submit", C.c_int, [C.c_void_p, C.POINTER(GfRequestC), C.POINTER(C.c_int64)]),
    ("adf_server_poll", C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_int),
                                  C.POINTER(C.c_double)]),
    ("adf_server_cancel", C.c_int, [C.c_void_p, C.c_int64]),
    ("adf_server_set_work_cap", C.c_int, [C.c_void_p, C.c_int64]),
    ("adf_step_resident_ctas", C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    ("adf_server_drain", C.c_int, [C.c_void_p]),
    ("adf_server_stop", C.c_int, [C.c_void_p]),
    ("adf_kh_pressure", C.c_int, [C.c_void_p, C.POINTER(KhDescC), C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    ("adf_kh_velocity", C.c_int, [C.c_void_p, C.POINTER(KhDescC), C.c_void_p, C.c_void_p,
                                  C.c_void_p]),
    ("adf_fp32_fma_peak", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("adf_fp64_fma_peak", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    ("adf_kh_test_fault", C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    ("adf_run_fdtd_kh", C.c_int, [C.c_void_p, C.POINTER(Domain), C.c_void_p,
                                  C.POINTER(TxGridC), C.POINTER(CpmlC), C.c_void_p, C.c_int64,
                                  C.c_int64, C.c_int, C.POINTER(KhDescC), C.c_void_p,
                                  C.c_void_p]),
    ("adf_last_kh_ms", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    ("adf_static_cpml_max_npml", C.c_int, []),
    ("adf_gf_postprocess", C.c_int, [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                     C.c_int64, C.c_double, C.c_double, C.c_void_p, C.c_void_p,
                                     C.c_double, C.c_int]),
    ("adf_injection_coefficients", C.c_int, [C.c_void_p, C.POINTER(Domain), C.c_double,
                                             C.c_int64, C.c_void_p]),
]

_lib = None


def lib():
    """Load libadfdtd.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run acoustic_disguising_b200.build() "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().adf_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> int:
    if rc < 0:
        raise AdfError(rc, f"{what}: {last_error()}")
    return rc
