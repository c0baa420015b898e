"""ctypes binding of libzb (the C ABI declared in include/zb.h).

The host package never computes on the CPU: every public solver call goes
through this library on a CUDA device, and importing a solver without the
built library or without a GPU raises instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import math
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent.parent / "lib" / "libzb.so"

ZB_F32, ZB_F64 = 0, 1
ZB_OK, ZB_E_ARG, ZB_E_CUDA, ZB_E_UNSUPPORTED, ZB_E_TOO_LARGE = 0, -1, -2, -3, -4
ZB_E_NOT_CONVERGED = -5
ZB_NOALLOC_MAX_CELLS = 1 << 20
ZB_ST_DT_INVALID, ZB_ST_TROUBLED, ZB_ST_NOT_CONVERGED = 1, 2, 4
BC = {"extrapolation": 0, "wall": 1, "periodic": 2}
RECON = {"constant": 0, "conservative": 1, "eta": 2}
RIEMANN = {"rusanov": 0, "rusanov_hr": 1, "hll_hr": 2}
LIMITER = {"minmod": 0, "barth_jespersen": 1, "venkatakrishnan": 2, "none": 3}


class ZbCtrl(C.Structure):
    _fields_ = [("amax", C.c_double * 3), ("t", C.c_double * 3),
                ("dt", C.c_double), ("mass", C.c_double),
                ("status", C.c_uint32), ("steps", C.c_uint32),
                ("troubled", C.c_uint32), ("pad", C.c_uint32),
                ("reserved", C.c_double * 6)]


CTRL_BYTES = C.sizeof(ZbCtrl)


class ZbSwe2dCfg(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32),
                ("x0", C.c_double), ("y0", C.c_double),
                ("dx", C.c_double), ("dy", C.c_double),
                ("order", C.c_int32), ("recon", C.c_int32),
                ("riemann", C.c_int32), ("limiter", C.c_int32),
                ("bc", C.c_int32 * 4),
                ("g", C.c_double), ("wet_dry_eps", C.c_double),
                ("eps_wet", C.c_double), ("manning_n", C.c_double),
                ("implicit_source", C.c_int32), ("dim_factor", C.c_int32),
                ("cfl", C.c_double), ("dt_max", C.c_double),
                ("t_end", C.c_double), ("degree", C.c_int32),
                ("dtype", C.c_int32), ("bed", C.c_void_p)]


class ZbTriCfg(C.Structure):
    _fields_ = [("order", C.c_int32), ("recon", C.c_int32), ("riemann", C.c_int32),
                ("limiter", C.c_int32), ("g", C.c_double), ("wet_dry_eps", C.c_double),
                ("eps_wet", C.c_double), ("manning_n", C.c_double),
                ("implicit_source", C.c_int32), ("dim_factor", C.c_int32),
                ("cfl", C.c_double), ("dt_max", C.c_double), ("t_end", C.c_double),
                ("degree", C.c_int32), ("dtype", C.c_int32)]


class ZbEnsInstance(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
                ("q_offset", C.c_int64), ("ws_offset", C.c_int64),
                ("manning_n", C.c_double), ("t_end", C.c_double)]


class ZbEnsTuning(C.Structure):
    _fields_ = [("tile_x", C.c_int32), ("ctas_per_sm", C.c_int32), ("n_classes", C.c_int32),
                ("class_max_side", C.c_int32 * 4), ("edge_rows", C.c_int32 * 4),
                ("interior_rows", C.c_int32 * 4)]


class ZbPoissonCfg(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double),
                ("cmin", C.c_double), ("cmax", C.c_double), ("nu", C.c_int32),
                ("coarse_sweeps", C.c_int32), ("coarsest", C.c_int32)]


class ZbSmoother(C.Structure):
    _fields_ = [("c1", C.c_int32), ("c2", C.c_int32), ("w", C.c_void_p),
                ("b", C.c_void_p), ("cmax", C.c_float), ("act", C.c_void_p),
                ("act_bytes", C.c_size_t), ("max_nx", C.c_int32), ("max_ny", C.c_int32)]


class ZbUnetTrainer(C.Structure):
    _fields_ = [("c1", C.c_int32), ("c2", C.c_int32), ("batch", C.c_int32), ("n", C.c_int32),
                ("cmax", C.c_float),
                ("w_master", C.c_void_p), ("b_master", C.c_void_p),
                ("m_w", C.c_void_p), ("v_w", C.c_void_p), ("m_b", C.c_void_p),
                ("v_b", C.c_void_p), ("g_w", C.c_void_p), ("g_b", C.c_void_p),
                ("w_bf16", C.c_void_p), ("b_shadow", C.c_void_p), ("act", C.c_void_p)]


PRECOND = {"none": 0, "mg": 1, "learned": 2, "learned_replace": 3}
# scalar slots of the Poisson workspace (float64)
S_REL, S_ITER = 7, 8

TRI_MESH_FIELDS = ["lsq_idx", "lsq_wx", "lsq_wy", "cf_rx", "cf_ry", "cell_face",
                   "cell_inv_area", "face_a", "face_b", "face_nx", "face_ny", "face_len",
                   "face_rax", "face_ray", "face_rbx", "face_rby", "face_inr", "bf_kind",
                   "bf_nx", "bf_ny"]


class ZbTriMesh(C.Structure):
    _fields_ = ([("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_bf", C.c_int32)]
                + [(n, C.c_void_p) for n in TRI_MESH_FIELDS])


# (name, restype, argtypes) of every symbol include/zb.h declares
_P = C.c_void_p
_CFG = C.POINTER(ZbSwe2dCfg)
_TCFG = C.POINTER(ZbTriCfg)
_TMESH = C.POINTER(ZbTriMesh)
_PCFG = C.POINTER(ZbPoissonCfg)
_SMO = C.POINTER(ZbSmoother)
_TRN = C.POINTER(ZbUnetTrainer)
SIGNATURES = [
    ("zb_version", C.c_char_p, []),
    ("zb_swe2d_workspace_bytes", C.c_size_t, [_CFG]),
    ("zb_swe2d_init", C.c_int, [_CFG, _P, _P, C.c_int, C.c_double, _P]),
    ("zb_swe2d_dt", C.c_int, [_CFG, _P, _P, C.c_double, _P]),
    ("zb_swe2d_step", C.c_int, [_CFG, _P, _P, C.c_size_t, _P, C.c_int, _P]),
    ("zb_swe2d_bed_bytes", C.c_size_t, [_CFG]),
    ("zb_swe2d_bed_prepare", C.c_int, [_CFG, _P, _P, C.c_size_t, _P]),
    ("zb_swe2d_step_part", C.c_int, [_CFG, _P, _P, C.c_size_t, _P, C.c_int, C.c_int, _P]),
    ("zb_swe2d_step_noalloc", C.c_int, [_CFG, _P, _P, C.c_int, _P]),
    ("zb_swe2d_stage", C.c_int, [_CFG, _P, _P, _P, C.c_double, C.c_double,
                                 C.c_double, _P, _P, _P, _P, _P]),
    ("zb_swe2d_source", C.c_int, [_CFG, _P, _P, C.c_double, _P]),
    ("zb_swe2d_mass_partials", C.c_size_t, [_CFG]),
    ("zb_swe2d_mass", C.c_int, [_CFG, _P, _P, _P, _P]),
    ("zb_swe2d_aux", C.c_int, [_CFG, _P, _P, _P]),
    ("zb_newton_check_f64", C.c_int, [_P, _P, _P, C.c_int64, _P]),
    ("zb_ens_table_bytes", C.c_size_t, [_CFG, _P, C.c_int, C.c_int]),
    ("zb_ens_prepare", C.c_int, [_CFG, _P, C.c_int, C.c_int, _P, C.c_size_t,
                                 C.POINTER(C.c_int)]),
    ("zb_ens_table_bytes_tuned", C.c_size_t, [_CFG, _P, C.c_int, C.POINTER(ZbEnsTuning)]),
    ("zb_ens_prepare_tuned", C.c_int, [_CFG, _P, C.c_int, C.POINTER(ZbEnsTuning), _P,
                                       C.c_size_t, C.POINTER(C.c_int)]),
    ("zb_ens_step_part_tuned", C.c_int, [_CFG, _P, C.c_int, C.c_int, C.POINTER(ZbEnsTuning),
                                         C.c_int, _P, _P, _P, C.c_int, C.c_int, _P]),
    ("zb_ens_init", C.c_int, [_CFG, _P, C.c_int, _P, _P, C.c_int, C.c_double, _P]),
    ("zb_ens_step_part", C.c_int, [_CFG, _P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P,
                                   _P, C.c_int, C.c_int, _P]),
    ("zb_tri_workspace_bytes", C.c_size_t, [_TCFG, _TMESH]),
    ("zb_tri_init", C.c_int, [_TCFG, _TMESH, _P, C.c_int, C.c_double, _P]),
    ("zb_tri_step", C.c_int, [_TCFG, _TMESH, _P, _P, C.c_size_t, _P, C.c_int, _P]),
    ("zb_tri_stage", C.c_int, [_TCFG, _TMESH, _P, _P, _P, C.c_double, C.c_double,
                               C.c_double, _P, _P, _P, _P, C.c_size_t, _P, _P]),
    ("zb_tri_dt", C.c_int, [_TCFG, _TMESH, _P, _P, C.c_size_t, _P, C.c_double, _P]),
    ("zb_tri_source", C.c_int, [_TCFG, _TMESH, _P, _P, C.c_double, _P]),
    ("zb_tri_aux", C.c_int, [_TCFG, _TMESH, _P, _P, _P]),
    ("zb_tri_mass_partials", C.c_size_t, []),
    ("zb_tri_mass", C.c_int, [_TCFG, _TMESH, _P, _P, _P, _P]),
    ("zb_trimesh_scratch_bytes", C.c_size_t, [C.c_int32]),
    ("zb_trimesh_match", C.c_int, [_P, C.c_int32, _P, C.c_int32, _P, C.c_size_t,
                                   C.POINTER(C.c_int32), C.POINTER(C.c_int32), _P]),
    ("zb_trimesh_fill", C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), C.c_int32, _P,
                                  C.c_size_t, _TMESH, _P]),
    ("zb_unet_conv_impl", C.c_int, [C.c_int]),
    ("zb_unet_status", C.c_int, [C.c_int]),
    ("zb_unet_param_count", C.c_size_t, [C.c_int, C.c_int, C.POINTER(C.c_size_t),
                                         C.POINTER(C.c_size_t)]),
    ("zb_smoother_workspace_bytes", C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ("zb_smoother_apply", C.c_int, [_SMO, _P, _P, _P, _P, _P, _P, C.c_int, C.c_int,
                                    C.c_double, C.c_int, _P]),
    ("zb_unet_train_workspace_bytes", C.c_size_t, [C.c_int, C.c_int, C.c_int, C.c_int]),
    ("zb_unet_forward", C.c_int, [_TRN, _P, _P, _P, C.c_double, _P, _P]),
    ("zb_unet_backward", C.c_int, [_TRN, _P, _P, _P, _P, C.c_double, _P, _P]),
    ("zb_unet_adam", C.c_int, [_TRN, C.c_float, C.c_int, _P]),
    ("zb_poisson_workspace_bytes", C.c_size_t, [_PCFG]),
    ("zb_poisson_layout", C.c_int, [_PCFG, C.POINTER(C.c_int64)]),
    ("zb_poisson_setup", C.c_int, [_PCFG, _P, C.c_int, _P, C.c_size_t, _P]),
    ("zb_poisson_apply", C.c_int, [_PCFG, _P, _P, _P, _P]),
    ("zb_poisson_vcycle", C.c_int, [_PCFG, _P, _P, _P, C.c_int, _SMO, _P]),
    ("zb_poisson_rhs", C.c_int, [_PCFG, _P, C.c_int, C.c_double, _P, _P]),
    ("zb_poisson_correct", C.c_int, [_PCFG, _P, _P, C.c_int, _P, C.c_double, _P]),
    ("zb_fcg_start", C.c_int, [_PCFG, _P, _P, _P, C.c_int, _SMO, _P]),
    ("zb_fcg_iterate", C.c_int, [_PCFG, _P, _P, C.c_int, _SMO, _P]),
    ("zb_fcg_graph_create", C.c_int, [_PCFG, _P, _P, _P, C.c_int, _SMO, C.c_double, C.c_int,
                                      C.POINTER(C.c_void_p), _P]),
    ("zb_fcg_graph_launch", C.c_int, [_P, _P]),
    ("zb_fcg_graph_destroy", None, [_P]),
    ("zb_poisson_solve", C.c_int, [_PCFG, _P, _P, _P, C.c_double, C.c_int, C.c_int, _SMO,
                                   C.POINTER(C.c_int), C.POINTER(C.c_double), _P]),
]

_lib = None


def load():
    """Load libzb.so (build it with ``python zoomy-jax_b200/build.py``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"libzb.so not found at {LIB_PATH}; build it with "
            f"`python zoomy-jax_b200/build.py` (nvcc, sm_100a). There is no "
            f"CPU fallback.")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class ZbError(RuntimeError):
    pass


def check(rc, what):
    if rc != ZB_OK:
        names = {ZB_E_ARG: "invalid argument", ZB_E_CUDA: "CUDA error",
                 ZB_E_UNSUPPORTED: "unsupported configuration",
                 ZB_E_TOO_LARGE: "too large for a fixed-size buffer",
                 ZB_E_NOT_CONVERGED: "not converged"}
        raise ZbError(f"{what} failed: {names.get(rc, rc)}")


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError(
            "zoomy_b200 runs on a CUDA device (sm_100a) only; no GPU is "
            "visible and there is no CPU fallback.")
    load()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def inf_or(x):
    return math.inf if x is None else float(x)
