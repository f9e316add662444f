"""ctypes binding of ``libattract_b200.so`` (the C ABI in include/attract_b200.h).

The shared library is built in-tree by ``attract_b200.build`` (nvcc, sm_100a).
There is no fallback: if the library is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libattract_b200.so")

ATT_OK = 0
ATT_GRAD_REFERENCE = 0
ATT_GRAD_ANALYTIC = 1
ATT_FLAG_TRILINEAR_QUIRK = 1
ATT_STATUS_NONFINITE_GRAD = 1
ATT_STATUS_NONFINITE_ENERGY = 2
ATT_STATUS_NONFINITE_POSE = 4
ATT_MAX_GRIDS = 8
ATT_KERR_COPY_TIMEOUT = 1
ATT_KERR_BOUNDS = 2
ATT_KERR_BAD_SEGMENT = 4
ATT_NB_EMPTY = 65535


class AttractError(RuntimeError):
    """Raised when a C-ABI call returns a non-zero status."""


class AttGridGeom(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("spacing", C.c_float), ("dim", C.c_int * 3),
                ("dim2", C.c_int * 3), ("extension", C.c_int), ("plateau", C.c_float),
                ("n_types", C.c_int), ("pad_", C.c_int)]


class AttGrid(C.Structure):
    _fields_ = [("geom", AttGridGeom), ("bricks", C.c_void_p), ("n_inner_bricks", C.c_longlong),
                ("n_outer_bricks", C.c_longlong), ("nb_hdr", C.c_void_p), ("nb_list", C.c_void_p),
                ("n_nb_entries", C.c_longlong), ("rec", C.c_void_p), ("n_rec", C.c_int),
                ("n_rtypes", C.c_int), ("n_ltypes", C.c_int), ("nb_rec_bytes", C.c_int), ("pair", C.c_void_p),
                ("nb_rec", C.c_void_p), ("nb_refine", C.c_int), ("pad2_", C.c_int)]


class AttLigands(C.Structure):
    _fields_ = [("beads", C.c_void_p), ("offset", C.c_void_p), ("n_lig", C.c_int), ("max_beads", C.c_int),
                ("n_beads", C.c_int), ("pad_", C.c_int)]


class AttSegment(C.Structure):
    _fields_ = [("grid", C.c_int), ("lig", C.c_int), ("pose0", C.c_int), ("n_poses", C.c_int),
                ("step0", C.c_int), ("pad_", C.c_int * 3)]


class AttEvalCfg(C.Structure):
    _fields_ = [("grad_mode", C.c_int), ("flags", C.c_int), ("gravity", C.c_float), ("pose_format", C.c_int)]


class AttAdamCfg(C.Structure):
    _fields_ = [("eval", AttEvalCfg), ("lr_rot", C.c_float), ("lr_trans", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("step0", C.c_int)]


ATT_MAX_STAGES = 8


class AttSchemaCfg(C.Structure):
    _fields_ = [("eval", AttEvalCfg), ("n_stages", C.c_int), ("epochs", C.c_int * ATT_MAX_STAGES),
                ("lr", C.c_float * ATT_MAX_STAGES), ("gravity", C.c_int * ATT_MAX_STAGES), ("beta1", C.c_float),
                ("beta2", C.c_float), ("eps", C.c_float), ("eps_root", C.c_float)]


class AttLaunchCfg(C.Structure):
    _fields_ = [("lanes_per_pose", C.c_int), ("block_threads", C.c_int), ("blocks", C.c_int), ("test_flags", C.c_int)]


P = C.c_void_p
I = C.c_int
F = C.c_float
LL = C.c_longlong

# name -> (restype, argtypes); every name here is declared in include/attract_b200.h
SIGNATURES = {
    "att_last_error_string": (C.c_char_p, []),
    "att_version": (C.c_char_p, []),
    "att_grid_brick_bytes": (LL, [C.POINTER(AttGridGeom), I]),
    "att_grid_repack": (I, [C.POINTER(AttGridGeom), P, P, P, P]),
    "att_energrad": (I, [C.POINTER(AttGrid), I, C.POINTER(AttLigands), P, I, P, I, I, P, P,
                         C.POINTER(AttEvalCfg), P, P, P, C.POINTER(AttLaunchCfg), P]),
    "att_minimise": (I, [C.POINTER(AttGrid), I, C.POINTER(AttLigands), P, I, P, I, I, P, P, P, P,
                         C.POINTER(AttAdamCfg), I, P, P, P, P, C.POINTER(AttLaunchCfg), P]),
    "att_energrad_backward": (I, [C.POINTER(AttGrid), I, C.POINTER(AttLigands), P, I, P, I, I, P, P,
                                  C.POINTER(AttEvalCfg), P, P, P, P, C.POINTER(AttLaunchCfg), P]),
    "att_build_potential_grid": (I, [C.POINTER(AttGridGeom), P, I, P, I, I, F, I, P, P]),
    "att_nbgrid_workspace_bytes": (LL, [LL]),
    "att_nbgrid_count": (I, [C.POINTER(AttGridGeom), P, I, F, P, P, P, LL, P]),
    "att_nbgrid_fill": (I, [C.POINTER(AttGridGeom), P, I, F, P, P, P]),
    "att_kernel_status": (I, [C.POINTER(C.c_int), I, P]),
    "att_nbgrid_count_noalloc": (I, [C.POINTER(AttGridGeom), P, I, F, P, P, P]),
    "att_nbgrid_pack_records": (I, [P, P, LL, I, P, P]),
    "att_kernel_debug_info": (I, [C.POINTER(C.c_ulonglong), I, P]),
    "att_allpairs_energy": (I, [P, I, P, I, P, I, I, P, I, I, F, P, P, P]),
    "att_minimise_schema": (I, [C.POINTER(AttGrid), I, C.POINTER(AttLigands), P, I, P, I, I, P, P, P,
                                C.POINTER(AttSchemaCfg), P, P, P, C.POINTER(AttLaunchCfg), P]),
}

_lib = None


def load(path: str | None = None):
    """Load the library once; raises if it has not been built.  The path may be
    overridden with $ATTRACT_B200_LIB (another build of the same sources)."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = os.environ.get("ATTRACT_B200_LIB") or LIB_PATH
    if not os.path.exists(path):
        raise AttractError(
            f"{path} is missing: build it with `python -m attract_b200.build` (nvcc, sm_100a); "
            "attract_b200 has no CPU fallback")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str = "") -> None:
    if rc != ATT_OK:
        msg = load().att_last_error_string().decode(errors="replace")
        raise AttractError(f"{what}: status {rc}: {msg}")


def kernel_status(clear: bool = True, stream=None) -> int:
    """The scoring kernels' device-wide error word (0 = no warp stopped early)."""
    import torch

    out = C.c_int(0)
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream
    check(load().att_kernel_status(C.byref(out), int(clear), st), "att_kernel_status")
    return out.value


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    if t is None:
        return None
    return t.data_ptr()
