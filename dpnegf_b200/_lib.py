"""ctypes binding of ``libnegf_b200.so`` (C ABI declared in include/negf_b200.h).

The shared library is built in-tree by ``dpnegf_b200/csrc/build.py`` (also run
by ``__graft_entry__.build()``).  There is no fallback: if the library is
missing or no CUDA device is present, every entry point raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnegf_b200.so")

# status codes (include/negf_b200.h)
NEGF_OK = 0
NEGF_WARN_LS_CONVERGENCE = 1
NEGF_ERR_LS_NOT_CONVERGED = 2
NEGF_ERR_LS_RESIDUAL = 3
NEGF_ERR_SINGULAR = 4
NEGF_ERR_NONFINITE = 5
NEGF_ERR_TIMEOUT = 6
NEGF_ERR_ARGUMENT = -1
NEGF_ERR_UNSUPPORTED = -2
NEGF_ERR_CUDA = -3
NEGF_MAX_BLOCK = 512

# RGF flags
OUT_GTRANS = 1 << 0
OUT_GR_LC = 1 << 1
OUT_GRD = 1 << 2
OUT_GRL = 1 << 3
OUT_GRU = 1 << 4
OUT_GR_LEFT = 1 << 5
TRANS = 1 << 6
ORB_DOS = 1 << 7
LESSER = 1 << 8
DOS = 1 << 9
ORB_GDIAG = 1 << 10
ORB_AR = 1 << 11
ADJOINT = 1 << 12
MIXED = 1 << 13
REFINE = 1 << 14
GREATER = 1 << 15
ADJ_DOS = 1 << 16
PHASES = ("form", "gemm_fwd", "inv_stage", "inv_panel", "inv_update", "inv_gather", "gemm_bwd", "lesser",
          "dos", "trans", "other", "refine")

# numpy mirrors of the descriptor structs (packed exactly like the C structs)
BLOCK_FIELDS = ["hd", "sd", "hu", "su", "hl", "sl", "sdT", "suT", "slT", "orb0", "g", "gc", "gu", "o_grd", "o_grl", "o_gru",
                "o_grlc",
                "o_grleft", "o_gnd", "o_gnl", "o_gnu", "o_ginleft", "s_in", "o_gpd", "o_gpl", "o_gpu",
                "o_gipleft", "s_out"]
BLOCK_DTYPE = np.dtype([("n", "<i4"), ("n_next", "<i4")] + [(f, "<i8") for f in BLOCK_FIELDS])
DEVICE_DTYPE = np.dtype([("n_blocks", "<i4"), ("blk0", "<i4"), ("n_orb", "<i4"), ("pad", "<i4"),
                         ("o_gtrans", "<i8"), ("g_slab", "<i8")])
ITEM_DTYPE = np.dtype([("dev", "<i4"), ("row", "<i4"), ("z_re", "<f8"), ("z_im", "<f8"),
                       ("se_l", "<u8"), ("se_r", "<u8"), ("nse_l", "<i4"), ("nse_r", "<i4"),
                       ("out", "<i8"), ("orb", "<i8"), ("w_t", "<f8"), ("gse_l", "<u8"), ("gse_r", "<u8"),
                       ("w_d", "<f8")])


LEAD_DTYPE = np.dtype([("n", "<i4"), ("nc", "<i4"), ("b", "<i4"), ("pad", "<i4"), ("h", "<i8"), ("s", "<i8"),
                       ("h01", "<i8"), ("s01", "<i8"), ("hdl", "<i8"), ("sdl", "<i8")])
LS_ITEM_DTYPE = np.dtype([("lead", "<i4"), ("mode", "<i4"), ("e_re", "<f8"), ("e_im", "<f8"), ("eta", "<f8"),
                          ("sigma", "<u8"), ("gs", "<u8"), ("out", "<i8")])
LS_DECIMATE = 0
LS_SIGMA_FROM_GS = 1
LEADADJ_ITEM_DTYPE = np.dtype([("e_re", "<f8"), ("e_im", "<f8"), ("gs", "<u8"), ("gsig", "<u8")])


class NegfLead(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nc", ctypes.c_int32), ("b", ctypes.c_int32), ("pad", ctypes.c_int32),
                ("h", ctypes.c_int64), ("s", ctypes.c_int64), ("h01", ctypes.c_int64), ("s01", ctypes.c_int64),
                ("hdl", ctypes.c_int64), ("sdl", ctypes.c_int64)]


class NegfGammaSum(ctypes.Structure):
    _fields_ = [
        ("g", ctypes.c_void_p),
        ("g_stride", ctypes.c_int64),
        ("gamma", ctypes.c_void_p),
        ("gamma_stride", ctypes.c_int64),
        ("w", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n_items", ctypes.c_int32),
        ("n", ctypes.c_int32),
        ("ldg", ctypes.c_int32),
        ("c0", ctypes.c_int32),
        ("k", ctypes.c_int32),
        ("ldgam", ctypes.c_int32),
        ("scratch", ctypes.c_void_p),
        ("scratch_bytes", ctypes.c_size_t),
    ]


class NegfLeadAdjProblem(ctypes.Structure):
    _fields_ = [
        ("lead", NegfLead),
        ("arena", ctypes.c_void_p),
        ("items", ctypes.c_void_p),
        ("n_items", ctypes.c_int32),
        ("form", ctypes.c_int32),
        ("eta", ctypes.c_double),
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("n_slots", ctypes.c_int32),
        ("grad", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("iters", ctypes.c_void_p),
        ("scratch", ctypes.c_void_p),
        ("scratch_bytes", ctypes.c_size_t),
    ]


class NegfLsProblem(ctypes.Structure):
    _fields_ = [
        ("leads", ctypes.c_void_p),
        ("items", ctypes.c_void_p),
        ("n_items", ctypes.c_int32),
        ("max_n", ctypes.c_int32),
        ("arena", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("iters", ctypes.c_void_p),
        ("resid", ctypes.c_void_p),
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("n_slots", ctypes.c_int32),
        ("scratch", ctypes.c_void_p),
        ("scratch_bytes", ctypes.c_size_t),
    ]


class NegfRgfProblem(ctypes.Structure):
    _fields_ = [
        ("blocks", ctypes.c_void_p),
        ("devices", ctypes.c_void_p),
        ("items", ctypes.c_void_p),
        ("n_items", ctypes.c_int32),
        ("max_n", ctypes.c_int32),
        ("max_g_slab", ctypes.c_int64),
        ("hs", ctypes.c_void_p),
        ("s_in", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("trans", ctypes.c_void_p),
        ("orb_dos", ctypes.c_void_p),
        ("dos", ctypes.c_void_p),
        ("orb_g", ctypes.c_void_p),
        ("orb_ar", ctypes.c_void_p),
        ("status", ctypes.c_void_p),
        ("flags", ctypes.c_uint32),
        ("n_slots", ctypes.c_int32),
        ("scratch", ctypes.c_void_p),
        ("scratch_bytes", ctypes.c_size_t),
        ("phase_cycles", ctypes.c_void_p),
        ("grad", ctypes.c_void_p),
        ("grad_slab", ctypes.c_int64),
        ("col_slab", ctypes.c_int64),
        ("refine_steps", ctypes.c_int32),
        ("inv_ob", ctypes.c_int32),
        ("s_out", ctypes.c_void_p),
        ("inv_mode", ctypes.c_int32),
        ("ckpt", ctypes.c_int32),
        ("ckpt_blocks", ctypes.c_int32),
    ]


_lib = None


class NegfError(RuntimeError):
    pass


def load():
    """Load the CUDA library once; raise loudly when it is unavailable."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.isfile(LIB_PATH):
        raise NegfError(f"{LIB_PATH} is missing: build it with `python dpnegf_b200/csrc/build.py` "
                        "(dpnegf_b200 has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    lib.negf_rgf_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_rgf_scratch_bytes.argtypes = [ctypes.POINTER(NegfRgfProblem)]
    lib.negf_rgf_run.restype = ctypes.c_int
    lib.negf_rgf_run.argtypes = [ctypes.POINTER(NegfRgfProblem), ctypes.c_void_p]
    lib.negf_sm_count.restype = ctypes.c_int
    lib.negf_sm_count.argtypes = []
    lib.negf_version.restype = ctypes.c_char_p
    lib.negf_abi_struct_size.restype = ctypes.c_size_t
    lib.negf_abi_struct_size.argtypes = [ctypes.c_int]
    lib.negf_lopez_sancho_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_lopez_sancho_scratch_bytes.argtypes = [ctypes.POINTER(NegfLsProblem)]
    lib.negf_lopez_sancho_run.restype = ctypes.c_int
    lib.negf_lopez_sancho_run.argtypes = [ctypes.POINTER(NegfLsProblem), ctypes.c_void_p]
    lib.negf_gamma_sum_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_gamma_sum_scratch_bytes.argtypes = [ctypes.POINTER(NegfGammaSum)]
    lib.negf_gamma_sum_run.restype = ctypes.c_int
    lib.negf_gamma_sum_run.argtypes = [ctypes.POINTER(NegfGammaSum), ctypes.c_void_p]
    lib.negf_lead_adjoint_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_lead_adjoint_scratch_bytes.argtypes = [ctypes.POINTER(NegfLeadAdjProblem)]
    lib.negf_lead_adjoint_run.restype = ctypes.c_int
    lib.negf_lead_adjoint_run.argtypes = [ctypes.POINTER(NegfLeadAdjProblem), ctypes.c_void_p]
    _lib = lib
    return lib


def check(code, what):
    if code != NEGF_OK:
        names = {NEGF_ERR_ARGUMENT: "invalid argument", NEGF_ERR_UNSUPPORTED: "unsupported size",
                 NEGF_ERR_CUDA: "CUDA error"}
        raise NegfError(f"{what} failed: {names.get(code, code)}")


def require_cuda():
    import torch
    if not torch.cuda.is_available():
        raise NegfError("dpnegf_b200 needs a CUDA device (B200, sm_100a); no CPU fallback exists")
    load()


def on_given_stream(fn):
    """Run ``fn`` with its ``stream`` keyword as torch's current stream.

    The wrappers stage descriptor tables and scratch in torch tensors, launch, and may read a
    status back; with the caller's stream current for the whole call, all of that is ordered on
    that one stream, so the caching allocator hands the staging memory to other work only behind
    the launch, and host reads see the kernel's writes.  Results belong to that stream."""
    import functools

    @functools.wraps(fn)
    def wrapped(*args, stream=None, **kw):
        if stream is None:
            return fn(*args, stream=None, **kw)
        import torch
        with torch.cuda.stream(stream):
            return fn(*args, stream=None, **kw)
    return wrapped


def stream_handle(torch_stream=None):
    import torch
    s = torch_stream if torch_stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
