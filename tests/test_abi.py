"""The C-ABI library loads on a CPU-only host and exports every declared symbol.

No compute is launched here (there is no GPU); this pins the boundary: the
entry points named in include/*.h exist, and the numpy/ctypes mirrors of the
descriptor structs have the C sizes.
"""
import ctypes
import glob
import os
import re

import pytest

from dpnegf_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*[A-Za-z_][\w\s\*]*?\b(negf_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "negf_rgf_run" in names and "negf_rgf_scratch_bytes" in names, names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_symbol(name):
    lib = ctypes.CDLL(_lib.LIB_PATH)
    assert hasattr(lib, name), f"{name} declared in include/ but not exported"


def test_struct_mirrors_match_c_sizes():
    lib = _lib.load()
    assert lib.negf_abi_struct_size(0) == _lib.BLOCK_DTYPE.itemsize
    assert lib.negf_abi_struct_size(1) == _lib.DEVICE_DTYPE.itemsize
    assert lib.negf_abi_struct_size(2) == _lib.ITEM_DTYPE.itemsize
    assert lib.negf_abi_struct_size(3) == ctypes.sizeof(_lib.NegfRgfProblem)
    assert lib.negf_abi_struct_size(4) == _lib.LEAD_DTYPE.itemsize
    assert lib.negf_abi_struct_size(5) == _lib.LS_ITEM_DTYPE.itemsize
    assert lib.negf_abi_struct_size(6) == ctypes.sizeof(_lib.NegfLsProblem)
    assert lib.negf_abi_struct_size(7) == ctypes.sizeof(_lib.NegfGammaSum)
    assert lib.negf_abi_struct_size(8) == _lib.LEADADJ_ITEM_DTYPE.itemsize
    assert lib.negf_abi_struct_size(9) == ctypes.sizeof(_lib.NegfLeadAdjProblem)
    assert ctypes.sizeof(_lib.NegfLead) == _lib.LEAD_DTYPE.itemsize


def test_scratch_query_without_gpu():
    lib = _lib.load()
    p = _lib.NegfRgfProblem()
    p.n_slots, p.max_n, p.max_g_slab, p.flags = 2, 64, 64 * 64 * 3, 0
    need = lib.negf_rgf_scratch_bytes(ctypes.byref(p))
    assert need >= 2 * (18 * 64 * 64 + 64 * 64 * 3) * 16
    p.flags = _lib.OUT_GR_LEFT
    assert lib.negf_rgf_scratch_bytes(ctypes.byref(p)) < need


def test_run_rejects_bad_arguments_without_launch():
    lib = _lib.load()
    p = _lib.NegfRgfProblem()
    assert lib.negf_rgf_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT


def test_gamma_sum_rejects_bad_descriptors_without_launch():
    """negf_gamma_sum_run validates its descriptor before any device call."""
    lib = _lib.load()
    p = _lib.NegfGammaSum()
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT
    fake = 1 << 20  # never dereferenced: every case below fails a host-side check first
    p.g = p.gamma = p.w = p.out = fake
    p.n_items, p.n, p.c0, p.k, p.ldg, p.ldgam = 4, 32, 20, 16, 32, 16
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # c0 + k > ldg
    p.c0 = 16
    p.ldgam = 8
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # ldgam < k
    p.ldgam = 16
    need = lib.negf_gamma_sum_scratch_bytes(ctypes.byref(p))
    assert need >= 2 * 32 * 4 * 16 * 16 and need % 256 == 0
    p.scratch, p.scratch_bytes = fake, need - 1
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # scratch too small
    p.scratch_bytes, p.g = need, fake + 8
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # G not 16-byte aligned
    p.g, p.n_items, p.k, p.ldg, p.ldgam = fake, 1 << 24, 512, 1024, 512
    assert lib.negf_gamma_sum_run(ctypes.byref(p), None) == _lib.NEGF_ERR_UNSUPPORTED  # n_items k > 2^31


def test_lead_adjoint_rejects_bad_descriptors_without_launch():
    """negf_lead_adjoint_run validates its descriptor before any device call."""
    lib = _lib.load()
    p = _lib.NegfLeadAdjProblem()
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT
    fake = 1 << 20
    p.arena = p.items = p.grad = p.status = p.scratch = fake
    p.lead.n, p.lead.nc, p.lead.b, p.lead.hdl, p.lead.sdl = 24, 10, 8, 0, 80
    p.n_items, p.n_slots, p.max_iter = 6, 2, 64
    p.form = 3
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # unknown form
    p.form = 0
    p.lead.nc = 0
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # coupling form, no H_DL
    p.lead.nc, p.lead.b = 10, 30
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # b > n
    p.lead.b = 8
    need = lib.negf_lead_adjoint_scratch_bytes(ctypes.byref(p))
    assert need == 2 * ((18 * 24 * 24 + 15) // 16 * 16) * 16
    p.scratch_bytes = need - 16
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_ARGUMENT  # scratch too small
    p.lead.n = 600
    p.scratch_bytes = lib.negf_lead_adjoint_scratch_bytes(ctypes.byref(p))
    assert lib.negf_lead_adjoint_run(ctypes.byref(p), None) == _lib.NEGF_ERR_UNSUPPORTED  # n > NEGF_MAX_BLOCK
