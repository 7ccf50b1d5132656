"""The no-allocation coordination-number entry point, d3_coordination_numbers_noalloc.

Some callers cannot let the library allocate device memory where they call it: an MD
engine plugin inside its time-step loop (cudaMalloc would synchronise the device and
stall the engine's other streams) or an application whose device memory is all owned by
its own pool allocator. This entry point takes caller-owned device buffers and keeps its
only scratch in a fixed device array; here its output is checked against the handle
API's coordination numbers (FP64, same 1e-12 relative tolerance as the parity tests),
on two calls in a row that reuse the shared scratch array with different systems.
"""
import ctypes

import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, TABLE_7REF, load_library

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.d3_coordination_numbers_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    return f


def _handle_cn(sys_, rc_cn, table=0):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=rc_cn, rc_cn=rc_cn, table=table)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    d.compute()
    cn, _, _ = d.atom_arrays()
    d.close()
    return cn


def _noalloc_cn(fn, sys_, rc_cn, table=0):
    import torch

    pos = torch.from_numpy(np.ascontiguousarray(sys_["pos"], np.float64)).cuda()
    z = torch.from_numpy(np.asarray(sys_["Z"], np.int16)).cuda()  # same bits as uint16 for Z < 32768
    out = torch.full((len(sys_["Z"]),), -1.0, dtype=torch.float64, device="cuda")
    cell = np.ascontiguousarray(sys_["cell"], np.float64).reshape(9)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(pos.data_ptr(), z.data_ptr(), len(sys_["Z"]), cell.ctypes.data, rc_cn, table, out.data_ptr(), stream)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_noalloc_matches_handle_api_on_two_calls_in_a_row():
    fn = _bind(load_library())
    big = S.triclinic_box(1500, seed=11)
    small = S.water_box(2)
    rc_cn = 40.0
    want_big, want_small = _handle_cn(big, rc_cn), _handle_cn(small, rc_cn)
    got_big = _noalloc_cn(fn, big, rc_cn)
    got_small = _noalloc_cn(fn, small, rc_cn)  # reuses the scratch left by the first call
    np.testing.assert_allclose(got_big, want_big, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(got_small, want_small, rtol=1e-12, atol=1e-12)


def test_noalloc_extended_table_and_element_outside_the_table():
    # 7-reference layout (slots by Z - 1) against a handle built with that table; then one
    # atom of an element outside the 5-reference table (Z = 100): its CN is NaN and it
    # contributes nothing to the other atoms
    fn = _bind(load_library())
    sys_ = S.triclinic_box(400, seed=21)
    np.testing.assert_allclose(_noalloc_cn(fn, sys_, 40.0, table=TABLE_7REF), _handle_cn(sys_, 40.0, TABLE_7REF),
                               rtol=1e-12, atol=1e-12)
    odd = dict(sys_)
    odd["Z"] = np.concatenate([sys_["Z"], [100]])
    odd["pos"] = np.concatenate([sys_["pos"], sys_["pos"][:1] + 0.9])
    got = _noalloc_cn(fn, odd, 40.0)
    assert np.isnan(got[-1])
    np.testing.assert_allclose(got[:-1], _handle_cn(sys_, 40.0), rtol=1e-12, atol=1e-12)


def test_noalloc_rejects_sizes_beyond_its_maximum():
    lib = load_library()
    fn = _bind(lib)
    n = 8193  # D3_NOALLOC_MAX_ATOMS + 1
    dummy = np.zeros(1)
    cell = np.eye(3).reshape(9) * 100.0
    rc = fn(dummy.ctypes.data, dummy.ctypes.data, n, cell.ctypes.data, 40.0, 0, dummy.ctypes.data, None)
    assert rc == 1
    assert b"exceed the maximum" in lib.d3_last_error()

