"""Failure paths of the drop-in ABI, caused on the host (no GPU fault is made): the status
word of compute_dispersion_energy_from_handle_status / d3_compute_f64 (bit 0 neighbour-list
overflow as in the reference, src/d3_internal.h:6-7; bit 1 non-finite input; bit 2
degenerate cell; bit 5 atoms or cell not set), errors instead of exit() for set_atoms
beyond the handle's capacity (the reference exits, src/d3_buffer.cu:380-383) and for
elements not given at init, and the ATM list's overflow -> grow -> run again loop of the
synchronous call, which inside a captured CUDA graph reports bit 0 instead of
reallocating."""
import ctypes

import numpy as np
import pytest

import d3_systems as S
from d3_b200 import D3, OPT_ATM_LIST_CAPACITY, OPT_PRECISION, load_library

pytestmark = pytest.mark.gpu

KW = dict(rc=40.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=1)


def _float_handle(lib, Z, max_len):
    z = np.ascontiguousarray(sorted(set(int(x) for x in Z)), np.uint16)
    lib.init_d3_handle_with_atm.restype = ctypes.c_void_p
    h = lib.init_d3_handle_with_atm(z.ctypes.data, len(z), max_len, ctypes.c_float(40.0), ctypes.c_float(40.0),
                                    ctypes.c_float(40.0), 1, 1)
    assert h
    return ctypes.c_void_p(h)


def _float_compute(lib, h, n):
    e = np.zeros(1, np.float32)
    f = np.zeros((n, 3), np.float32)
    s = np.zeros(9, np.float32)
    return int(lib.compute_dispersion_energy_from_handle_status(h, e.ctypes.data, f.ctypes.data, s.ctypes.data))


def test_non_finite_coordinate_sets_bit_1():
    s = S.gtest_small_system()
    pos = s["pos"].copy()
    pos[3, 1] = np.nan
    d = D3(s["Z"], len(s["Z"]), **KW)
    d.set_cell(s["cell"])
    d.set_atoms(pos, s["Z"])
    d.compute(check=False)
    assert d.status & 0x02
    d.close()
    lib = load_library()
    h = _float_handle(lib, s["Z"], len(s["Z"]))
    cf = np.ascontiguousarray(s["cell"], np.float32)
    lib.set_cell(h, cf.ctypes.data)
    pf = np.ascontiguousarray(pos, np.float32)
    z = np.ascontiguousarray(s["Z"], np.uint16)
    lib.set_atoms(h, pf.ctypes.data, z.ctypes.data, len(z))
    assert _float_compute(lib, h, len(z)) & 0x02
    lib.free_d3_handle(h)


def test_degenerate_cell_sets_bit_2():
    s = S.gtest_small_system()
    flat = np.array([[10.0, 0, 0], [20.0, 0, 0], [0, 0, 10.0]])  # two parallel lattice vectors
    d = D3(s["Z"], len(s["Z"]), **KW)
    d.set_atoms(s["pos"], s["Z"])
    with pytest.raises(RuntimeError, match="degenerate"):
        d.set_cell(flat)
    d.compute(check=False)
    assert d.status == 0x04
    d.close()
    lib = load_library()
    h = _float_handle(lib, s["Z"], len(s["Z"]))
    z = np.ascontiguousarray(s["Z"], np.uint16)
    pf = np.ascontiguousarray(s["pos"], np.float32)
    lib.set_atoms(h, pf.ctypes.data, z.ctypes.data, len(z))
    lib.set_cell(h, np.ascontiguousarray(flat, np.float32).ctypes.data)  # void: reports through the status
    assert _float_compute(lib, h, len(z)) == 0x04
    assert b"degenerate" in lib.d3_last_error()
    # a valid cell afterwards clears it
    lib.set_cell(h, np.ascontiguousarray(s["cell"], np.float32).ctypes.data)
    assert _float_compute(lib, h, len(z)) == 0
    lib.free_d3_handle(h)


def test_element_not_given_at_init_is_rejected():
    s = S.gtest_small_system()  # C, O, H
    d = D3([1, 6], len(s["Z"]), **KW)
    d.set_cell(s["cell"])
    with pytest.raises(RuntimeError, match="element 8 was not given"):
        d.set_atoms(s["pos"], s["Z"])
    d.compute(check=False)
    assert d.status == 0x20  # atoms never set
    d.close()


def test_set_atoms_beyond_capacity_returns_an_error_instead_of_exiting():
    s = S.gtest_small_system()
    lib = load_library()
    h = _float_handle(lib, s["Z"], 5)  # capacity 5, ten atoms given
    lib.set_cell(h, np.ascontiguousarray(s["cell"], np.float32).ctypes.data)
    z = np.ascontiguousarray(s["Z"], np.uint16)
    lib.set_atoms(h, np.ascontiguousarray(s["pos"], np.float32).ctypes.data, z.ctypes.data, len(z))
    assert b"capacity" in lib.d3_last_error()
    assert _float_compute(lib, h, len(z)) == 0x20
    lib.set_atoms(h, np.ascontiguousarray(s["pos"][:5], np.float32).ctypes.data, z.ctypes.data, 5)
    assert _float_compute(lib, h, 5) == 0  # the process and the handle are still usable
    lib.free_d3_handle(h)


@pytest.mark.parametrize("precision", [0, 1])
def test_list_overflow_grows_and_runs_again(precision):
    s = S.triclinic_box(400, seed=12)
    kw = dict(rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)
    ref = D3(s["Z"], len(s["Z"]), **kw)
    ref.set_option(OPT_PRECISION, precision)
    ref.set_cell(s["cell"])
    ref.set_atoms(s["pos"], s["Z"])
    e0, f0, s0 = ref.compute()
    ref.close()
    d = D3(s["Z"], len(s["Z"]), **kw)
    d.set_option(OPT_PRECISION, precision)
    d.set_option(OPT_ATM_LIST_CAPACITY, 64)  # far below the ~1e5 entries needed
    assert d.atm_list_capacity() == 64
    d.set_cell(s["cell"])
    d.set_atoms(s["pos"], s["Z"])
    e1, f1, s1 = d.compute()  # status 0: the call grew the list and ran again
    assert d.atm_list_capacity() > 64
    # the ATM scatter's FP64 atomics add in run-dependent order: FP64 to 1e-12, the
    # precision form's FP32 partial sums to 1e-9
    tol = 1e-12 if precision == 0 else 1e-9
    assert abs(e1 - e0) <= tol * abs(e0)
    assert np.abs(f1 - f0).max() <= 100 * tol
    d.close()


def test_list_overflow_inside_a_graph_sets_bit_0_without_reallocating():
    import torch

    s = S.triclinic_box(400, seed=12)
    d = D3(s["Z"], len(s["Z"]), rc=95.0, rc_cn=40.0, rc_atm=40.0, damping=1, functional=0)
    d.set_option(OPT_ATM_LIST_CAPACITY, 64)
    d.set_cell(s["cell"])
    d.set_atoms(s["pos"], s["Z"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    with torch.cuda.stream(stream):
        graph.replay()
    torch.cuda.synchronize()
    assert d.fetch_status() & 0x01
    assert d.atm_list_capacity() == 64
    del graph
    d.close()
