"""ctypes access to the reference's own CUDA build (oracle/_ref/libd3_ref*.so).

Test infrastructure: used by tests/ as a second checker (at FP32-level tolerance, the
reference computes in float) and by bench.py's reference arm. The library is built by
oracle/build_ref.py from the reference's unmodified sources.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libd3_ref.so")
REF_EXT_SO = os.path.join(HERE, "_ref", "libd3_ref_ext.so")

_libs = {}


def available(extended=False):
    return os.path.exists(REF_EXT_SO if extended else REF_SO)


def load(extended=False):
    if extended in _libs:
        return _libs[extended]
    path = REF_EXT_SO if extended else REF_SO
    if not os.path.exists(path):
        raise OSError("reference build missing: %s (run python oracle/build_ref.py)" % path)
    lib = ctypes.CDLL(path)
    vp, u64, f32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_float, ctypes.c_int
    lib.init_d3_handle.restype = vp
    lib.init_d3_handle.argtypes = [vp, u64, u64, f32, f32, i32, i32]
    lib.init_d3_handle_with_atm.restype = vp
    lib.init_d3_handle_with_atm.argtypes = [vp, u64, u64, f32, f32, f32, i32, i32]
    lib.set_atoms.restype = None
    lib.set_atoms.argtypes = [vp, vp, vp, u64]
    lib.set_cell.restype = None
    lib.set_cell.argtypes = [vp, vp]
    lib.clear_d3_handle.restype = None
    lib.clear_d3_handle.argtypes = [vp]
    lib.free_d3_handle.restype = None
    lib.free_d3_handle.argtypes = [vp]
    lib.compute_dispersion_energy_from_handle_status.restype = ctypes.c_uint16
    lib.compute_dispersion_energy_from_handle_status.argtypes = [vp, vp, vp, vp]
    _libs[extended] = lib
    return lib


class RefHandle:
    """The reference's handle API (src/d3.h), float in / float out."""

    def __init__(self, elements, max_len, rc, rc_cn, rc_atm=None, damping=1, functional=0, extended=False):
        self.lib = load(extended)
        el = np.ascontiguousarray(elements, np.uint16)
        if rc_atm is None:
            self.h = self.lib.init_d3_handle(el.ctypes.data, len(el), int(max_len), rc, rc_cn, damping, functional)
        else:
            self.h = self.lib.init_d3_handle_with_atm(el.ctypes.data, len(el), int(max_len), rc, rc_cn, rc_atm,
                                                      damping, functional)
        if not self.h:
            raise RuntimeError("reference init failed")
        self.n = 0

    def set_system(self, pos, Z, cell):
        pos = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
        z = np.ascontiguousarray(Z, np.uint16)
        c = np.ascontiguousarray(cell, np.float32).reshape(3, 3)
        self.lib.set_atoms(self.h, pos.ctypes.data, z.ctypes.data, len(z))
        self.lib.set_cell(self.h, c.ctypes.data)
        self.n = len(z)

    def compute(self):
        e = np.zeros(1, np.float32)
        f = np.zeros((self.n, 3), np.float32)
        s = np.zeros(9, np.float32)
        self.lib.clear_d3_handle(self.h)
        st = self.lib.compute_dispersion_energy_from_handle_status(self.h, e.ctypes.data, f.ctypes.data, s.ctypes.data)
        return float(e[0]), f, s.reshape(3, 3), int(st)

    def close(self):
        if self.h:
            self.lib.free_d3_handle(self.h)
            self.h = None


def run(pos, Z, cell, rc=95.0, rc_cn=40.0, rc_atm=None, damping=1, functional=0, extended=False, init_elements=None):
    h = RefHandle(init_elements if init_elements is not None else Z, len(Z), rc, rc_cn, rc_atm, damping, functional,
                  extended)
    try:
        h.set_system(pos, Z, cell)
        return h.compute()
    finally:
        h.close()
