"""ctypes binding of libd3.so for Python callers that want the FP64 path and the
engine extensions (the reference-compatible cffi binding is d3_cffi.py).

    from d3_b200 import D3
    d3 = D3(elements=[1, 6, 8], max_atoms=96, rc=95.0, rc_cn=40.0, rc_atm=40.0)
    d3.set_cell(cell)            # Angstrom, rows = lattice vectors
    d3.set_atoms(pos, Z)         # Angstrom
    e, f, s = d3.compute()       # eV, eV/A [n,3], eV/A^3 [3,3] (float64)

The library must be built (python lasp-d3_b200/build.py); loading fails loudly when
it is missing -- there is no CPU fallback.
"""
import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libd3.so")
HEADER = os.path.join(HERE, "..", "include", "d3.h")

ZERO_DAMPING, BJ_DAMPING = 0, 1
OPT_ATM_FORCE_SCALED, OPT_SMOOTH_CN, OPT_PRECISION = 1, 2, 3
OPT_BIN_DIVISOR, OPT_ATM_TILE, OPT_ATM_CTAS_PER_SM = 4, 5, 6
OPT_ATM_SURROGATE = 7
OPT_ATM_SCHEDULE = 8
OPT_ATM_LIST_CAPACITY = 9
OPT_PAIR_KERNEL = 10
OPT_ATMB_WARPS, OPT_ATMB_LIST_CAPACITY, OPT_ATMB_SPLIT, OPT_ATMB_FINE_SKIP = 11, 12, 13, 14
TABLE_5REF, TABLE_7REF = 0, 1

_lib = None


def load_library(path=None):
    """Load libd3.so (raises OSError when it is not built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError("libd3.so not found at %s; build it with python lasp-d3_b200/build.py" % p)
    lib = ctypes.CDLL(p)
    vp, u64, i64, f32, f64 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int64, ctypes.c_float, ctypes.c_double
    lib.init_d3_handle.restype = vp
    lib.init_d3_handle.argtypes = [vp, u64, u64, f32, f32, ctypes.c_int, ctypes.c_int]
    lib.init_d3_handle_with_atm.restype = vp
    lib.init_d3_handle_with_atm.argtypes = [vp, u64, u64, f32, f32, f32, ctypes.c_int, ctypes.c_int]
    lib.set_atoms.restype = None
    lib.set_atoms.argtypes = [vp, vp, vp, u64]
    lib.set_cell.restype = None
    lib.set_cell.argtypes = [vp, vp]
    lib.free_d3_handle.restype = None
    lib.free_d3_handle.argtypes = [vp]
    lib.clear_d3_handle.restype = None
    lib.clear_d3_handle.argtypes = [vp]
    lib.compute_dispersion_energy_from_handle.restype = None
    lib.compute_dispersion_energy_from_handle.argtypes = [vp, vp, vp, vp]
    lib.compute_dispersion_energy_from_handle_status.restype = ctypes.c_uint16
    lib.compute_dispersion_energy_from_handle_status.argtypes = [vp, vp, vp, vp]
    lib.compute_dispersion_energy.restype = None
    lib.compute_dispersion_energy.argtypes = [vp, vp, u64, vp, f32, f32, ctypes.c_int, ctypes.c_int, vp, vp, vp]
    lib.d3_init_handle_ex.restype = vp
    lib.d3_init_handle_ex.argtypes = [vp, u64, u64, f64, f64, f64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.d3_set_atoms_f64.restype = ctypes.c_int
    lib.d3_set_atoms_f64.argtypes = [vp, vp, vp, u64]
    lib.d3_set_cell_f64.restype = ctypes.c_int
    lib.d3_set_cell_f64.argtypes = [vp, vp]
    lib.d3_compute_f64.restype = ctypes.c_uint16
    lib.d3_compute_f64.argtypes = [vp, vp, vp, vp]
    lib.d3_set_option.restype = ctypes.c_int
    lib.d3_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.d3_set_functional_params.restype = ctypes.c_int
    lib.d3_set_functional_params.argtypes = [vp, f64, f64, f64, f64]
    lib.d3_compute_async.restype = ctypes.c_uint16
    lib.d3_compute_async.argtypes = [vp, vp]
    lib.d3_device_results.restype = vp
    lib.d3_device_results.argtypes = [vp]
    lib.d3_init_batch.restype = vp
    lib.d3_init_batch.argtypes = [vp, u64, u64, u64, f64, f64, f64, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.d3_set_batch_f64.restype = ctypes.c_int
    lib.d3_set_batch_f64.argtypes = [vp, u64, vp, vp, vp, vp]
    lib.d3_compute_batch_f64.restype = ctypes.c_uint16
    lib.d3_compute_batch_f64.argtypes = [vp, vp, vp, vp]
    lib.d3_fetch_results.restype = ctypes.c_int
    lib.d3_fetch_results.argtypes = [vp, vp, vp, vp]
    lib.d3_num_structures.restype = ctypes.c_int
    lib.d3_num_structures.argtypes = [vp]
    lib.d3_set_positions_device.restype = ctypes.c_int
    lib.d3_set_positions_device.argtypes = [vp, vp, vp]
    lib.d3_pass_times.restype = ctypes.c_int
    lib.d3_pass_times.argtypes = [vp, vp, ctypes.c_int, vp]
    lib.d3_launches_per_eval.restype = ctypes.c_int
    lib.d3_launches_per_eval.argtypes = [vp]
    lib.d3_peak_probe.restype = ctypes.c_double
    lib.d3_peak_probe.argtypes = [ctypes.c_int]
    lib.d3_selftest_math.restype = ctypes.c_int
    lib.d3_selftest_math.argtypes = [vp]
    lib.d3_last_error.restype = ctypes.c_char_p
    lib.d3_last_error.argtypes = []
    lib.d3_debug_atom_arrays.restype = ctypes.c_int
    lib.d3_debug_atom_arrays.argtypes = [vp, vp, vp, vp]
    lib.d3_fetch_status.restype = ctypes.c_uint16
    lib.d3_fetch_status.argtypes = [vp]
    lib.d3_atm_list_capacity.restype = i64
    lib.d3_atm_list_capacity.argtypes = [vp]
    lib.d3_debug_pass_terms.restype = ctypes.c_int
    lib.d3_debug_pass_terms.argtypes = [vp, vp]
    lib.d3_debug_atm_pairs.restype = i64
    lib.d3_debug_atm_pairs.argtypes = [vp, vp, i64]
    lib.d3_debug_bins.restype = ctypes.c_int
    lib.d3_debug_bins.argtypes = [vp, vp, vp, vp]
    ci = ctypes.c_int
    lib.d3_set_surrogate.restype = ci
    lib.d3_set_surrogate.argtypes = [vp, vp, ci, ci, vp, vp, vp, vp, f32]
    lib.d3_set_surrogate_threshold.restype = ci
    lib.d3_set_surrogate_threshold.argtypes = [vp, f64]
    lib.d3_surrogate_flagged.restype = ci
    lib.d3_surrogate_flagged.argtypes = [vp]
    lib.d3_surrogate_descriptors.restype = ci
    lib.d3_surrogate_descriptors.argtypes = [vp, vp, ci, vp, vp, vp, vp]
    lib.d3_mlp_layout.restype = ci
    lib.d3_mlp_layout.argtypes = [ci, vp]
    lib.d3_mlp_acts_elems.restype = u64
    lib.d3_mlp_acts_elems.argtypes = [ci, ci]
    lib.d3_mlp_pack.restype = ci
    lib.d3_mlp_pack.argtypes = [ci, ci, vp, vp, vp]
    lib.d3_mlp_forward.restype = ci
    lib.d3_mlp_forward.argtypes = [ci, ci, vp, vp, vp, vp, vp, vp, ci, vp, vp, vp]
    lib.d3_mlp_train_batch.restype = ci
    lib.d3_mlp_train_batch.argtypes = [ci, ci, vp, vp, vp, vp, vp, vp, vp, vp, ci, vp, vp, vp, vp, vp]
    lib.d3_copy_results_device.restype = ci
    lib.d3_copy_results_device.argtypes = [vp, vp, vp]
    lib.d3_shard_length.restype = u64
    lib.d3_shard_length.argtypes = [vp]
    lib.d3_shard_begin.restype = ctypes.c_uint16
    lib.d3_shard_begin.argtypes = [vp, ci, ci, vp, vp]
    lib.d3_shard_end.restype = ctypes.c_uint16
    lib.d3_shard_end.argtypes = [vp, vp, vp, vp]
    lib.d3_mlp_adam.restype = ci
    lib.d3_mlp_adam.argtypes = [ci, ci, vp, vp, vp, vp, vp, ci, f32, f32, f32, f32, f32, ci, vp]
    if path is None:
        _lib = lib
    return lib


def declared_symbols(header=HEADER):
    """Function names declared in include/d3.h."""
    txt = open(header).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)) - {"if", "sizeof", "defined"})


def selftest_math():
    """Max relative errors of the ATM kernel's refined rsqrt, reciprocal, rcbrt
    (one Newton step, then two Newton steps)."""
    lib = load_library()
    e = np.zeros(6)
    if lib.d3_selftest_math(_ptr(e)):
        raise RuntimeError(lib.d3_last_error().decode())
    return e


def peak_probe(fp64=True):
    """Measured FMA throughput of the FP64 / FP32 pipe (TFLOP/s)."""
    return float(load_library().d3_peak_probe(1 if fp64 else 0))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class _Surrogate:
    """Learned ATM surrogate methods shared by D3 and D3Batch (model: d3_surrogate.Model)."""

    def set_surrogate(self, model, threshold_ev=None, enable=True):
        cz = np.ascontiguousarray(model.channel_z, np.int32)
        params = np.ascontiguousarray(model.params, np.float32)
        mean = np.ascontiguousarray(model.mean, np.float32)
        istd = np.ascontiguousarray(model.inv_std, np.float32)
        shift = np.ascontiguousarray(model.e_shift, np.float32)
        if self.lib.d3_set_surrogate(self.h, _ptr(cz), len(cz), int(model.members), _ptr(params), _ptr(mean),
                                     _ptr(istd), _ptr(shift), float(model.e_scale)):
            raise RuntimeError(self.lib.d3_last_error().decode())
        if threshold_ev is not None:
            self.set_surrogate_threshold(threshold_ev)
        self.set_option(OPT_ATM_SURROGATE, 1 if enable else 0)

    def set_surrogate_threshold(self, threshold_ev):
        if self.lib.d3_set_surrogate_threshold(self.h, float(threshold_ev)):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def surrogate_flagged(self):
        return int(self.lib.d3_surrogate_flagged(self.h))

    def surrogate_descriptors(self, channel_z, G_ptr=None, center_ptr=None, e_atm_ptr=None, stream_ptr=None):
        """Descriptors of the current atoms into device buffers (caller order); see
        d3_surrogate_descriptors in include/d3.h."""
        cz = np.ascontiguousarray(channel_z, np.int32)
        vp = ctypes.c_void_p
        if self.lib.d3_surrogate_descriptors(self.h, _ptr(cz), len(cz), vp(G_ptr) if G_ptr else None,
                                             vp(center_ptr) if center_ptr else None,
                                             vp(e_atm_ptr) if e_atm_ptr else None,
                                             vp(stream_ptr) if stream_ptr else None):
            raise RuntimeError(self.lib.d3_last_error().decode())


class _Shard:
    """Sharded-evaluation stages shared by D3 and D3Batch (driver: d3_shard.py)."""

    def shard_length(self):
        return int(self.lib.d3_shard_length(self.h))

    def shard_structures(self):
        """Structures of this handle: d3_shard_end writes 10 S + 3 n result values."""
        return int(self.lib.d3_num_structures(self.h))

    def shard_begin(self, rank, world, dedcn_ptr, stream_ptr=None):
        st = int(self.lib.d3_shard_begin(self.h, int(rank), int(world), ctypes.c_void_p(dedcn_ptr),
                                         ctypes.c_void_p(stream_ptr) if stream_ptr else None))
        if st:
            raise RuntimeError("d3_shard_begin status %d: %s" % (st, self.lib.d3_last_error().decode()))

    def shard_end(self, dedcn_ptr, results_ptr, stream_ptr=None):
        st = int(self.lib.d3_shard_end(self.h, ctypes.c_void_p(dedcn_ptr), ctypes.c_void_p(results_ptr),
                                       ctypes.c_void_p(stream_ptr) if stream_ptr else None))
        if st:
            raise RuntimeError("d3_shard_end status %d: %s" % (st, self.lib.d3_last_error().decode()))


class D3(_Surrogate, _Shard):
    """One engine handle (FP64 path)."""

    def __init__(self, elements, max_atoms, rc=95.0, rc_cn=40.0, rc_atm=None, damping=BJ_DAMPING, functional=0,
                 table=TABLE_5REF):
        self.lib = load_library()
        el = np.ascontiguousarray(sorted(set(int(z) for z in elements)), np.uint16)
        self.h = self.lib.d3_init_handle_ex(_ptr(el), len(el), int(max_atoms), float(rc), float(rc_cn),
                                            float(rc_atm) if rc_atm else 0.0, int(damping), int(functional),
                                            int(table))
        if not self.h:
            raise RuntimeError("d3_init_handle_ex failed: %s" % self.lib.d3_last_error().decode())
        self.n = 0

    def set_option(self, opt, value):
        if self.lib.d3_set_option(self.h, int(opt), int(value)):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def set_functional_params(self, s6, s8, p1, p2):
        self.lib.d3_set_functional_params(self.h, s6, s8, p1, p2)

    def set_atoms(self, pos, Z):
        pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
        z = np.ascontiguousarray(Z, np.uint16)
        if self.lib.d3_set_atoms_f64(self.h, _ptr(pos), _ptr(z), len(z)):
            raise RuntimeError(self.lib.d3_last_error().decode())
        self.n = len(z)

    def set_cell(self, cell):
        c = np.ascontiguousarray(cell, np.float64).reshape(9)
        if self.lib.d3_set_cell_f64(self.h, _ptr(c)):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def compute(self, check=True):
        e = np.zeros(1)
        f = np.zeros((self.n, 3))
        s = np.zeros(9)
        st = self.lib.d3_compute_f64(self.h, _ptr(e), _ptr(f), _ptr(s))
        self.status = int(st)
        if check and st != 0:
            raise RuntimeError("d3_compute_f64 status %d: %s" % (st, self.lib.d3_last_error().decode()))
        return float(e[0]), f, s.reshape(3, 3)

    def set_positions_device(self, ptr, stream_ptr=None):
        """Positions from device memory (double [n,3], Angstrom), stream-ordered."""
        if self.lib.d3_set_positions_device(self.h, ctypes.c_void_p(ptr),
                                            ctypes.c_void_p(stream_ptr) if stream_ptr else None):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def pass_times(self):
        """Device ms per pass of the last evaluation and the work counters."""
        ms = np.zeros(8, np.float32)
        cnt = np.zeros(4, np.uint64)
        k = self.lib.d3_pass_times(self.h, _ptr(ms), 8, _ptr(cnt))
        names = ["bin", "cn", "twobody", "atm_list", "atm", "chain", "finalize"]
        return dict(zip(names, ms[:k].tolist())), cnt

    def launches_per_eval(self):
        return int(self.lib.d3_launches_per_eval(self.h))

    def compute_async(self, stream_ptr=None):
        """Enqueue one evaluation on a CUDA stream (int handle or None); no host sync."""
        return int(self.lib.d3_compute_async(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def fetch_results(self):
        """Results of the last (asynchronous) evaluation; synchronise its stream first."""
        e = np.zeros(1)
        f = np.zeros((self.n, 3))
        s = np.zeros(9)
        if self.lib.d3_fetch_results(self.h, _ptr(e), _ptr(f), _ptr(s)):
            raise RuntimeError(self.lib.d3_last_error().decode())
        return float(e[0]), f, s.reshape(3, 3)

    def device_results_ptr(self):
        return self.lib.d3_device_results(self.h)

    def copy_results_device(self, dst_ptr, stream_ptr=None):
        """Stream-ordered copy of the device results [1 + 3n + 9] (double) to dst_ptr."""
        if self.lib.d3_copy_results_device(self.h, ctypes.c_void_p(dst_ptr),
                                           ctypes.c_void_p(stream_ptr) if stream_ptr else None):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def atom_arrays(self):
        cn, g, e = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.lib.d3_debug_atom_arrays(self.h, _ptr(cn), _ptr(g), _ptr(e))
        return cn, g, e

    def fetch_status(self):
        """Status word of the last enqueued evaluation (synchronise its stream first)."""
        return int(self.lib.d3_fetch_status(self.h))

    def atm_list_capacity(self):
        return int(self.lib.d3_atm_list_capacity(self.h))

    def pass_terms(self):
        """Per-pass per-atom terms of the last evaluation ([n, 31], see d3_debug_pass_terms)."""
        t = np.zeros((self.n, 31))
        if self.lib.d3_debug_pass_terms(self.h, _ptr(t)):
            raise RuntimeError(self.lib.d3_last_error().decode())
        return t

    def atm_pairs(self):
        m = self.lib.d3_debug_atm_pairs(self.h, None, 0)
        rows = np.zeros((max(m, 1), 5), np.int64)
        k = self.lib.d3_debug_atm_pairs(self.h, _ptr(rows), m)
        return rows[:k]

    def bins(self):
        sh = np.zeros((self.n, 3), np.int64)
        b = np.zeros(self.n, np.int64)
        nb = np.zeros(3, np.int32)
        self.lib.d3_debug_bins(self.h, _ptr(sh), _ptr(b), _ptr(nb))
        return sh, b, nb

    def close(self):
        if getattr(self, "h", None):
            self.lib.free_d3_handle(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class D3Batch(_Surrogate, _Shard):
    """Many independent periodic structures in one handle (batching form)."""

    def __init__(self, elements, max_structures, max_total_atoms, rc=95.0, rc_cn=40.0, rc_atm=None,
                 damping=BJ_DAMPING, functional=0, table=TABLE_5REF):
        self.lib = load_library()
        el = np.ascontiguousarray(sorted(set(int(z) for z in elements)), np.uint16)
        self.h = self.lib.d3_init_batch(_ptr(el), len(el), int(max_structures), int(max_total_atoms), float(rc),
                                        float(rc_cn), float(rc_atm) if rc_atm else 0.0, int(damping),
                                        int(functional), int(table))
        if not self.h:
            raise RuntimeError("d3_init_batch failed: %s" % self.lib.d3_last_error().decode())
        self.counts = None

    def set_option(self, opt, value):
        if self.lib.d3_set_option(self.h, int(opt), int(value)):
            raise RuntimeError(self.lib.d3_last_error().decode())

    def set_structures(self, structures):
        """structures: list of dicts with pos [n,3], Z [n], cell [3,3] (Angstrom)."""
        counts = np.array([len(s["Z"]) for s in structures], np.uint64)
        pos = np.ascontiguousarray(np.concatenate([s["pos"] for s in structures]), np.float64)
        z = np.ascontiguousarray(np.concatenate([s["Z"] for s in structures]), np.uint16)
        cells = np.ascontiguousarray(np.stack([np.asarray(s["cell"], np.float64).reshape(9) for s in structures]))
        if self.lib.d3_set_batch_f64(self.h, len(counts), _ptr(counts), _ptr(pos), _ptr(z), _ptr(cells)):
            raise RuntimeError(self.lib.d3_last_error().decode())
        self.counts = counts

    def compute(self, check=True):
        S, n = len(self.counts), int(self.counts.sum())
        e = np.zeros(S)
        f = np.zeros((n, 3))
        s = np.zeros((S, 9))
        st = self.lib.d3_compute_batch_f64(self.h, _ptr(e), _ptr(f), _ptr(s))
        if check and st != 0:
            raise RuntimeError("d3_compute_batch_f64 status %d: %s" % (st, self.lib.d3_last_error().decode()))
        off = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        return e, [f[off[k]:off[k + 1]] for k in range(S)], s.reshape(S, 3, 3)

    def compute_async(self, stream_ptr=None):
        return int(self.lib.d3_compute_async(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def launches_per_eval(self):
        return int(self.lib.d3_launches_per_eval(self.h))

    def atm_list_capacity(self):
        return int(self.lib.d3_atm_list_capacity(self.h))

    def pass_times(self):
        ms = np.zeros(8, np.float32)
        cnt = np.zeros(4, np.uint64)
        k = self.lib.d3_pass_times(self.h, _ptr(ms), 8, _ptr(cnt))
        names = ["bin", "cn", "twobody", "atm_list", "atm", "chain", "finalize"]
        return dict(zip(names, ms[:k].tolist())), cnt

    def close(self):
        if getattr(self, "h", None):
            self.lib.free_d3_handle(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
