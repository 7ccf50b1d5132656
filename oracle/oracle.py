"""Python side of the FP64 CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module,
as the checker. It restates the host-side logic of the reference around the kernels:

  * unique element list, sorted ascending (Unique_Elements, src/d3_buffer.cu:86-126)
    and the per-handle gather of the parameter tables (src/d3_buffer.cu:193-277);
  * Angstrom -> bohr on input and hartree/bohr -> eV/Angstrom on output
    (src/d3.cu:49-60, 78-85, 203-219), here in double precision;
  * functional parameters (src/d3_types.h:46-54) and damping selection
    (src/d3_kernel.cu:1139-1152);
  * the image box / workload decision of set_cell (src/d3_buffer.cu:431-477).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(HERE, "_build", "libd3_oracle.so")
_TABLE_SO = os.path.join(HERE, "_build", "libd3_tables.so")

BOHR_ANG = 0.52917726  # src/d3.cu:50
ANG2BOHR = 1.0 / BOHR_ANG
HARTREE_EV = 27.211396641308  # src/d3.cu:205

ZERO_DAMPING, BJ_DAMPING = 0, 1
FUNCTIONALS = {"PBE": 0, "PBE0": 1, "B3LYP": 2, "BLYP": 3, "BP86": 4, "REVPBE": 5, "CUSTOM": 99}
# (s6, s8_zero, s8_bj, sr6, sr8, a1, a2), src/d3_types.h:46-54, stored as float there
_FP = [
    (1.0, 0.722, 0.7875, 1.217, 1.0, 0.4289, 4.4407),
    (1.0, 0.928, 1.2177, 1.287, 1.0, 0.4145, 4.8593),
    (1.0, 1.703, 1.9889, 1.261, 1.0, 0.3981, 4.4211),
    (1.0, 1.682, 2.6996, 1.094, 1.0, 0.4298, 4.2359),
    (1.0, 1.683, 3.2822, 1.139, 1.0, 0.3946, 4.8516),
    (1.0, 1.010, 2.3550, 0.923, 1.0, 0.5238, 3.5016),
    (1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0),
]


def functional_params(functional: int):
    """Float-rounded functional parameters, as the reference stores them (real_t)."""
    idx = 6 if functional == 99 else functional
    return tuple(float(np.float32(v)) for v in _FP[idx])


def _build():
    os.makedirs(os.path.dirname(_SO), exist_ok=True)
    src = os.path.join(HERE, "d3_oracle.c")
    if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", src, "-o", _SO, "-lm"])
    tsrc = os.path.join(HERE, "tables.c")
    hdr = os.path.join(HERE, "..", "lasp-d3_b200", "csrc", "d3_synth_params.h")
    if (not os.path.exists(_TABLE_SO) or os.path.getmtime(_TABLE_SO) < max(os.path.getmtime(tsrc),
                                                                            os.path.getmtime(hdr))):
        subprocess.check_call(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", tsrc, "-o", _TABLE_SO, "-lm"])


def build():
    _build()
    return _SO


class _Params(ctypes.Structure):
    _fields_ = [
        ("ne", ctypes.c_int), ("nref", ctypes.c_int),
        ("c6ab", ctypes.c_void_p), ("r0ab", ctypes.c_void_p), ("rcov", ctypes.c_void_p), ("r2r4", ctypes.c_void_p),
        ("s6", ctypes.c_double), ("s8", ctypes.c_double), ("p1", ctypes.c_double), ("p2", ctypes.c_double),
        ("damping", ctypes.c_int),
        ("rc", ctypes.c_double), ("rc_cn", ctypes.c_double), ("rc_atm", ctypes.c_double),
        ("use_atm", ctypes.c_int), ("atm_force_scaled", ctypes.c_int), ("c6_mode", ctypes.c_int),
        ("smooth_cn", ctypes.c_int),
    ]


class _Out(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_void_p), ("forces", ctypes.c_void_p), ("virial", ctypes.c_void_p),
                ("cn", ctypes.c_void_p), ("dedcn", ctypes.c_void_p)]


_lib = None
_tlib = None


def _libs():
    global _lib, _tlib
    if _lib is None:
        _build()
        _lib = ctypes.CDLL(_SO)
        vp, i64 = ctypes.c_void_p, ctypes.c_int64
        _lib.oracle_compute.restype = ctypes.c_int
        _lib.oracle_compute.argtypes = [vp, i64, vp, vp, vp, vp, vp, i64, ctypes.c_int, vp]
        _lib.oracle_terms.restype = ctypes.c_int
        _lib.oracle_terms.argtypes = [vp, i64, vp, vp, vp, vp, vp, i64, vp, ctypes.c_int, vp, vp]
        _lib.oracle_counts.restype = ctypes.c_int
        _lib.oracle_counts.argtypes = [vp, i64, vp, vp, vp, ctypes.c_int, vp]
        _lib.oracle_cell_box.restype = ctypes.c_int
        _lib.oracle_cell_box.argtypes = [vp, ctypes.c_float, ctypes.c_float, vp, vp]
        _lib.oracle_grid_assign.restype = None
        _lib.oracle_grid_assign.argtypes = [vp, i64, vp, vp, vp, vp]
        _tlib = ctypes.CDLL(_TABLE_SO)
        _tlib.oracle_synth_tables.restype = None
        _tlib.oracle_synth_tables.argtypes = [ctypes.c_int, vp, vp, vp, vp]
    return _lib, _tlib


_TABLES = {}


def full_tables(extended=False):
    """The whole synthetic table (all element slots), from the shared generator."""
    if extended in _TABLES:
        return _TABLES[extended]
    _, tl = _libs()
    ne, nr = (103, 7) if extended else (95, 5)
    c6 = np.zeros((ne, ne, nr, nr, 3), np.float32)
    r0 = np.zeros((ne, ne), np.float32)
    rc = np.zeros(ne, np.float32)
    rr = np.zeros(ne, np.float32)
    tl.oracle_synth_tables(ctypes.c_int(1 if extended else 0), c6.ctypes.data, r0.ctypes.data, rc.ctypes.data,
                           rr.ctypes.data)
    _TABLES[extended] = (c6, r0, rc, rr)
    return _TABLES[extended]


def handle_tables(elements, extended=False):
    """Per-handle tables for the sorted unique element list (src/d3_buffer.cu:86-277)."""
    c6, r0, rc, rr = full_tables(extended)
    uniq = sorted(set(int(z) for z in elements))
    idx = [z - 1 if extended else z for z in uniq]
    ix = np.array(idx)
    return (uniq, np.ascontiguousarray(c6[np.ix_(ix, ix)]), np.ascontiguousarray(r0[np.ix_(ix, ix)]),
            np.ascontiguousarray(rc[ix]), np.ascontiguousarray(rr[ix]))


def cell_box(cell_ang, rc, rc_cn):
    """Reference image box and workload mode from the float cell (set_cell path)."""
    lib, _ = _libs()
    # reference: bohr_cell = cell * (1.0f / 0.52917726f), float multiply
    f = np.float32(1.0) / np.float32(BOHR_ANG)
    cell_f = (np.asarray(cell_ang, np.float32).reshape(9) * f).astype(np.float32)
    mcb = np.zeros(3, np.int64)
    ng = np.zeros(3, np.int64)
    mode = lib.oracle_cell_box(cell_f.ctypes.data, ctypes.c_float(rc), ctypes.c_float(rc_cn), mcb.ctypes.data,
                               ng.ctypes.data)
    return int(mode), mcb, ng


def grid_assign(cell_ang, pos_ang_f32, num_grid):
    """Host cell-list assignment of construct_grids, from float inputs."""
    lib, _ = _libs()
    f = np.float32(1.0) / np.float32(BOHR_ANG)
    cell_f = (np.asarray(cell_ang, np.float32).reshape(9) * f).astype(np.float32)
    pos_f = (np.asarray(pos_ang_f32, np.float32).reshape(-1) * f).astype(np.float32)
    n = pos_f.size // 3
    gi = np.zeros(n, np.int64)
    si = np.zeros((n, 3), np.int64)
    ng = np.ascontiguousarray(num_grid, np.int64)
    lib.oracle_grid_assign(cell_f.ctypes.data, ctypes.c_int64(n), pos_f.ctypes.data, ng.ctypes.data, gi.ctypes.data,
                           si.ctypes.data)
    return gi, si


def _setup(pos_ang, elements, cell_ang, rc, rc_cn, rc_atm, damping, functional, init_elements, extended,
           atm_force_scaled, c6_mode, smooth_cn, mcb):
    """Per-handle tables, parameter block, bohr positions and cell, image box."""
    pos_ang = np.asarray(pos_ang, np.float64).reshape(-1, 3)
    elements = [int(z) for z in elements]
    uniq, c6, r0, rcv, rr4 = handle_tables(init_elements if init_elements is not None else elements, extended)
    types = np.array([uniq.index(z) for z in elements], np.int32)
    s6, s8z, s8bj, sr6, sr8, a1, a2 = functional_params(functional)
    if damping == BJ_DAMPING:
        s8, p1, p2 = s8bj, a1, a2
    else:
        s8, p1, p2 = s8z, sr6, sr8
    if mcb is None:
        _, mcb, _ = cell_box(cell_ang, rc, rc_cn)
    mcb = np.ascontiguousarray(mcb, np.int64)
    prm = _Params(ne=len(uniq), nref=c6.shape[2], c6ab=c6.ctypes.data, r0ab=r0.ctypes.data, rcov=rcv.ctypes.data,
                  r2r4=rr4.ctypes.data, s6=s6, s8=s8, p1=p1, p2=p2, damping=int(damping),
                  rc=float(np.float32(rc)), rc_cn=float(np.float32(rc_cn)),
                  rc_atm=float(np.float32(rc_atm)) if rc_atm is not None else 0.0,
                  use_atm=1 if rc_atm is not None else 0, atm_force_scaled=1 if atm_force_scaled else 0,
                  c6_mode=int(c6_mode), smooth_cn=1 if smooth_cn else 0)
    pos = np.ascontiguousarray(pos_ang * ANG2BOHR)
    cell = np.ascontiguousarray(np.asarray(cell_ang, np.float64).reshape(9) * ANG2BOHR)
    # the arrays the parameter block points into must outlive the call
    keep = (c6, r0, rcv, rr4)
    return prm, keep, types, pos, cell, mcb


def compute(pos_ang, elements, cell_ang, rc=95.0, rc_cn=40.0, rc_atm=None, damping=BJ_DAMPING, functional=0,
            init_elements=None, extended=False, atm_force_scaled=False, c6_mode=0, smooth_cn=False, nthreads=0,
            subset=None, mcb=None, raw=False):
    """FP64 oracle evaluation.

    pos_ang: [n,3] Angstrom (converted to bohr in double); cell_ang: 3x3 rows = vectors.
    Cutoffs in bohr (passed through unconverted, as in the reference ABI).
    Returns dict with energy (eV), forces (eV/A, caller order), stress (eV/A^3, 3x3),
    plus cn and dedcn (internal units) and the image box used.
    """
    lib, _ = _libs()
    prm, keep, types, pos, cell, mcb = _setup(pos_ang, elements, cell_ang, rc, rc_cn, rc_atm, damping, functional,
                                              init_elements, extended, atm_force_scaled, c6_mode, smooth_cn, mcb)
    n = len(types)
    e = np.zeros(n)
    f = np.zeros((n, 3))
    v = np.zeros(9)
    cn = np.zeros(n)
    g = np.zeros(n)
    out = _Out(energy=e.ctypes.data, forces=f.ctypes.data, virial=v.ctypes.data, cn=cn.ctypes.data, dedcn=g.ctypes.data)
    if subset is not None:
        sub = np.ascontiguousarray(subset, np.int64)
        sp, ns = sub.ctypes.data, len(sub)
    else:
        sub, sp, ns = None, None, 0
    lib.oracle_compute(ctypes.byref(prm), ctypes.c_int64(n), pos.ctypes.data, types.ctypes.data, cell.ctypes.data,
                       mcb.ctypes.data, ctypes.c_void_p(sp), ctypes.c_int64(ns), ctypes.c_int(nthreads),
                       ctypes.byref(out))
    res = {"cn": cn, "dedcn": g, "mcb": mcb, "energy_atoms_hartree": e}
    if raw:
        res.update(energy_hartree=e.sum(), forces_raw=f, virial_raw=v)
    res["energy"] = -e.sum() * HARTREE_EV
    res["forces"] = f * HARTREE_EV * ANG2BOHR
    res["stress"] = (v * HARTREE_EV * ANG2BOHR ** 3).reshape(3, 3)
    return res


def terms(pos_ang, elements, cell_ang, subset, rc=95.0, rc_cn=40.0, rc_atm=None, damping=BJ_DAMPING, functional=0,
          extended=False, dedcn=None, c6_mode=1, nthreads=0, mcb=None):
    """Per-pass per-atom terms of the atoms in `subset` ([len(subset), 31], the column
    layout of the engine's d3_debug_pass_terms, hartree and bohr) and the CN of every
    atom. dedcn: complete dE/dCN of every atom for the chain-rule columns (else zero)."""
    lib, _ = _libs()
    prm, keep, types, pos, cell, mcb = _setup(pos_ang, elements, cell_ang, rc, rc_cn, rc_atm, damping, functional,
                                              None, extended, False, c6_mode, False, mcb)
    n = len(types)
    sub = np.ascontiguousarray(subset, np.int64)
    cn = np.zeros(n)
    t = np.zeros((len(sub), 31))
    g = None if dedcn is None else np.ascontiguousarray(dedcn, np.float64)
    lib.oracle_terms(ctypes.byref(prm), ctypes.c_int64(n), pos.ctypes.data, types.ctypes.data, cell.ctypes.data,
                     mcb.ctypes.data, sub.ctypes.data, ctypes.c_int64(len(sub)),
                     ctypes.c_void_p(None if g is None else g.ctypes.data), ctypes.c_int(nthreads), cn.ctypes.data,
                     t.ctypes.data)
    return t, cn


def counts(pos_ang, cell_ang, rc=95.0, rc_cn=40.0, rc_atm=None, nthreads=0, mcb=None):
    """Exact counts of the reference enumeration over every atom: (CN ordered pairs,
    two-body ordered pairs, ATM triplets)."""
    lib, _ = _libs()
    pos_ang = np.asarray(pos_ang, np.float64).reshape(-1, 3)
    n = pos_ang.shape[0]
    prm, keep, types, pos, cell, mcb = _setup(pos_ang, [1] * n, cell_ang, rc, rc_cn, rc_atm, BJ_DAMPING, 0, None,
                                              False, False, 0, False, mcb)
    out = np.zeros(3, np.int64)
    lib.oracle_counts(ctypes.byref(prm), ctypes.c_int64(n), pos.ctypes.data, cell.ctypes.data, mcb.ctypes.data,
                      ctypes.c_int(nthreads), out.ctypes.data)
    return tuple(int(x) for x in out)


def cell_list_pairs(cell_ang, pos_ang, rc, rc_cn, r2max, inclusive):
    """The pair set of the reference's CELL_LIST path (test infrastructure): the grid of
    set_cell (counts floor(1 / |row k of the cell inverse| / max(rc, rc_CN)),
    src/d3_buffer.cu:443-461), atoms wrapped and binned as construct_grids does
    (:496-634, here through grid_assign), and for each atom the 27 neighbouring grid cells
    with their periodic shift flags (calculate_neighboring_grids, src/d3_kernel.cu:437-485).
    Returns the set of (i, j, Tx, Ty, Tz) with 0 < r^2 < r2max (<= when inclusive), T the
    lattice shift in the positions as given: r = x_i - (x_j + T h)."""
    mode, mcb, ng = cell_box(cell_ang, rc, rc_cn)
    if mode != 1:
        raise ValueError("not a cell-list box (grid %s)" % (ng.tolist(),))
    pos32 = np.asarray(pos_ang, np.float32).reshape(-1, 3)
    gi, si = grid_assign(cell_ang, pos32, ng)
    f = np.float32(1.0) / np.float32(BOHR_ANG)
    cell = (np.asarray(cell_ang, np.float32).reshape(3, 3) * f).astype(np.float64)
    pos = (pos32 * f).astype(np.float32).astype(np.float64)
    wrapped = pos - si @ cell
    g3 = np.stack([gi % ng[0], (gi // ng[0]) % ng[1], gi // (ng[0] * ng[1])], 1)
    by_cell = {}
    for i, g in enumerate(gi.tolist()):
        by_cell.setdefault(g, []).append(i)
    out = set()
    for i in range(len(pos)):
        for oz in (-1, 0, 1):
            for oy in (-1, 0, 1):
                for ox in (-1, 0, 1):
                    nb = g3[i] + np.array([ox, oy, oz])
                    S = np.where(nb < 0, -1, np.where(nb >= ng, 1, 0))
                    nb = nb - S * ng
                    for j in by_cell.get(int(nb[0] + nb[1] * ng[0] + nb[2] * ng[0] * ng[1]), []):
                        d = wrapped[i] - (wrapped[j] + S @ cell)
                        d2 = float(d @ d)
                        if d2 > 0.0 and (d2 <= r2max if inclusive else d2 < r2max):
                            T = S + si[i] - si[j]
                            out.add((i, j, int(T[0]), int(T[1]), int(T[2])))
    return out


def all_pairs(cell_ang, pos_ang, r2max, inclusive, reach=(2, 2, 2), float_input=True):
    """Every (i, j, T) with 0 < r^2 < r2max (<= when inclusive) over the images
    T in [-reach, reach] per direction of the positions as given; bohr from Angstrom in
    float as the reference's float ABI converts them (float_input), else in double as
    the FP64 oracle does."""
    if float_input:
        f = np.float32(1.0) / np.float32(BOHR_ANG)
        cell = (np.asarray(cell_ang, np.float32).reshape(3, 3) * f).astype(np.float64)
        pos = (np.asarray(pos_ang, np.float32).reshape(-1, 3) * f).astype(np.float32).astype(np.float64)
    else:
        cell = np.asarray(cell_ang, np.float64).reshape(3, 3) * ANG2BOHR
        pos = np.asarray(pos_ang, np.float64).reshape(-1, 3) * ANG2BOHR
    reach = np.broadcast_to(np.asarray(reach, int), (3,))
    T = np.array([(x, y, z) for z in range(-reach[2], reach[2] + 1) for y in range(-reach[1], reach[1] + 1)
                  for x in range(-reach[0], reach[0] + 1)])
    sh = T @ cell
    out = set()
    for i in range(len(pos)):
        d = pos[i][None, None, :] - (pos[None, :, :] + sh[:, None, :])
        d2 = (d * d).sum(-1)
        ok = (d2 > 0.0) & ((d2 <= r2max) if inclusive else (d2 < r2max))
        for t, j in zip(*np.nonzero(ok)):
            out.add((i, int(j), *T[t].tolist()))
    return out
