"""CPU checker of the learned ATM surrogate (test infrastructure only).

The surrogate has no counterpart in the reference. This module restates the engine's
surrogate in FP64 so that its kernels can be checked; only tests/ use it:

  * descriptors and the force / stress / dE/dCN chain of a per-atom energy over them
    (oracle_surrogate in d3_oracle.c, on this oracle's CN and C6);
  * the MLP ensemble: forward, input gradient and the weight gradients of the training
    loss, in numpy. The kernels' roundings are emulated (BF16 weights, inputs, hidden
    activations and backward signals; FP16 SiLU derivatives), so that a comparison
    isolates accumulation-order differences.
"""
import ctypes

import numpy as np

import oracle as orc

NRBF = 32
MU0_A, MU1_A, SIGMA_A = 0.8, 21.0, 0.7
HID = 128


def bf16(x):
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).astype(np.float64)


def fp16(x):
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float64)


def layout(nch):
    in_dim = nch * NRBF + nch
    in_pad = (in_dim + 15) // 16 * 16
    L = {"nch": nch, "in_dim": in_dim, "in_pad": in_pad}
    o = 0
    for name, size in (("oW1", in_pad * HID), ("ob1", HID), ("oW2", HID * HID), ("ob2", HID), ("oW3", HID * HID),
                       ("ob3", HID), ("ow4", HID), ("ob4", 1)):
        L[name] = o
        o += size
    L["nparam"] = (o + 3) // 4 * 4
    return L


def unpack(params, L):
    """One member's parameter vector -> (W1 [in_pad,128], b1, W2, b2, W3, b3, w4, b4)."""
    p = np.asarray(params, np.float64)
    ip = L["in_pad"]
    W1 = p[L["oW1"]:L["ob1"]].reshape(ip, HID)
    W2 = p[L["oW2"]:L["ob2"]].reshape(HID, HID)
    W3 = p[L["oW3"]:L["ob3"]].reshape(HID, HID)
    return (W1, p[L["ob1"]:L["oW2"]], W2, p[L["ob2"]:L["oW3"]], W3, p[L["ob3"]:L["ow4"]], p[L["ow4"]:L["ob4"]],
            p[L["ob4"]])


def inputs(G, center, mean, inv_std, L):
    """Network input rows as the kernel stages them (FP32 normalisation, BF16)."""
    n = G.shape[0]
    nf = L["nch"] * NRBF
    X = np.zeros((n, L["in_pad"]), np.float64)
    X[:, :nf] = (np.asarray(G, np.float32) - np.asarray(mean, np.float32)) * np.asarray(inv_std, np.float32)
    ok = np.asarray(center) >= 0
    X[np.arange(n)[ok], nf + np.asarray(center)[ok]] = 1.0
    return bf16(X)


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def _ident(x):
    return np.asarray(x, np.float64)


def forward(params, X, L, rounding=True):
    """Member forward: E [n] and the cache for the backward passes. rounding=False gives
    the exact FP64 network (for finite-difference checks of this module)."""
    rb, rh = (bf16, fp16) if rounding else (_ident, _ident)
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(params, L)
    W1, W2, W3 = rb(W1), rb(W2), rb(W3)
    w4 = np.asarray(w4, np.float32 if rounding else np.float64).astype(np.float64)
    Z1 = X @ W1 + b1
    H1, D1 = _silu(Z1)
    H1 = rb(H1)
    Z2 = H1 @ W2 + b2
    H2, D2 = _silu(Z2)
    H2 = rb(H2)
    Z3 = H2 @ W3 + b3
    H3, D3 = _silu(Z3)
    E = H3 @ w4 + b4
    return E, dict(X=X, H1=H1, H2=H2, H3=H3, D1=rh(D1), D2=rh(D2), D3=rh(D3), W1=W1, W2=W2, W3=W3, w4=w4,
                   rounding=rounding)


def backward(cache, gE):
    """Backward of a member with per-row output gradient gE: (dX [n, in_pad], dZ1, dZ2, dZ3)."""
    c = cache
    rb = bf16 if c["rounding"] else _ident
    dZ3 = rb(gE[:, None] * c["w4"][None, :] * c["D3"])
    dZ2 = rb((dZ3 @ c["W3"].T) * c["D2"])
    dZ1 = rb((dZ2 @ c["W2"].T) * c["D1"])
    dX = dZ1 @ c["W1"].T
    return dX, dZ1, dZ2, dZ3


def ensemble(model, G, center):
    """Network outputs E [members, n] and sum over members of dE/dG [n, nch*32]."""
    L = layout(len(model["channel_z"]))
    X = inputs(G, center, model["mean"], model["inv_std"], L)
    nf = L["nch"] * NRBF
    Es, dG = [], np.zeros((G.shape[0], nf))
    for m in range(model["members"]):
        E, cache = forward(model["params"][m], X, L)
        dX, _, _, _ = backward(cache, np.ones(G.shape[0]))
        Es.append(E)
        dG += dX[:, :nf] * np.asarray(model["inv_std"], np.float32)
    return np.array(Es), dG


def train_gradients(params, G, center, target, mean, inv_std, L, rounding=True):
    """Loss (mean squared error over the rows), its gradient as a parameter vector, and E."""
    X = inputs(G, center, mean, inv_std, L)
    if not rounding:
        X = np.zeros_like(X)
        nf = L["nch"] * NRBF
        X[:, :nf] = (np.asarray(G, np.float64) - mean) * inv_std
        X[np.arange(len(X)), nf + np.asarray(center)] = 1.0
    E, c = forward(params, X, L, rounding)
    B = len(E)
    gE = 2.0 * (E - target) / B
    _, dZ1, dZ2, dZ3 = backward(c, gE)
    g = np.zeros(L["nparam"])
    g[L["oW1"]:L["ob1"]] = (X.T @ dZ1).ravel()
    g[L["ob1"]:L["oW2"]] = dZ1.sum(0)
    g[L["oW2"]:L["ob2"]] = (c["H1"].T @ dZ2).ravel()
    g[L["ob2"]:L["oW3"]] = dZ2.sum(0)
    g[L["oW3"]:L["ob3"]] = (c["H2"].T @ dZ3).ravel()
    g[L["ob3"]:L["ow4"]] = dZ3.sum(0)
    g[L["ow4"]:L["ob4"]] = (bf16(c["H3"]) if rounding else c["H3"]).T @ gE
    g[L["ob4"]] = gE.sum()
    return float(np.mean((E - target) ** 2)), g, E


def _lib():
    lib, _ = orc._libs()
    if not hasattr(lib, "_surrogate_set"):
        vp, i64, ci, cd = ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_double
        lib.oracle_surrogate.restype = ci
        lib.oracle_surrogate.argtypes = [vp, i64, vp, vp, vp, vp, vp, ci, ci, cd, cd, cd, vp, vp, vp, vp, vp, ci]
        lib._surrogate_set = True
    return lib


def _params(elements, rc, rc_cn, rc_atm, extended, init_elements=None):
    uniq, c6, r0, rcv, rr4 = orc.handle_tables(init_elements if init_elements is not None else elements, extended)
    s6, s8z, s8bj, sr6, sr8, a1, a2 = orc.functional_params(0)
    prm = orc._Params(ne=len(uniq), nref=c6.shape[2], c6ab=c6.ctypes.data, r0ab=r0.ctypes.data, rcov=rcv.ctypes.data,
                      r2r4=rr4.ctypes.data, s6=s6, s8=s8bj, p1=a1, p2=a2, damping=orc.BJ_DAMPING,
                      rc=float(np.float32(rc)), rc_cn=float(np.float32(rc_cn)), rc_atm=float(np.float32(rc_atm)),
                      use_atm=1, atm_force_scaled=1, c6_mode=1, smooth_cn=0)
    return uniq, prm, (c6, r0, rcv, rr4)


def descriptors_and_chain(pos_ang, elements, cell_ang, channel_z, dEdG=None, rc=95.0, rc_cn=40.0, rc_atm=40.0,
                          extended=False, nthreads=0):
    """Descriptors G [n, nch*32] (C6 in hartree bohr^6, r in bohr) and, when dEdG is given
    (eV per descriptor unit, true sign), the forces (eV/A) and stress (eV/A^3) of that energy."""
    lib = _lib()
    pos_ang = np.asarray(pos_ang, np.float64).reshape(-1, 3)
    n = len(pos_ang)
    elements = [int(z) for z in elements]
    uniq, prm, keep = _params(elements, rc, rc_cn, rc_atm, extended)
    types = np.array([uniq.index(z) for z in elements], np.int32)
    chan = np.array([list(channel_z).index(z) if z in channel_z else -1 for z in uniq], np.int32)
    _, mcb, _ = orc.cell_box(cell_ang, rc, rc_cn)
    mcb = np.ascontiguousarray(mcb, np.int64)
    pos = np.ascontiguousarray(pos_ang * orc.ANG2BOHR)
    cell = np.ascontiguousarray(np.asarray(cell_ang, np.float64).reshape(9) * orc.ANG2BOHR)
    nch = len(channel_z)
    G = np.zeros((n, nch * NRBF))
    F = np.zeros((n, 3))
    V = np.zeros(9)
    cn = np.zeros(n)
    mu0 = MU0_A * orc.ANG2BOHR
    dmu = (MU1_A - MU0_A) / (NRBF - 1) * orc.ANG2BOHR
    sig = SIGMA_A * orc.ANG2BOHR
    g = None
    if dEdG is not None:
        # engine convention: stored energy = -E (hartree)
        g = np.ascontiguousarray(-np.asarray(dEdG, np.float64) / orc.HARTREE_EV)
    lib.oracle_surrogate(ctypes.byref(prm), ctypes.c_int64(n), pos.ctypes.data, types.ctypes.data, cell.ctypes.data,
                         mcb.ctypes.data, chan.ctypes.data, nch, NRBF, mu0, dmu, 1.0 / (2.0 * sig * sig),
                         G.ctypes.data, g.ctypes.data if g is not None else None, F.ctypes.data, V.ctypes.data,
                         cn.ctypes.data, nthreads)
    out = {"G": G, "cn": cn, "center": chan[types]}
    if g is not None:
        out["forces"] = F * orc.HARTREE_EV * orc.ANG2BOHR
        out["stress"] = (V * orc.HARTREE_EV * orc.ANG2BOHR ** 3).reshape(3, 3)
    return out


def surrogate_atm(model, pos_ang, elements, cell_ang, rc=95.0, rc_cn=40.0, rc_atm=40.0, extended=False):
    """ATM energy (eV), forces (eV/A), stress (eV/A^3) of the surrogate alone (no fallback),
    with the per-atom ensemble mean and standard deviation (eV)."""
    d = descriptors_and_chain(pos_ang, elements, cell_ang, model["channel_z"], rc=rc, rc_cn=rc_cn, rc_atm=rc_atm,
                              extended=extended)
    E, dG = ensemble(model, d["G"], d["center"])
    M = model["members"]
    e_atoms = model["e_scale"] * E.mean(0) + np.asarray(model["e_shift"])[d["center"]]
    std = model["e_scale"] * E.std(0)
    dEdG = dG * model["e_scale"] / M
    b = descriptors_and_chain(pos_ang, elements, cell_ang, model["channel_z"], dEdG=dEdG, rc=rc, rc_cn=rc_cn,
                              rc_atm=rc_atm, extended=extended)
    return {"energy": float(e_atoms.sum()), "forces": b["forces"], "stress": b["stress"], "e_atoms": e_atoms,
            "std": std, "G": d["G"], "center": d["center"]}
