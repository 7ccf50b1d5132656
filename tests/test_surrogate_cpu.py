"""Learned ATM surrogate, host side: parameter layout shared by the library, the model
file and the CPU checker; model file round trip; the CPU checker's own derivatives
against finite differences (so that it can check the kernels' gradients)."""
import os

import numpy as np
import pytest

import d3_surrogate as SU
import surrogate_oracle as SO


@pytest.mark.parametrize("nch", [1, 5, 6, 8])
def test_layout_agrees_with_library(nch):
    a, b, c = SU.layout(nch), SU.layout_py(nch), SO.layout(nch)
    for k in ("in_dim", "in_pad", "oW1", "ob1", "oW2", "ob2", "oW3", "ob3", "ow4", "ob4", "nparam"):
        assert a[k] == b[k] == c[k], k
    assert a["in_pad"] % 16 == 0 and a["in_pad"] >= 33 * nch


def test_layout_rejects_bad_channel_counts():
    lib = SU.load_library()
    out = np.zeros(12, np.uint64)
    assert lib.d3_mlp_layout(0, out.ctypes.data) != 0
    assert lib.d3_mlp_layout(9, out.ctypes.data) != 0


def test_model_file_round_trip(tmp_path):
    m = SU.Model.init(SU.CHANNELS_HCNOSICU, members=3, seed=5)
    rng = np.random.default_rng(0)
    m.mean = rng.normal(size=m.mean.shape).astype(np.float32)
    m.inv_std = rng.uniform(0.5, 2, size=m.inv_std.shape).astype(np.float32)
    m.e_shift = rng.normal(size=m.nch).astype(np.float32)
    m.e_scale = 1.25e-3
    m.params += rng.normal(scale=0.01, size=m.params.shape).astype(np.float32)
    m.meta = {"note": "round trip"}
    p = os.path.join(tmp_path, "m.d3s")
    m.save(p)
    r = SU.Model.load(p)
    L = SU.layout_py(m.nch)
    assert r.channel_z == m.channel_z and r.members == 3 and r.e_scale == m.e_scale
    np.testing.assert_array_equal(r.mean, m.mean)
    np.testing.assert_array_equal(r.inv_std, m.inv_std)
    np.testing.assert_array_equal(r.e_shift, m.e_shift)
    for o0, o1 in ((L["oW1"], L["ob1"]), (L["oW2"], L["ob2"]), (L["oW3"], L["ob3"])):
        # weight matrices are stored in BF16: exactly the kernels' rounding of them
        np.testing.assert_array_equal(r.params[:, o0:o1], SO.bf16(m.params[:, o0:o1]).astype(np.float32))
    for o0, o1 in ((L["ob1"], L["oW2"]), (L["ob2"], L["oW3"]), (L["ob3"], L["ow4"]), (L["ow4"], L["ob4"] + 1)):
        np.testing.assert_array_equal(r.params[:, o0:o1], m.params[:, o0:o1])
    assert r.meta["note"] == "round trip"
    with open(p, "r+b") as f:
        f.write(b"XXXXXXXX")
    with pytest.raises(ValueError):
        SU.Model.load(p)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-5, 65504.0], np.float32)
    r = SO.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0  # tie -> even
    assert r[2] == 1.0 + 4 * 2 ** -8  # tie -> even (up)
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-5) / 3.0e-5 < 2 ** -8
    assert r[5] == 65536.0


def _small_model(nch=2, seed=0):
    m = SU.Model.init(list(range(1, nch + 1)), members=1, seed=seed)
    rng = np.random.default_rng(seed)
    m.params += rng.normal(scale=0.05, size=m.params.shape).astype(np.float32)
    return m


def test_oracle_weight_gradients_match_finite_differences():
    m = _small_model()
    L = SO.layout(m.nch)
    rng = np.random.default_rng(1)
    n = 24
    G = rng.normal(size=(n, m.nch * 32))
    center = rng.integers(0, m.nch, n)
    target = rng.normal(size=n)
    mean, istd = np.zeros(m.nch * 32), np.ones(m.nch * 32)
    p = m.params[0].astype(np.float64)
    loss, g, _ = SO.train_gradients(p, G, center, target, mean, istd, L, rounding=False)
    h = 1e-6
    for k in list(rng.choice(L["ob4"] + 1, 25, replace=False)) + [L["ob4"], L["ow4"], L["ob1"], L["oW2"] + 7]:
        q = p.copy()
        q[k] += h
        lp = SO.train_gradients(q, G, center, target, mean, istd, L, rounding=False)[0]
        q[k] -= 2 * h
        lm = SO.train_gradients(q, G, center, target, mean, istd, L, rounding=False)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * (abs(fd) + 1e-3), (k, fd, g[k])


def test_oracle_input_gradient_matches_finite_differences():
    m = _small_model(seed=3)
    L = SO.layout(m.nch)
    rng = np.random.default_rng(2)
    n = 5
    nf = m.nch * 32
    X = np.zeros((n, L["in_pad"]))
    X[:, :nf] = rng.normal(size=(n, nf))
    X[np.arange(n), nf + rng.integers(0, m.nch, n)] = 1.0
    p = m.params[0].astype(np.float64)
    E, c = SO.forward(p, X, L, rounding=False)
    dX = SO.backward(c, np.ones(n))[0]
    h = 1e-6
    for r in range(n):
        for f in rng.choice(nf, 6, replace=False):
            Xp = X.copy()
            Xp[r, f] += h
            Xm = X.copy()
            Xm[r, f] -= h
            fd = (SO.forward(p, Xp, L, rounding=False)[0][r] - SO.forward(p, Xm, L, rounding=False)[0][r]) / (2 * h)
            assert abs(fd - dX[r, f]) <= 1e-6 * (abs(fd) + 1e-3)


def test_oracle_descriptor_chain_matches_finite_differences():
    """Forces and stress of a linear energy E = sum w . G over the oracle's descriptors
    (C6 through CN included) against central differences of E."""
    rng = np.random.default_rng(4)
    cell = np.array([[6.2, 0.0, 0.0], [0.4, 5.9, 0.0], [-0.3, 0.5, 6.4]])
    n = 8
    pos = rng.uniform(0, 1, (n, 3)) @ cell
    Z = np.array([1, 6, 8, 6, 1, 29, 8, 1])
    ch = (1, 6, 8, 29)
    kw = dict(rc=20.0, rc_cn=20.0, rc_atm=20.0)
    w = rng.normal(size=(n, len(ch) * 32)) * 1e-4  # eV per descriptor unit

    def energy(p, c=cell):
        G = SO.descriptors_and_chain(p, Z, c, ch, **kw)["G"]
        return float((w * G).sum())

    out = SO.descriptors_and_chain(pos, Z, cell, ch, dEdG=w, **kw)
    h = 1e-5
    for i in range(n):
        for k in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[i, k] += h
            pm[i, k] -= h
            fd = -(energy(pp) - energy(pm)) / (2 * h)
            assert abs(fd - out["forces"][i, k]) <= 1e-6 * (abs(fd) + 1e-4), (i, k, fd, out["forces"][i, k])
    # stress: sigma_ab = (1/V) dE/d(eps_ab), symmetric strain x -> (I + eps) x on cell and positions
    V = abs(np.linalg.det(cell))
    for a, b in ((0, 0), (1, 1), (2, 2), (0, 1), (1, 2)):
        eps = np.zeros((3, 3))
        eps[a, b] = eps[b, a] = h
        Ep = energy(pos @ (np.eye(3) + eps), cell @ (np.eye(3) + eps))
        Em = energy(pos @ (np.eye(3) - eps), cell @ (np.eye(3) - eps))
        fd = (Ep - Em) / (2 * h) / V / (1.0 if a == b else 2.0)
        assert abs(fd - out["stress"][a, b]) <= 1e-5 * (abs(fd) + 1e-6), (a, b, fd, out["stress"][a, b])
