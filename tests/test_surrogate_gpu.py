"""Learned ATM surrogate on the GPU against the CPU checker.

  * descriptors (FP32 kernel) against the FP64 oracle's;
  * per-atom exact ATM labels: they sum to the ATM energy and match the oracle's E/3 shares;
  * the fused MLP kernel (BF16 tensor-core GEMMs, FP32 accumulation): outputs and input
    gradients against the numpy network with the same roundings;
  * the training kernels: loss, outputs and every parameter gradient of one batch;
  * training on the GPU lowers the loss on held-out atoms;
  * the whole surrogate path (threshold = infinity): energy, forces and stress against
    the oracle's two-body + surrogate; with threshold 0 every atom falls back and the
    result equals the exact ATM path; a threshold in between partitions the energy into
    surrogate and exact per-atom shares exactly.
"""
import numpy as np
import pytest

import d3_surrogate as SU
import d3_systems as S
import oracle
import surrogate_oracle as SO
from d3_b200 import D3, OPT_ATM_FORCE_SCALED, OPT_ATM_SURROGATE, OPT_PRECISION

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
CH = SU.CHANNELS_HCNOSICU


def mixed_box(n, seed, edge=None):
    comp = (("H", 0.3), ("C", 0.25), ("N", 0.1), ("O", 0.15), ("Si", 0.1), ("Cu", 0.1))
    L = edge or (n / 0.1) ** (1.0 / 3.0)
    cell = L * np.array([[1.0, 0.0, 0.0], [0.06, 1.0, 0.0], [-0.04, 0.05, 1.0]])
    return S.random_box(n, cell, composition=comp, seed=seed)


def random_model(seed=0, members=4, scale=1.0):
    """A model with random weights and a normalisation fitted to real descriptors."""
    m = SU.Model.init(CH, members=members, seed=seed)
    rng = np.random.default_rng(seed)
    L = SU.layout_py(len(CH))
    m.params[:, L["ob1"]:L["oW2"]] = rng.normal(scale=0.1, size=(members, 128))
    m.params[:, L["ob4"]] = rng.normal(scale=0.1, size=members)
    m.e_scale = 1e-3 * scale
    m.e_shift = rng.normal(scale=1e-3, size=len(CH)).astype(np.float32)
    return m


def handle_for(sys_, precision=0, rc=95.0):
    d = D3(sys_["Z"], len(sys_["Z"]), rc=rc, rc_cn=40.0, rc_atm=40.0)
    d.set_option(OPT_PRECISION, precision)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    return d


def fit_norm(model, G):
    g = G.double().cpu().numpy()
    model.mean = g.mean(0).astype(np.float32)
    sd = g.std(0)
    model.inv_std = np.where(sd > 0, 1.0 / np.maximum(sd, 1e-30), 1.0).astype(np.float32)


@pytest.fixture(scope="module")
def small():
    sys_ = mixed_box(96, seed=11)
    d = handle_for(sys_)
    d.compute()
    G, c, e = SU.descriptors_of(d, CH)
    return sys_, d, G, c, e


def test_descriptors_match_oracle(small):
    sys_, d, G, c, e = small
    ref = SO.descriptors_and_chain(sys_["pos"], sys_["Z"], sys_["cell"], CH)
    g = G.double().cpu().numpy()
    assert np.array_equal(c.cpu().numpy(), ref["center"])
    scale = np.abs(ref["G"]).max()
    err = np.abs(g - ref["G"]).max()
    assert err <= 2e-6 * scale, (err, scale)
    assert (g >= 0).all()


def test_descriptors_small_cell_many_images():
    # 12 atoms in a 5 A cell: thousands of images inside rc_ATM
    sys_ = mixed_box(12, seed=5, edge=5.0)
    d = handle_for(sys_)
    d.compute()
    G, c, _ = SU.descriptors_of(d, CH)
    ref = SO.descriptors_and_chain(sys_["pos"], sys_["Z"], sys_["cell"], CH)
    err = np.abs(G.double().cpu().numpy() - ref["G"]).max()
    assert err <= 2e-6 * np.abs(ref["G"]).max()


def test_atom_labels_partition_atm_energy(small):
    sys_, d, G, c, e = small
    ea = e.cpu().numpy()
    e_atm, _, _ = d.compute()
    d0 = D3(sys_["Z"], len(sys_["Z"]), rc=95.0, rc_cn=40.0, rc_atm=None)
    d0.set_cell(sys_["cell"])
    d0.set_atoms(sys_["pos"], sys_["Z"])
    e_two, _, _ = d0.compute()
    assert abs(ea.sum() - (e_atm - e_two)) <= 1e-9 * abs(e_atm - e_two) + 1e-12
    # oracle per-atom ATM shares: per-atom energies with ATM minus without
    kw = dict(rc=95.0, rc_cn=40.0, c6_mode=1)
    a = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc_atm=40.0, **kw)["energy_atoms_hartree"]
    b = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc_atm=None, **kw)["energy_atoms_hartree"]
    ref = -(a - b) * oracle.HARTREE_EV
    assert np.abs(ea - ref).max() <= 1e-9 * np.abs(ref).max() + 1e-14


def test_mlp_forward_and_input_gradient_match_oracle(small):
    _, _, G, c, _ = small
    model = random_model(seed=1)
    fit_norm(model, G)
    e, dG = SU.predict(model, G, c, with_grad=True)
    E_ref, dG_ref = SO.ensemble(model.as_dict(), G.double().cpu().numpy(), c.cpu().numpy())
    E_gpu = ((e - torch.as_tensor(model.e_shift, device="cuda").double()[c.long()][None, :]) / model.e_scale).cpu().numpy()
    assert np.abs(E_gpu - E_ref).max() <= 2e-3 * (np.abs(E_ref).max() + 1e-3)
    g = dG.cpu().numpy() * model.members / model.e_scale
    assert np.abs(g - dG_ref).max() <= 5e-3 * np.abs(dG_ref).max()
    # row-count edge cases: one row, and a count that is not a multiple of the tile
    for rows in (1, 130):
        e1 = SU.predict(model, G[:rows].contiguous(), c[:rows].contiguous())
        assert torch.allclose(e1, e[:, :rows], rtol=0, atol=1e-12)


def test_mlp_train_batch_gradients_match_oracle(small):
    _, _, G, c, e = small
    lib = SU.load_library()
    model = random_model(seed=2, members=2)
    fit_norm(model, G)
    L = SU.layout(len(CH))
    B = 256
    rng = np.random.default_rng(0)
    idx = np.stack([rng.choice(G.shape[0], B) for _ in range(2)]).astype(np.int32)
    target = (e.cpu().numpy() / 1e-3).astype(np.float32)
    tr = SU.Trainer(model, G, c, torch.as_tensor(target), np.arange(G.shape[0]), batch=B)
    idx_d = torch.as_tensor(idx, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    assert lib.d3_mlp_train_batch(len(CH), 2, tr.params.data_ptr(), tr.packed.data_ptr(), tr.mean.data_ptr(),
                                  tr.inv_std.data_ptr(), G.data_ptr(), c.data_ptr(), tr.target.data_ptr(),
                                  idx_d.data_ptr(), B, tr.E.data_ptr(), tr.acts.data_ptr(), tr.partial.data_ptr(),
                                  tr.loss.data_ptr(), s) == 0
    torch.cuda.synchronize()
    P = tr.partial.view(2, B // 128, -1).sum(1).double().cpu().numpy()
    Gn, cn = G.double().cpu().numpy(), c.cpu().numpy()
    for m in range(2):
        loss, g, E = SO.train_gradients(model.params[m].astype(np.float64), Gn[idx[m]], cn[idx[m]],
                                        target[idx[m]].astype(np.float64), model.mean, model.inv_std, SO.layout(6))
        Eg = tr.E.view(2, B)[m].double().cpu().numpy()
        assert np.abs(Eg - E).max() <= 2e-3 * (np.abs(E).max() + 1e-3)
        lg = tr.loss.view(2, -1)[m].double().sum().item() / B
        assert abs(lg - loss) <= 2e-3 * loss + 1e-9
        for o0, o1 in ((L["oW1"], L["ob1"]), (L["ob1"], L["oW2"]), (L["oW2"], L["ob2"]), (L["ob2"], L["oW3"]),
                       (L["oW3"], L["ob3"]), (L["ob3"], L["ow4"]), (L["ow4"], L["ob4"]), (L["ob4"], L["ob4"] + 1)):
            ref = g[o0:o1]
            err = np.abs(P[m, o0:o1] - ref).max()
            assert err <= 1e-2 * np.abs(ref).max() + 1e-9, (o0, err, np.abs(ref).max())


def test_training_on_gpu_lowers_heldout_error():
    structs = S.batch_structs(count=48, seed=21, nmin=16, nmax=400)
    G, c, e, sid = SU.label_structures(structs, CH)
    rows = np.arange(G.shape[0])
    val = rows[sid >= 40]
    tr = rows[sid < 40]
    model, hist = SU.train(G, c, e, tr, val, CH, members=2, epochs=30, batch=512, lr=3e-3, seed=0)
    y = e.cpu().numpy()
    base = np.sqrt(np.mean((y[val] - model.e_shift[c.cpu().numpy()[val]]) ** 2))
    assert hist[-1]["val_rmse_ev"] < 0.6 * base, (hist[-1], base)
    assert hist[-1]["val_rmse_ev"] < hist[0]["val_rmse_ev"]


def run_with(sys_, model, threshold, precision=0, force_scaled=False):
    d = handle_for(sys_, precision)
    if force_scaled:
        d.set_option(OPT_ATM_FORCE_SCALED, 1)
    if model is not None:
        d.set_surrogate(model, threshold_ev=threshold)
    e, f, s = d.compute()
    flagged = d.surrogate_flagged() if model is not None else 0
    return e, f, s, flagged, d


@pytest.fixture(scope="module")
def box128():
    sys_ = mixed_box(128, seed=3)
    d = handle_for(sys_)
    d.compute()
    G, c, _ = SU.descriptors_of(d, CH)
    model = random_model(seed=4)
    fit_norm(model, G)
    return sys_, model


def test_surrogate_path_matches_oracle(box128):
    sys_, model = box128
    e, f, s, flagged, _ = run_with(sys_, model, threshold=1e9)
    assert flagged == 0
    two = oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], rc=95.0, rc_cn=40.0, rc_atm=None, c6_mode=1)
    sur = SO.surrogate_atm(model.as_dict(), sys_["pos"], sys_["Z"], sys_["cell"])
    E = two["energy"] + sur["energy"]
    F = two["forces"] + sur["forces"]
    St = two["stress"] + sur["stress"]
    assert abs(e - E) <= 1e-4 * abs(sur["energy"]) + 1e-7, (e, E)
    fs = np.abs(sur["forces"]).max()
    assert np.abs(f - F).max() <= 5e-3 * fs + 1e-7, (np.abs(f - F).max(), fs)
    ss = np.abs(sur["stress"]).max()
    assert np.abs(s - St).max() <= 5e-3 * ss + 1e-9
    assert np.abs(f.sum(0)).max() <= 1e-9 * len(f) * (np.abs(f).max() + 1)


@pytest.mark.parametrize("precision", [0, 1])
def test_threshold_zero_falls_back_to_exact(box128, precision):
    sys_, model = box128
    e0, f0, s0, _, _ = run_with(sys_, None, None, precision, force_scaled=True)
    e1, f1, s1, flagged, d = run_with(sys_, model, 0.0, precision)
    assert flagged == len(sys_["Z"])
    tol = 1e-10 if precision == 0 else 1e-6
    assert abs(e1 - e0) <= tol * abs(e0)
    assert np.abs(f1 - f0).max() <= tol * np.abs(f0).max() * 10
    assert np.abs(s1 - s0).max() <= tol * np.abs(s0).max() * 10
    # the option switches the surrogate off again
    d.set_option(OPT_ATM_SURROGATE, 0)
    e2, _, _ = d.compute()
    ex, _, _, _, _ = run_with(sys_, None, None, precision)
    assert abs(e2 - ex) <= 1e-12 * abs(ex) + (0 if precision == 0 else 1e-6 * abs(ex))


def test_fallback_partitions_energy(box128):
    sys_, model = box128
    n = len(sys_["Z"])
    d = handle_for(sys_)
    d.compute()
    G, c, e_exact = SU.descriptors_of(d, CH)
    ens = SU.predict(model, G, c)
    std = ens.std(0, unbiased=False).cpu().numpy()
    thr = float(np.median(std))
    e_sur, f, s, flagged, _ = run_with(sys_, model, thr)
    fl = std > thr
    assert flagged == int(fl.sum()) and 0 < flagged < n
    d0 = D3(sys_["Z"], n, rc=95.0, rc_cn=40.0, rc_atm=None)
    d0.set_cell(sys_["cell"])
    d0.set_atoms(sys_["pos"], sys_["Z"])
    e_two, _, _ = d0.compute()
    mean = ens.mean(0).cpu().numpy()
    expect = e_two + mean[~fl].sum() + e_exact.cpu().numpy()[fl].sum()
    assert abs(e_sur - expect) <= 1e-6 * abs(expect - e_two) + 1e-9
    assert np.abs(f.sum(0)).max() <= 1e-9 * n * (np.abs(f).max() + 1)


def test_surrogate_rejects_uncovered_element():
    sys_ = mixed_box(32, seed=1)
    Z = sys_["Z"].copy()
    Z[0] = 26  # Fe: not a channel of the model
    d = D3(Z, len(Z), rc=95.0, rc_cn=40.0, rc_atm=40.0)
    with pytest.raises(RuntimeError):
        d.set_surrogate(random_model(seed=0))


def test_trained_model_beats_dropping_atm():
    # the shipped model on a held-out box of the benchmark generator (3,000 atoms): its
    # error against the exact ATM term is far below the error of leaving ATM out, and
    # within the surrogate bars (0.5 meV/atom energy, 5 meV/A forces)
    import os

    path = os.path.join(os.path.dirname(SU.__file__), "surrogate", "atm_hcnosicu.d3s")
    model = SU.Model.load(path)
    sys_ = S.triclinic_box(3000, seed=41)
    n = len(sys_["Z"])
    e_x, f_x, _, _, _ = run_with(sys_, None, None, precision=1, force_scaled=True)
    e_s, f_s, _, flagged, _ = run_with(sys_, model, 1e9, precision=1)
    assert flagged == 0
    d0 = D3(sys_["Z"], n, rc=95.0, rc_cn=40.0, rc_atm=None)
    d0.set_option(OPT_PRECISION, 1)
    d0.set_cell(sys_["cell"])
    d0.set_atoms(sys_["pos"], sys_["Z"])
    e_0, f_0, _ = d0.compute()
    d0.close()
    err_s, err_0 = abs(e_s - e_x) / n, abs(e_0 - e_x) / n
    ferr_s, ferr_0 = np.abs(f_s - f_x).max(), np.abs(f_0 - f_x).max()
    assert err_s <= 5e-4 and ferr_s <= 5e-3, (err_s, ferr_s)
    assert err_s <= 0.1 * err_0, (err_s, err_0)
    assert ferr_s <= 0.5 * ferr_0, (ferr_s, ferr_0)
