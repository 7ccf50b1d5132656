"""Train the learned ATM surrogate on the GPU and evaluate it on a held-out box.

    python lasp-d3_b200/surrogate_train.py --structures 20000 --epochs 40 \\
        --out lasp-d3_b200/surrogate/atm_hcnosicu.d3s --eval-atoms 100000 --report report.json

1. Training structures: independent periodic cells, atom counts log-uniform in [8, 2000],
   cubic at 0.1 atoms/A^3 sheared by +-10 % tilts, 1.0 A minimum distance, Dirichlet(1)
   composition over H, C, N, O, Si, Cu (generated on the host cores, seeded).
2. Labels: exact per-atom ATM energies (one third of every triplet through the atom) and
   descriptors from the engine (batching form, FP32 pair/triplet arithmetic).
3. Training: 4-member ensemble, Adam with cosine learning rate, one permutation of the
   rows per member per epoch; the last 5 % of the structures are held out.
4. Evaluation: the 20,000-atom triclinic benchmark generator scaled to --eval-atoms atoms,
   exact ATM (FP64) against the surrogate path (default fallback threshold), reporting the
   energy error per atom, the per-atom RMSE, force and stress errors, the fraction of atoms
   that fell back and the device time of the three-body term and of the whole evaluation.
"""
import argparse
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import d3_systems as S  # noqa: E402


def _gen(args):
    count, seed = args
    return S.batch_structs(count=count, seed=seed)


def make_structures(n, seed, procs):
    chunk = 250
    jobs = [(min(chunk, n - k), seed * 100003 + k // chunk) for k in range(0, n, chunk)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        parts = pool.map(_gen, jobs)
    return [s for p in parts for s in p]


def evaluate(model, n_atoms, seed, threshold=None, log=print):
    """Exact ATM (FP64) against the surrogate path on the scaled benchmark box."""
    import torch

    import d3_surrogate as SU
    from d3_b200 import D3, OPT_PRECISION

    box = S.triclinic_box(n_atoms, seed=seed)
    n = len(box["Z"])
    out = {"atoms": n, "seed": seed}

    def handle(rc_atm=40.0, precision=0):
        d = D3(model.channel_z, n, rc=95.0, rc_cn=40.0, rc_atm=rc_atm)
        d.set_option(OPT_PRECISION, precision)
        d.set_cell(box["cell"])
        d.set_atoms(box["pos"], box["Z"])
        return d

    def timed(d, reps=2):
        d.compute()
        best = None
        for _ in range(reps):
            r = d.compute()
            pt, _ = d.pass_times()
            tot = sum(pt.values())
            if best is None or tot < best[1]:
                best = (r, tot, pt)
        return best

    d0 = handle(None)
    (e0, f0, s0), t0, _ = timed(d0, 1)
    d0.close()
    dx = handle()
    (ex, fx, sx), tx, ptx = timed(dx)
    G, c, e_lab = SU.descriptors_of(dx, model.channel_z)
    dx.close()
    ens = SU.predict(model, G, c)
    mean, std = ens.mean(0), ens.std(0, unbiased=False)
    out["exact"] = {"energy_ev": ex, "atm_energy_ev": ex - e0, "atm_ms": ptx["atm_list"] + ptx["atm"],
                    "total_ms": tx, "atoms_per_s": n / (tx * 1e-3), "force_max_ev_a": float(np.abs(fx - f0).max())}
    out["network"] = {"rmse_mev_atom": 1e3 * float((mean - e_lab).pow(2).mean().sqrt()),
                      "max_abs_mev_atom": 1e3 * float((mean - e_lab).abs().max()),
                      "mean_std_mev": 1e3 * float(std.mean()),
                      "max_std_mev": 1e3 * float(std.max()),
                      "energy_error_mev_atom": 1e3 * float((mean - e_lab).sum()) / n}
    for prec in (0, 1):
        d = handle(precision=prec)
        d.set_surrogate(model, threshold_ev=threshold)
        (es, fs, ss), ts, pts = timed(d)
        flagged = d.surrogate_flagged()
        d.close()
        df = fs - fx
        out["surrogate_p%d" % prec] = {
            "energy_ev": es, "energy_error_mev_atom": 1e3 * (es - ex) / n,
            "force_max_err_mev_a": 1e3 * float(np.abs(df).max()),
            "force_rms_err_mev_a": 1e3 * float(np.sqrt((df ** 2).sum(1).mean())),
            "stress_max_err_ev_a3": float(np.abs(ss - sx).max()),
            "flagged": flagged, "flagged_fraction": flagged / n,
            "atm_ms": pts["atm_list"] + pts["atm"], "total_ms": ts, "atoms_per_s": n / (ts * 1e-3),
            "atm_speedup_vs_exact_fp64": (ptx["atm_list"] + ptx["atm"]) / (pts["atm_list"] + pts["atm"]),
            "passes_ms": pts,
        }
    out["no_atm"] = {"energy_error_mev_atom": 1e3 * (e0 - ex) / n,
                     "force_max_err_mev_a": 1e3 * float(np.abs(f0 - fx).max()), "total_ms": t0}
    del G, c, e_lab, ens
    torch.cuda.empty_cache()
    if log:
        log(json.dumps(out, indent=1))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--structures", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--members", type=int, default=4)
    ap.add_argument("--procs", type=int, default=min(32, os.cpu_count() or 1))
    ap.add_argument("--out", default=os.path.join(HERE, "surrogate", "atm_hcnosicu.d3s"))
    ap.add_argument("--eval-atoms", type=int, default=100000)
    ap.add_argument("--eval-seed", type=int, default=77)
    ap.add_argument("--eval-only", default=None, help="evaluate this model file instead of training")
    ap.add_argument("--report", default=None)
    a = ap.parse_args()

    def log(msg):
        print(msg, flush=True)

    if a.eval_only:
        import d3_surrogate as SU

        report = {"eval": evaluate(SU.Model.load(a.eval_only), a.eval_atoms, a.eval_seed, log=log)}
        if a.report:
            with open(a.report, "w") as f:
                json.dump(report, f, indent=1)
        return

    t0 = time.time()
    structs = make_structures(a.structures, a.seed, a.procs)
    n_atoms = sum(len(s["Z"]) for s in structs)
    log("generated %d structures, %d atoms (%.1f s)" % (len(structs), n_atoms, time.time() - t0))

    import torch

    import d3_surrogate as SU

    t1 = time.time()
    G, c, e, sid = SU.label_structures(structs, SU.CHANNELS_HCNOSICU, log=log)
    t_label = time.time() - t1
    del structs
    rows = np.arange(G.shape[0])
    cut = int(0.95 * a.structures)
    tr, va = rows[sid < cut], rows[sid >= cut]
    t2 = time.time()
    model, hist = SU.train(G, c, e, tr, va, SU.CHANNELS_HCNOSICU, members=a.members, epochs=a.epochs, batch=a.batch,
                           lr=a.lr, seed=a.seed, log=log)
    t_train = time.time() - t2
    model.meta.update({"structures": a.structures, "atoms": n_atoms, "train_atoms": int(len(tr)),
                       "val_atoms": int(len(va)), "epochs": a.epochs, "batch": a.batch, "lr": a.lr, "seed": a.seed,
                       "val_rmse_ev": hist[-1]["val_rmse_ev"], "val_std_ev": hist[-1]["val_std_ev"],
                       "label_seconds": t_label, "train_seconds": t_train, "rc_atm_bohr": 40.0})
    model.save(a.out)
    log("saved %s" % a.out)
    del G, c, e
    torch.cuda.empty_cache()
    report = {"label_seconds": t_label, "train_seconds": t_train, "atoms": n_atoms, "history": hist}
    if a.eval_atoms > 0:
        report["eval"] = evaluate(model, a.eval_atoms, a.eval_seed, log=log)
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
