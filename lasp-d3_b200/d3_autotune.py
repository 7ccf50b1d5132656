"""Autotuner for the engine's launch parameters.

Tunables (engine options):
  D3_OPT_BIN_DIVISOR      cell-list bin width = smallest cutoff / divisor  (pair passes)
  D3_OPT_ATM_TILE         ATM partner-tile entries                           (ATM pass)
  D3_OPT_ATM_CTAS_PER_SM  persistent ATM CTAs per SM                         (ATM pass)

`tune(handle_factory, ...)` times each candidate with the engine's per-pass CUDA-event
timers (d3_pass_times) on the caller's own workload and keeps the fastest; the pair
passes and the ATM pass are tuned independently (bin width first, then tile and CTAs).
Results are cached in a JSON file keyed by GPU name, atom-count bucket (powers of two),
density bucket, cutoffs, ATM on/off and precision form, so a workload of the same kind
reuses them without timing. Cache path: $D3_AUTOTUNE_CACHE or
~/.cache/d3_b200/autotune.json.
"""
import json
import math
import os

from d3_b200 import OPT_ATM_CTAS_PER_SM, OPT_ATM_TILE, OPT_BIN_DIVISOR, OPT_PRECISION

BIN_DIVISORS = (3, 4, 6, 8)
ATM_TILES = (64, 128, 256)
ATM_CTAS = (0, 2, 3)


def cache_path():
    return os.environ.get("D3_AUTOTUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "d3_b200",
                                                               "autotune.json")


def gpu_name():
    try:
        import torch

        return torch.cuda.get_device_name()
    except Exception:
        return "unknown-gpu"


def workload_key(n_atoms, volume_a3, rc, rc_cn, rc_atm, precision):
    nb = int(round(math.log2(max(n_atoms, 1))))
    rho = n_atoms / max(volume_a3, 1e-9)
    rb = round(math.log2(rho) * 2) / 2 if rho > 0 else 0
    return "%s|n2^%d|rho2^%.1f|rc%.1f/%.1f/%.1f|p%d" % (gpu_name(), nb, rb, rc, rc_cn, rc_atm or 0.0, precision)


def _load():
    try:
        return json.load(open(cache_path()))
    except (OSError, ValueError):
        return {}


def _save(db):
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    json.dump(db, open(tmp, "w"), indent=1, sort_keys=True)
    os.replace(tmp, p)


def apply(handle, params):
    handle.set_option(OPT_BIN_DIVISOR, params["bin_divisor"])
    handle.set_option(OPT_ATM_TILE, params["atm_tile"])
    handle.set_option(OPT_ATM_CTAS_PER_SM, params["atm_ctas_per_sm"])


def _time(handle, repeats):
    best = None
    for _ in range(repeats):
        handle.compute()
        pt, _ = handle.pass_times()
        best = pt if best is None else {k: min(best[k], pt[k]) for k in pt}
    return best


def tune(handle, key, repeats=2, use_cache=True, atm=True):
    """Choose bin divisor, ATM tile and ATM CTAs/SM for `handle` (a D3 or D3Batch whose
    structures are set); applies and returns the parameters."""
    db = _load() if use_cache else {}
    if key in db:
        apply(handle, db[key])
        return dict(db[key], cached=True)
    params = {"bin_divisor": 6, "atm_tile": 0, "atm_ctas_per_sm": 0}
    apply(handle, params)
    pair_passes = ("bin", "cn", "twobody", "atm_list", "chain")
    best = None
    trials = []
    for bd in BIN_DIVISORS:
        handle.set_option(OPT_BIN_DIVISOR, bd)
        pt = _time(handle, repeats)
        t = sum(pt[k] for k in pair_passes)
        trials.append({"bin_divisor": bd, "pair_ms": t})
        if best is None or t < best[0]:
            best = (t, bd)
    params["bin_divisor"] = best[1]
    handle.set_option(OPT_BIN_DIVISOR, best[1])
    if atm:
        best = None
        for tile in ATM_TILES:
            for ctas in ATM_CTAS:
                handle.set_option(OPT_ATM_TILE, tile)
                handle.set_option(OPT_ATM_CTAS_PER_SM, ctas)
                t = _time(handle, repeats)["atm"]
                trials.append({"atm_tile": tile, "atm_ctas_per_sm": ctas, "atm_ms": t})
                if best is None or t < best[0]:
                    best = (t, tile, ctas)
        params["atm_tile"], params["atm_ctas_per_sm"] = best[1], best[2]
    apply(handle, params)
    if use_cache:
        db = _load()
        db[key] = params
        _save(db)
    return dict(params, cached=False, trials=trials)
