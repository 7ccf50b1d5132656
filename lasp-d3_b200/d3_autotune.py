"""Autotuner for the engine's launch parameters.

Tunables (engine options):
  D3_OPT_BIN_DIVISOR        cell-list bin width = smallest cutoff / divisor   (pair passes)
  D3_OPT_PAIR_KERNEL        two-body threads per atom: 1 (groups of 32 atoms,  (two-body)
                            one lane each) or 32 (one warp per atom)
  D3_OPT_ATMB_WARPS         block-pair ATM kernel: warps per CTA (up to 8 with (ATM pass,
                            two y buffers per warp, 9-12 with one)               precision)
  D3_OPT_ATM_CTAS_PER_SM    CTAs per SM (block-pair: 2 CTAs of 4 warps when they fit;
                            mirror / FP64 kernels: persistent CTAs per SM)
  D3_OPT_ATMB_LIST_CAPACITY longest list of the block-pair kernel (the rest go to the
                            mirror kernel)
  D3_OPT_ATMB_FINE_SKIP     block-pair kernel: skip out-of-range visits per two steps
  D3_OPT_ATM_TILE           partner-tile entries of the mirror and FP64 ATM kernels

`tune(handle, key)` times each candidate with the engine's per-pass CUDA-event timers
(d3_pass_times) on the caller's own workload and keeps the fastest; the pair passes and
the ATM pass are tuned independently (bin width and pair kernel first, then the ATM
kernel's shape: block-pair shapes in the precision form, tile and CTAs in the FP64 form).
Results are cached in a JSON file keyed by GPU name, atom-count bucket (powers of two),
density bucket, cutoffs, ATM on/off and precision form, so a workload of the same kind
reuses them without timing. Cache path: $D3_AUTOTUNE_CACHE or
~/.cache/d3_b200/autotune.json.
"""
import json
import math
import os

from d3_b200 import (OPT_ATM_CTAS_PER_SM, OPT_ATM_TILE, OPT_ATMB_FINE_SKIP, OPT_ATMB_LIST_CAPACITY, OPT_ATMB_WARPS,
                     OPT_BIN_DIVISOR, OPT_PAIR_KERNEL)

BIN_DIVISORS = (3, 4, 6, 8)
PAIR_KERNELS = (0, 1)
ATM_TILES = (64, 128, 256)
ATM_CTAS = (0, 2, 3)
# block-pair shapes: (warps per CTA, CTAs per SM, list capacity; 0 = automatic; skip
# out-of-range visits per two steps)
ATMB_SHAPES = ((0, 0, 0, 0), (0, 0, 0, 1), (8, 0, 0, 0), (10, 0, 0, 0), (4, 2, 0, 0), (12, 0, 4096, 0))


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
    # v2: the parameter set includes the pair kernel and the block-pair ATM shape
    return "v2|%s|n2^%d|rho2^%.1f|rc%.1f/%.1f/%.1f|p%d" % (gpu_name(), nb, rb, rc, rc_cn, rc_atm or 0.0, precision)


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
    handle.set_option(OPT_PAIR_KERNEL, params.get("pair_kernel", 0))
    handle.set_option(OPT_ATM_TILE, params["atm_tile"])
    handle.set_option(OPT_ATM_CTAS_PER_SM, params["atm_ctas_per_sm"])
    handle.set_option(OPT_ATMB_WARPS, params.get("atmb_warps", 0))
    handle.set_option(OPT_ATMB_LIST_CAPACITY, params.get("atmb_mcap", 0))
    handle.set_option(OPT_ATMB_FINE_SKIP, params.get("atmb_fine_skip", 0))


def _time(handle, repeats):
    best = None
    for _ in range(repeats):
        handle.compute()
        pt, _ = handle.pass_times()
        best = pt if best is None else {k: min(best[k], pt[k]) for k in pt}
    return best


def tune(handle, key, repeats=2, use_cache=True, atm=True, precision=None):
    """Choose bin divisor, pair kernel and the ATM kernel's shape for `handle` (a D3 or
    D3Batch whose structures are set); applies and returns the parameters. precision: the
    handle's form (taken from `key` when None)."""
    db = _load() if use_cache else {}
    if key in db:
        apply(handle, db[key])
        return dict(db[key], cached=True)
    if precision is None:
        precision = key.endswith("|p1")
    params = {"bin_divisor": 6, "pair_kernel": 0, "atm_tile": 0, "atm_ctas_per_sm": 0, "atmb_warps": 0,
              "atmb_mcap": 0, "atmb_fine_skip": 1}
    apply(handle, params)
    pair_passes = ("bin", "cn", "twobody", "atm_list", "chain")
    best = None
    trials = []
    for bd in BIN_DIVISORS:
        for pk in PAIR_KERNELS:
            handle.set_option(OPT_BIN_DIVISOR, bd)
            handle.set_option(OPT_PAIR_KERNEL, pk)
            pt = _time(handle, repeats)
            t = sum(pt[k] for k in pair_passes)
            trials.append({"bin_divisor": bd, "pair_kernel": pk, "pair_ms": t})
            if best is None or t < best[0]:
                best = (t, bd, pk)
    params["bin_divisor"], params["pair_kernel"] = best[1], best[2]
    apply(handle, params)
    if atm:
        best = None
        if precision:
            # the block-pair kernel takes the lists up to its capacity, the mirror kernel
            # (tile, CTAs per SM at their defaults) the longer ones
            for w, c, m, f in ATMB_SHAPES:
                handle.set_option(OPT_ATMB_WARPS, w)
                handle.set_option(OPT_ATM_CTAS_PER_SM, c)
                handle.set_option(OPT_ATMB_LIST_CAPACITY, m)
                handle.set_option(OPT_ATMB_FINE_SKIP, f)
                t = _time(handle, repeats)["atm"]
                trials.append({"atmb_warps": w, "atm_ctas_per_sm": c, "atmb_mcap": m, "atmb_fine_skip": f, "atm_ms": t})
                if best is None or t < best[0]:
                    best = (t, w, c, m, f)
            (params["atmb_warps"], params["atm_ctas_per_sm"], params["atmb_mcap"],
             params["atmb_fine_skip"]) = best[1:]
        else:
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
