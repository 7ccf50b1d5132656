"""Benchmark of the D3(BJ)+ATM energy/force/stress path on B200.

Workload (one "step" = one full evaluation: wrap/bin, CN, C6 weights, two-body, ATM
list + triplets, dE/dCN chain rule, reductions, E + F + stress):
  20,000-atom triclinic periodic box, cell rows a=(58,0,0), b=(5,58,0), c=(3,4,58) A,
  uniform positions with a 1.0 A minimum-image rejection, H 40 / C 30 / N 10 / O 15 /
  Cu 5 %, PBE-D3(BJ) (s6 1, s8 0.7875, a1 0.4289, a2 4.4407) with ATM, 5-reference
  table, cutoffs 95 (two-body) / 40 (CN) / 40 (ATM) bohr. Seeded synthetic input; the
  parameter table is the seeded synthetic table (the real D3 tables are not available).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Multi-GPU (torchrun, one process per GPU): every rank evaluates its own box (different
seed), no data-path collective; value = all atoms / max-over-ranks time ("weak"). With
--shard the ranks evaluate ONE box together (d3_shard.py: round-robin split of central
atoms and ATM apexes, NCCL all-reduce of dE/dCN and of the results; "strong").
The reference arm times the reference's own CUDA build (oracle/_ref) through its C ABI
on a bounded sample of the same generator (rank 0 only).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lasp-d3_b200"))

METRIC = "D3(BJ)+ATM atoms/s (E+F+stress) on 1 B200: plain vs chosen form at stated error"
RC, RC_CN, RC_ATM = 95.0, 40.0, 40.0
N_ATOMS = 20000
# Algorithmic FLOPs of one in-range ATM triplet term as the reference writes it
# (src/d3_kernel.cu:1331-1447: distances and range test 20, distance powers 24, r^2/r 3,
# cosine numerators 6, cosine and angular term 8, three angular derivatives 72, C9 and
# its CN derivatives 19, damping and its derivative 21, energy 7, dE/dCN 15, the three
# force scalars once 18, 3x3 stress 99, forces 33), counted with add/mul/cmp = 1,
# div/sqrt/pow = 1, each accumulation as one add; the C6 interpolation (per atom pair)
# and the image translation (enumeration) are not included.
ATM_FLOP_PER_TRIPLET = 345
L2_FLUSH_BYTES = 256 << 20


# Algorithmic FLOPs of one in-range ordered two-body pair as the reference writes it
# (src/d3_kernel.cu:1105-1154): distance 8, r powers 6, BJ damping terms 12, energy 6,
# dE/dr and dE/dCN 12, force 6, half of the 3x3 stress 10; C6 interpolation excluded.
TWOBODY_FLOP_PER_PAIR = 60


def system_for(args, seed):
    import d3_systems as S

    if args.system == "water":
        return S.water_box(seed=0)
    return S.triclinic_box(args.atoms, seed=seed)


def workload_config(n, args=None):
    """The workload: identical in the engine arm and the reference arm (the form each arm
    computes in is reported beside it, under "form")."""
    water = args is not None and args.system == "water"
    table = 7 if (args is not None and args.table == 7) else 5
    atm = not (args is not None and args.no_atm)
    if water:
        box = ("32 rigid H2O (96 atoms) in a cubic 9.86 A cell, O on a jittered 4x4x2 grid, random "
               "orientations (seed 0)")
    else:
        box = ("%d-atom triclinic periodic box (a=(58,0,0) b=(5,58,0) c=(3,4,58) A, scaled for other sizes), "
               "H40/C30/N10/O15/Cu5 %%, 1.0 A min-image rejection" % n)
    return {
        "workload": "%s; PBE-D3(BJ)%s, %d-reference synthetic table, rc 95 / rc_CN 40%s bohr; "
                    "energy+forces+stress" % (box, "+ATM" if atm else " (two-body + CN, no ATM)", table,
                                               " / rc_ATM 40" if atm else ""),
        "atoms_per_gpu": n,
        "l2": "flushed between timed steps (256 MiB device write)",
        "parallelism": "replicas: one box per GPU, no collective",
    }


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_cpu_baseline(sys_, sample=48, seed=7, rc_atm=RC_ATM, extended=False):
    """FP64 oracle (C/OpenMP, all host threads) on a bounded sample: CN for every atom,
    then two-body, ATM (as apex) and chain rule for `sample` random central atoms."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    n = len(sys_["Z"])
    rng = np.random.default_rng(seed)
    sample = min(sample, n)
    sub = np.sort(rng.choice(n, size=sample, replace=False))
    cores = os.cpu_count() or 1
    kw = dict(rc=RC, rc_cn=RC_CN, rc_atm=rc_atm, damping=1, functional=0, c6_mode=1, nthreads=cores,
              extended=extended)
    t0 = time.perf_counter()
    oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], subset=np.zeros(0, np.int64), **kw)
    t_cn = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.compute(sys_["pos"], sys_["Z"], sys_["cell"], subset=sub, **kw)
    t_sub = time.perf_counter() - t0 - t_cn
    per_atom_s = t_sub / sample + t_cn / n
    return {"value": 1.0 / per_atom_s, "unit": "atoms/s", "cores": cores, "kind": "port",
            "sample": "FP64 C/OpenMP oracle of the reference formulas (factorised C6) on the same box: CN for all "
                      "%d atoms (%.1f s) plus two-body, ATM apex and chain rule for %d random atoms (%.1f s); "
                      "atoms/s = 1 / (t_sample/%d + t_cn/%d)" % (n, t_cn, sample, t_sub, sample, n)}


def apply_options(handle, args):
    """--option NAME=VALUE: engine options (d3_b200.OPT_*) set on a handle."""
    import d3_b200

    for kv in args.option:
        name, val = kv.split("=")
        key = name if name.startswith("OPT_") else "OPT_" + name.upper()
        handle.set_option(getattr(d3_b200, key), int(val))


def time_form(d, args, flush, stream, barrier):
    """Warm-up and K timed evaluations of one engine handle on `stream` (device time by
    CUDA events, L2 flushed between steps). Returns per-step ms, ATM ms, passes, counters."""
    import torch

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            d.compute_async(stream.cuda_stream)
    barrier()
    step_ms, atm_ms, passes = [], [], []
    counters = None
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            s_ev = torch.cuda.Event(enable_timing=True)
            e_ev = torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            st = d.compute_async(stream.cuda_stream)
            e_ev.record(stream)
            e_ev.synchronize()
            if st != 0:
                raise RuntimeError("engine status %d" % st)
            step_ms.append(s_ev.elapsed_time(e_ev))
            pt, counters = d.pass_times()
            passes.append(pt)
            atm_ms.append(pt["atm"])
    barrier()
    return step_ms, atm_ms, passes, counters


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def engine_arm(args, world, rank, local):
    import torch

    import d3_systems as S
    from d3_b200 import D3, OPT_PRECISION, TABLE_5REF, TABLE_7REF, peak_probe

    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    sys_ = system_for(args, 1 + rank)
    n = len(sys_["Z"])
    rc_atm = None if args.no_atm else RC_ATM
    table = TABLE_7REF if args.table == 7 else TABLE_5REF
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    forms = {}
    sampler = ClockSampler(local)
    sampler.start()
    for form, prec in (("plain", 0), ("precision", 1)):
        d = D3(sys_["Z"], n, rc=RC, rc_cn=RC_CN, rc_atm=rc_atm, damping=1, functional=0, table=table)
        apply_options(d, args)
        d.set_option(OPT_PRECISION, prec)
        d.set_cell(sys_["cell"])
        d.set_atoms(sys_["pos"], sys_["Z"])
        energy, forces, stress = d.compute()  # sizes the ATM list; result checked below
        step_ms, atm_ms, passes, counters = time_form(d, args, flush, stream, barrier)
        total_ms = max_over_ranks(float(sum(step_ms)), world)
        ms_per_step = total_ms / args.steps
        forms[form] = {"value": world * n / (ms_per_step * 1e-3), "ms_per_step": ms_per_step,
                       "atm_ms": statistics.mean(atm_ms), "counters": counters,
                       "twobody_ms": statistics.mean(p["twobody"] for p in passes),
                       "passes_ms": {k: statistics.mean(p[k] for p in passes) for k in passes[0]},
                       "energy": energy, "forces": forces, "stress": stress,
                       "launches": d.launches_per_eval()}
        d.close()
    clocks = sampler.stop()
    ref = forms["plain"]
    prec = forms["precision"]
    err = {"energy_rel": abs(prec["energy"] - ref["energy"]) / abs(ref["energy"]),
           "force_max_ev_per_a": float(np.abs(prec["forces"] - ref["forces"]).max()),
           "force_rms_ev_per_a": float(np.sqrt(np.mean((prec["forces"] - ref["forces"]) ** 2))),
           "stress_max_ev_per_a3": float(np.abs(prec["stress"] - ref["stress"]).max()),
           "against": "the FP64 plain form on the same input (which matches the FP64 oracle to 1e-9 relative)"}
    meets = err["energy_rel"] <= 1e-6 and err["force_max_ev_per_a"] <= 1e-4
    chosen = "precision" if meets else "plain"
    ch = forms[chosen]

    # end to end through the reference-facing C ABI: float host buffers in, float out,
    # host<->device copies inside the timed region, in the chosen form
    from d3_b200 import load_library

    lib = load_library()
    z16 = np.ascontiguousarray(sys_["Z"], np.uint16)
    posf = np.ascontiguousarray(sys_["pos"], np.float32)
    cellf = np.ascontiguousarray(sys_["cell"], np.float32)
    if table == TABLE_7REF:
        el = np.ascontiguousarray(sorted(set(int(z) for z in sys_["Z"])), np.uint16)
        h = lib.d3_init_handle_ex(el.ctypes.data, len(el), n, RC, RC_CN, rc_atm or 0.0, 1, 0, table)
    elif rc_atm:
        h = lib.init_d3_handle_with_atm(z16.ctypes.data, n, n, RC, RC_CN, RC_ATM, 1, 0)
    else:
        h = lib.init_d3_handle(z16.ctypes.data, n, n, RC, RC_CN, 1, 0)
    import d3_b200

    for kv in args.option:
        name, val = kv.split("=")
        lib.d3_set_option(h, getattr(d3_b200, name if name.startswith("OPT_") else "OPT_" + name.upper()), int(val))
    lib.d3_set_option(h, OPT_PRECISION, 1 if chosen == "precision" else 0)
    lib.set_cell(h, cellf.ctypes.data)
    ef = np.zeros(1, np.float32)
    ff = np.zeros((n, 3), np.float32)
    sf = np.zeros(9, np.float32)
    for _ in range(max(1, args.warmup)):
        lib.set_atoms(h, posf.ctypes.data, z16.ctypes.data, n)
        lib.compute_dispersion_energy_from_handle_status(h, ef.ctypes.data, ff.ctypes.data, sf.ctypes.data)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        lib.set_atoms(h, posf.ctypes.data, z16.ctypes.data, n)
        lib.compute_dispersion_energy_from_handle_status(h, ef.ctypes.data, ff.ctypes.data, sf.ctypes.data)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    lib.free_d3_handle(h)
    e2e = {"value": world * n * args.steps / e2e_s, "unit": "atoms/s",
           "h2d_bytes_per_step": 3 * n * 8 + n * 4, "d2h_bytes_per_step": (1 + 3 * n + 9) * 8 + 4,
           "path": "set_atoms(float coords) + compute_dispersion_energy_from_handle_status, host buffers, %s form"
                   % chosen}

    # roofline of the dominant kernel of the chosen form (ATM triplets; two-body pairs
    # when ATM is off)
    fp64 = chosen == "plain"
    peak = peak_probe(fp64)
    triplets = int(ch["counters"][0]) // 2
    pairs = int(ch["counters"][1])
    traffic = None
    if rc_atm:
        achieved = triplets * ATM_FLOP_PER_TRIPLET / (ch["atm_ms"] * 1e-3) / 1e12
        tfile = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        if os.path.exists(tfile) and args.system == "triclinic" and n == N_ATOMS and table == TABLE_5REF:
            traffic = json.load(open(tfile)).get("atm_fp64_bytes_per_launch" if fp64 else "atm_fp32_bytes_per_launch")
        kernel = ("k_atm (ATM triplets, FP64)" if fp64 else
                  "k_atm32b + k_atm32 (ATM triplets, FP32 arithmetic; block pairs, packed f32x2 pairs of visits; lists beyond the per-launch block-pair capacity mirrored)")
        algorithmic = "%d in-range triplets x %d FLOP per launch" % (triplets, ATM_FLOP_PER_TRIPLET)
    else:
        achieved = pairs * TWOBODY_FLOP_PER_PAIR / (ch["twobody_ms"] * 1e-3) / 1e12
        kernel = ("k_twobody_g (two-body pairs on atom groups, FP64)" if fp64 else
                  "k_twobody_g (two-body pairs on atom groups, FP32 pair arithmetic)")
        algorithmic = "%d in-range ordered pairs x %d FLOP per launch" % (pairs, TWOBODY_FLOP_PER_PAIR)
    roofline = {"bound": "fp64" if fp64 else "fp32", "kernel": kernel,
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": "measured %s FMA throughput of this GPU by d3_peak_probe (MEASURED_PEAKS.json has no "
                               "FP64/FP32 figure)" % ("FP64" if fp64 else "FP32"),
                "algorithmic": algorithmic}
    model_path = os.path.join(ROOT, "lasp-d3_b200", "surrogate", "atm_hcnosicu.d3s")
    sur = None
    if os.path.exists(model_path) and rc_atm and table == TABLE_5REF and args.system == "triclinic":
        import d3_surrogate as SU

        sur = surrogate_form(sys_, SU.Model.load(model_path), args, flush, stream, barrier, forms["plain"])
    forms_out = {}
    for k, f in forms.items():
        forms_out[k] = {"value": f["value"], "unit": "atoms/s", "ms_per_step": f["ms_per_step"],
                        "passes_ms": f["passes_ms"], "energy_ev": f["energy"]}
    forms_out["precision"]["error_vs_fp64"] = err
    if sur is not None:
        sur["note"] = ("learned ATM surrogate; not eligible as the headline form: its error is above the "
                       "1e-6 relative energy bar")
        forms_out["surrogate"] = {k: v for k, v in sur.items() if k != "launches"}
    line = {"metric": METRIC, "value": ch["value"], "unit": "atoms/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ch["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if fp64 else "f32", "data": "synthetic",
            "config": workload_config(n, args),
            "form": "%s form (%s)" % (chosen, "FP64 throughout" if fp64 else
                                      "FP32 pair/triplet arithmetic, FP64 C6 weights, dE/dCN and reductions"),
            "chosen_form": chosen, "forms": forms_out, "options": args.option,
            "roofline": roofline, "e2e": e2e, "gpu_launches": ch["launches"] * args.steps, "clocks": clocks,
            "counters": {"atm_triplets": triplets, "twobody_ordered_pairs": int(ch["counters"][1]),
                         "cn_ordered_pairs": int(ch["counters"][2])}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = run_cpu_baseline(sys_, rc_atm=rc_atm, extended=table == TABLE_7REF)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def shard_arm(args, world, rank, local):
    """One structure evaluated by all ranks (strong scaling): every world-th atom / ATM apex
    per rank, all-reduce of dE/dCN and of the results (NCCL); precision form."""
    import datetime

    import torch
    import torch.distributed as dist

    import d3_shard
    from d3_b200 import D3, OPT_PRECISION

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    else:
        dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % (29500 + os.getpid() % 1000), rank=0,
                                world_size=1)
    sys_ = system_for(args, 1)
    n = len(sys_["Z"])
    d = D3(sys_["Z"], n, rc=RC, rc_cn=RC_CN, rc_atm=None if args.no_atm else RC_ATM, damping=1, functional=0)
    d.set_option(OPT_PRECISION, 1)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    ev = d3_shard.ShardedEvaluator(d)
    for _ in range(args.warmup):
        ev.compute_device()
    dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_ev.record()
    for _ in range(args.steps):
        ev.compute_device()
    e_ev.record()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = sampler.stop()
    ms = s_ev.elapsed_time(e_ev)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda" if world > 1 else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    out = ev.out.cpu().numpy()
    if rank == 0:
        line = {"metric": METRIC, "value": n * args.steps / (ms * 1e-3), "unit": "atoms/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "form": "precision form, sharded",
                "config": dict(workload_config(n, args),
                               parallelism="shard%d: central atoms and ATM apexes split round-robin over ranks; "
                                           "all-reduce of dE/dCN (n doubles) and of the results (NCCL)" % world,
                               l2="not flushed; the inputs are larger than L2 (ATM half lists about 330 MB at "
                                  "20,000 atoms)"),
                "energy_ev": float(out[0]), "clocks": clocks, "gpu_launches": d.launches_per_eval() * args.steps}
        print(json.dumps(line), flush=True)
    d.close()
    dist.destroy_process_group()


def reference_arm(args, world, rank, local):
    """The reference's own CUDA build (oracle/_ref/libd3_ref.so) through its C ABI."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_lib

    import d3_systems as S

    ext = args.table == 7
    if not ref_lib.available(ext):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/libd3_ref.so is missing"}))
        return
    if args.system == "water":
        sys_ = S.water_box(seed=0)
    else:
        sys_ = S.triclinic_box(args.ref_atoms, seed=1)
    n = len(sys_["Z"])
    # the reference's compute call is synchronous (src/d3.cu:201): wall clock around it
    h = ref_lib.RefHandle(sys_["Z"], n, RC, RC_CN, None if args.no_atm else RC_ATM, damping=1, functional=0,
                          extended=ext)
    h.set_system(sys_["pos"], sys_["Z"], sys_["cell"])
    for _ in range(args.warmup):
        h.compute()
    times = []
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e, f, s, st = h.compute()
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    h.close()
    sec = statistics.mean(times)
    value = n / sec
    full_n = 96 if args.system == "water" else args.atoms
    sample = ("reference CUDA build (LASP-D3 sources, sm_100a, synthetic table) through "
              "compute_dispersion_energy_from_handle_status on the same generator at %d atoms (cell scaled to "
              "density)%s" % (n, "" if n == full_n else "; its cost per atom grows with N (all-pairs ATM), so this "
                              "overstates its throughput at %d atoms" % full_n))
    line = {"metric": METRIC, "value": value, "unit": "atoms/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": workload_config(full_n, args),
            "form": "reference CUDA build (float)%s" % ("" if n == full_n else ", each step a bounded sample: the "
                                                                             "same generator at %d atoms" % n),
            "cpu_baseline": {"value": value, "unit": "atoms/s", "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": "atoms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "clocks": clocks, "energy_ev": e}
    print(json.dumps(line), flush=True)


def batch_mode(args):
    """Batching form: many independent structures in one handle (one launch per pass, the
    ATM pass one persistent launch over every structure's apexes), autotuned."""
    import torch

    import d3_autotune
    import d3_systems as S
    from d3_b200 import D3Batch, OPT_PRECISION

    torch.cuda.set_device(0)
    sts = S.batch_structs(count=args.batch, seed=3)
    elements = sorted(set(int(z) for s in sts for z in s["Z"]))
    ntot = sum(len(s["Z"]) for s in sts)
    vol = sum(abs(np.linalg.det(s["cell"])) for s in sts)
    out = {"metric": "D3(BJ)+ATM atoms/s (E+F+stress), %d-structure batch in one launch per pass" % len(sts),
           "unit": "atoms/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
           "data": "synthetic",
           "config": {"workload": "%d periodic structures, atom counts log-uniform in [8, 2000] (%d atoms in total), "
                                  "cubic cells at 0.1 atoms/A^3 sheared by +-10 %% tilts, Dirichlet(1) compositions over "
                                  "H/C/N/O/Si/Cu; PBE-D3(BJ)+ATM, rc 95 / 40 / 40 bohr" % (len(sts), ntot),
                      "l2": "not flushed: the ATM half lists of the batch (several GB) are far larger than L2"},
           "forms": {}}
    stream = torch.cuda.Stream()
    # the autotuner times candidates on a subset of the structures (same generator, so the
    # same per-structure sizes and densities) and the result is applied to the whole batch
    sub = sts[:min(len(sts), args.tune_structs)]
    nsub = sum(len(s["Z"]) for s in sub)
    for form, prec in (("plain", 0), ("precision", 1)):
        t = D3Batch(elements, len(sub), nsub, rc=RC, rc_cn=RC_CN, rc_atm=RC_ATM, damping=1, functional=0)
        t.set_option(OPT_PRECISION, prec)
        t.set_structures(sub)
        key = d3_autotune.workload_key(ntot / len(sts), vol / len(sts), RC, RC_CN, RC_ATM, prec) + "|batch"
        tuned = d3_autotune.tune(t, key, repeats=1, precision=bool(prec))
        t.close()
        b = D3Batch(elements, len(sts), ntot, rc=RC, rc_cn=RC_CN, rc_atm=RC_ATM, damping=1, functional=0)
        b.set_option(OPT_PRECISION, prec)
        b.set_structures(sts)
        d3_autotune.apply(b, tuned)
        e, _, _ = b.compute()
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                b.compute_async(stream.cuda_stream)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            b.compute_async(stream.cuda_stream)
            e_ev.record(stream)
            e_ev.synchronize()
            ms.append(s_ev.elapsed_time(e_ev))
        pt, cnt = b.pass_times()
        # the same evaluation captured once in a CUDA graph and replayed: one graph launch
        # per evaluation of every structure (list capacity sized by the calls above)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            b.compute_async(stream.cuda_stream)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            graph.replay()
        torch.cuda.synchronize()
        gms = []
        for _ in range(args.steps):
            s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_ev.record(stream)
            with torch.cuda.stream(stream):
                graph.replay()
            e_ev.record(stream)
            e_ev.synchronize()
            gms.append(s_ev.elapsed_time(e_ev))
        del graph
        out["forms"][form] = {"value": ntot / (statistics.mean(ms) * 1e-3), "ms_per_step": statistics.mean(ms),
                              "graph": {"value": ntot / (statistics.mean(gms) * 1e-3),
                                        "ms_per_step": statistics.mean(gms),
                                        "kernels_per_eval": b.launches_per_eval()},
                              "atm_list_capacity_entries": b.atm_list_capacity(),
                              "passes_ms": pt, "autotuned": {k: v for k, v in tuned.items() if k != "trials"},
                              "tuned_on_structures": len(sub),
                              "energy_sum_ev": float(np.sum(e))}
        b.close()
    out["value"] = out["forms"]["precision"]["value"]
    print(json.dumps(out), flush=True)


def md_mode(args):
    """200 MD-style steps of the 20,000-atom box (Gaussian displacement sigma = 0.01 A per
    step, cell fixed) captured once in a CUDA graph and replayed; precision form, autotuned."""
    import torch

    import d3_autotune
    import d3_systems as S
    from d3_b200 import D3, OPT_PRECISION

    torch.cuda.set_device(0)
    n = args.atoms
    sys_ = S.triclinic_box(n, seed=1)
    d = D3(sys_["Z"], n, rc=RC, rc_cn=RC_CN, rc_atm=RC_ATM, damping=1, functional=0)
    d.set_option(OPT_PRECISION, 1)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    vol = abs(np.linalg.det(sys_["cell"]))
    tuned = d3_autotune.tune(d, d3_autotune.workload_key(n, vol, RC, RC_CN, RC_ATM, 1), repeats=1, precision=True)
    d.compute()  # list capacity for the trajectory (the list grows on overflow only outside capture)
    pos = torch.tensor(sys_["pos"], dtype=torch.float64, device="cuda")
    noise = torch.empty_like(pos)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        # warm-up step outside capture
        noise.normal_(0.0, 0.01)
        pos.add_(noise)
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        noise.normal_(0.0, 0.01)
        pos.add_(noise)
        d.set_positions_device(pos.data_ptr(), stream.cuda_stream)
        d.compute_async(stream.cuda_stream)
    torch.cuda.synchronize()
    steps = args.md_steps
    s_ev, e_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s_ev.record(stream)
        for _ in range(steps):
            graph.replay()
        e_ev.record(stream)
    e_ev.synchronize()
    ms = s_ev.elapsed_time(e_ev)
    out = {"metric": "D3(BJ)+ATM MD steps/s (E+F+stress per step), CUDA graph, %d-atom box" % n,
           "value": steps / (ms * 1e-3), "unit": "steps/s", "atoms_per_s": n * steps / (ms * 1e-3),
           "ms_per_step": ms / steps, "steps": steps, "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
           "config": {"workload": "%d-atom triclinic box, Gaussian displacement 0.01 A per step, cell fixed; "
                                  "precision form; graph = displacement + set_positions_device + evaluation" % n},
           "autotuned": {k: v for k, v in tuned.items() if k != "trials"}}
    del graph
    d.close()
    print(json.dumps(out), flush=True)


def surrogate_form(sys_, model, args, flush, stream, barrier, ref):
    """The learned-surrogate form (precision-form exact parts, ATM through the surrogate
    with the exact fallback) timed like the other forms, with its error against the FP64
    plain form `ref` (energy, forces, stress of the same box)."""
    from d3_b200 import D3, OPT_PRECISION

    n = len(sys_["Z"])
    d = D3(sys_["Z"], n, rc=RC, rc_cn=RC_CN, rc_atm=RC_ATM, damping=1, functional=0)
    d.set_option(OPT_PRECISION, 1)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    d.set_surrogate(model)
    energy, forces, stress = d.compute()
    step_ms, atm_ms, passes, _ = time_form(d, args, flush, stream, barrier)
    flagged = d.surrogate_flagged()
    launches = d.launches_per_eval()

    def errors(e, f, st):
        df = f - ref["forces"]
        return {"energy_mev_per_atom": 1e3 * (e - ref["energy"]) / n,
                "energy_rel": abs(e - ref["energy"]) / abs(ref["energy"]),
                "force_max_mev_per_a": 1e3 * float(np.abs(df).max()),
                "force_rms_mev_per_a": 1e3 * float(np.sqrt((df ** 2).sum(1).mean())),
                "stress_max_ev_per_a3": float(np.abs(st - ref["stress"]).max())}

    # the exact fallback exercised: a threshold at the 99th percentile of the ensemble
    # spread sends about 1 % of the atoms (all triplets through them) to the exact kernel
    import d3_surrogate as SU

    G, c, _ = SU.descriptors_of(d, model.channel_z)
    spread = SU.predict(model, G, c).std(0, unbiased=False).double().cpu().numpy()
    thr = float(np.quantile(spread, 0.99))
    d.set_surrogate_threshold(thr)
    e_fb, f_fb, s_fb = d.compute()
    fb_ms, _, fb_passes, _ = time_form(d, args, flush, stream, barrier)
    fallback = {"threshold_mev": 1e3 * thr, "flagged_atoms": d.surrogate_flagged(),
                "ms_per_step": statistics.mean(fb_ms), "value": n / (statistics.mean(fb_ms) * 1e-3),
                "passes_ms": {k: statistics.mean(p[k] for p in fb_passes) for k in fb_passes[0]},
                "error_vs_fp64": errors(e_fb, f_fb, s_fb)}
    d.close()
    ms = statistics.mean(step_ms)
    pm = {k: statistics.mean(p[k] for p in passes) for k in passes[0]}
    return {"value": n / (ms * 1e-3), "unit": "atoms/s", "ms_per_step": ms, "passes_ms": pm,
            "three_body_ms": pm["atm_list"] + pm["atm"], "flagged_atoms": flagged, "launches": launches,
            "energy_ev": energy, "error_vs_fp64": errors(energy, forces, stress), "with_fallback": fallback}


def surrogate_mode(args):
    """Learned-part form on the benchmark generator scaled to --atoms atoms (default
    100,000): the surrogate form against the FP64 plain path on the same box, both timed
    by CUDA events with the L2 flushed between steps."""
    import torch

    import d3_surrogate as SU
    import d3_systems as S
    from d3_b200 import D3

    torch.cuda.set_device(0)
    model = SU.Model.load(args.model)
    n = args.atoms
    sys_ = S.triclinic_box(n, seed=args.seed)
    stream = torch.cuda.Stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        torch.cuda.synchronize()

    sampler = ClockSampler(0)
    sampler.start()
    d = D3(sys_["Z"], n, rc=RC, rc_cn=RC_CN, rc_atm=RC_ATM, damping=1, functional=0)
    d.set_cell(sys_["cell"])
    d.set_atoms(sys_["pos"], sys_["Z"])
    e, f, st = d.compute()
    ref = {"energy": e, "forces": f, "stress": st}
    step_ms, _, passes, _ = time_form(d, args, flush, stream, barrier)
    plain_launches = d.launches_per_eval()
    d.close()
    pm = {k: statistics.mean(p[k] for p in passes) for k in passes[0]}
    plain = {"value": n / (statistics.mean(step_ms) * 1e-3), "unit": "atoms/s", "ms_per_step": statistics.mean(step_ms),
             "passes_ms": pm, "three_body_ms": pm["atm_list"] + pm["atm"], "energy_ev": e}
    sur = surrogate_form(sys_, model, args, flush, stream, barrier, ref)
    clocks = sampler.stop()
    line = {"metric": "D3(BJ)+ATM atoms/s (E+F+stress), learned ATM surrogate vs the FP64 plain path",
            "value": sur["value"], "unit": "atoms/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sur["ms_per_step"], "higher_is_better": True, "data": "synthetic", "dtype": "bf16/f32/f64",
            "config": {"workload": "%d-atom triclinic box (benchmark generator scaled by (N/20000)^(1/3)), seed %d, "
                                   "held out from training; PBE-D3(BJ)+ATM rc 95 / 40 / 40 bohr" % (n, args.seed),
                       "form": "surrogate ATM (4 x MLP 128-128-128 SiLU, BF16 weights, FP32 accumulation) with exact "
                               "fallback above 0.2 meV ensemble std; other passes in the precision form",
                       "model": os.path.relpath(args.model, ROOT), "l2": "flushed between timed steps"},
            "plain": plain, "surrogate": sur,
            "three_body_speedup": plain["three_body_ms"] / sur["three_body_ms"],
            "end_to_end_speedup": sur["value"] / plain["value"],
            "gpu_launches": (sur["launches"] + plain_launches) * args.steps, "clocks": clocks}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--atoms", type=int, default=None,
                    help="atoms per box (default 20,000; 100,000 in --mode surrogate)")
    ap.add_argument("--ref-atoms", type=int, default=2000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", choices=["single", "batch", "md", "surrogate"], default="single")
    ap.add_argument("--system", choices=["triclinic", "water"], default="triclinic")
    ap.add_argument("--table", type=int, choices=[5, 7], default=5)
    ap.add_argument("--no-atm", action="store_true", help="two-body + CN only")
    ap.add_argument("--shard", action="store_true",
                    help="one structure over all ranks (strong scaling) instead of one replica per rank")
    ap.add_argument("--model", default=os.path.join(ROOT, "lasp-d3_b200", "surrogate", "atm_hcnosicu.d3s"))
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--tune-structs", type=int, default=128)
    ap.add_argument("--md-steps", type=int, default=200)
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="engine option for every handle of the run (name as in d3_b200: OPT_..., repeatable)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.mode in ("batch", "md"):
        args.atoms = args.atoms or N_ATOMS
    if args.mode == "batch":
        batch_mode(args)
        return
    if args.mode == "md":
        md_mode(args)
        return
    if args.mode == "surrogate":
        args.atoms = args.atoms or 100000
        surrogate_mode(args)
        return
    args.atoms = args.atoms or N_ATOMS
    if args.impl == "reference":
        reference_arm(args, world, rank, local)
    elif args.shard:
        shard_arm(args, world, rank, local)
    else:
        engine_arm(args, world, rank, local)


if __name__ == "__main__":
    main()
