#!/usr/bin/env python3
"""Tree-gravity benchmark: particles/s of one force evaluation step on B200.

A step is one pass of the hot path over one system held in HBM: root cube,
Peano-Hilbert keys, radix sort, permutation, oct-tree build with FP64 moments,
and the relative-criterion walk (ErrTolForceAcc, OldAcc left on the device by
the previous step) -- what every GIZMO step pays when the tree is rebuilt.
The default workload is the 4,194,304-particle galaxy (Hernquist halo +
exponential disk).  Inputs are larger than L2 (no flush needed).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank evaluates its own independent system (weak scaling,
no collective on the data path; the process group only carries the barrier
and the max-over-ranks timing).  --impl reference times the reference
algorithm on the host cores (compiled GIZMO objects when present, else the C
restatement) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gizmo-public_b200"))

import ics  # noqa: E402
import multi  # noqa: E402

FLOPS_PER_INTERACTION = 20   # monopole force convention (3 sub, r^2, rsqrt, m/r^3, 3 fma)
METRIC = "tree-gravity particles/s at p99 force err<=2e-3 vs FP64 direct; serve p50/p99 ms"

WORKLOADS = {
    "galaxy": ("galaxy_hernquist_halo_3000000_exp_disk_1194304", lambda seed: ics.galaxy(seed=seed)),
    "plummer": ("plummer_65536", lambda seed: ics.plummer(65536, seed=seed)),
    "clustered": ("clustered_1000_clumps_16777216", lambda seed: ics.clustered(seed=seed)),
    # small cases of the same models, used for ncu captures
    "galaxy1m": ("galaxy_hernquist_halo_715000_exp_disk_285000", lambda seed: ics.galaxy(715000, 285000, seed=seed)),
    "clustered1m": ("clustered_250_clumps_1048576", lambda seed: ics.clustered(1048576, seed=seed, n_clumps=250)),
}
SEEDS = {"galaxy": ics.SEED_GALAXY, "plummer": ics.SEED_PLUMMER, "clustered": ics.SEED_CLUSTERED,
         "galaxy1m": ics.SEED_GALAXY, "clustered1m": ics.SEED_CLUSTERED}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", "clocks_rank%d.csv" % index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["active", "hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names[1:], p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU baselines
def cpu_reference_rate(ic, seconds=15.0, seed=1, tol=0.0025):
    """Time the reference algorithm on the host cores on a bounded sample.

    Cost model of one step: tree build (serial in the reference) plus the walk
    of every particle; the walk is timed on a seeded random sample of targets
    and scaled to N.  Uses the compiled reference when present, else the C
    restatement in oracle/."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    try:
        import ref_runner
        if ref_runner.available():
            return ref_runner.rate(ic, seconds=seconds, seed=seed, tol=tol)
    except ImportError:
        pass
    n = ic["pos"].shape[0]
    cores = os.cpu_count() or 1
    old = np.linalg.norm(ic.get("acc_hint", np.zeros((n, 3))), axis=1) if "acc_hint" in ic else None
    if old is None:
        # OldAcc from a cheap BH pass over a small sample is not enough for all particles;
        # use |a| of the GPU pass when the caller supplied it, else the BH pass itself
        old = np.full(n, 0.0)
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    oracle.tree_gravity(ic["pos"], ic["mass"], ic["h"], old, tol, 0.0, targets=np.zeros(0, np.int32),
                        nthreads=cores)
    t_build = time.perf_counter() - t0
    ns = 256
    while True:
        tg = np.sort(rng.choice(n, ns, replace=False)).astype(np.int32)
        t0 = time.perf_counter()
        oracle.tree_gravity(ic["pos"], ic["mass"], ic["h"], old, tol, 0.0, targets=tg, nthreads=cores)
        t = time.perf_counter() - t0 - t_build
        if t > 0.25 * seconds or ns >= n:
            break
        ns = min(n, int(ns * max(2.0, 0.3 * seconds / max(t, 1e-3))))
    per = max(t, 1e-9) / ns
    step = t_build + per * n
    return {"value": n / step, "unit": "particles/s", "cores": cores, "kind": "port",
            "sample": "C restatement (oracle/gg_oracle.c, FP64, OpenMP): full tree build + relative walk of %d "
                      "seeded random targets of %d, walk time scaled to all targets" % (ns, n),
            "t_build_s": t_build, "t_walk_per_particle_us": per * 1e6}


def run_reference_arm(args):
    """Time the reference's own CPU tree gravity (all host threads) on this
    arm's workload: W+K steady-state steps, each a bounded sample of targets."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    name, gen = WORKLOADS[args.workload]
    ic = gen(SEEDS[args.workload])
    n = ic["pos"].shape[0]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if ref_runner.available():
        rates, info = ref_runner.steps_rate(ic, steps=args.steps, warmup=args.warmup, sample_n=args.ref_sample,
                                            tol=args.tol)
        v = float(np.mean(rates))
    else:
        vals = [cpu_reference_rate(ic, seconds=args.ref_seconds, seed=1000 + i, tol=args.tol)
                for i in range(args.warmup + args.steps)][args.warmup:]
        v = float(np.mean([x["value"] for x in vals]))
        info = vals[-1]
    out = {"metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1e3 * n / v, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "n": n, "err_tol_force_acc": args.tol},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "particles/s", "cores": info["cores"], "kind": info["kind"],
                            "sample": info["sample"]},
           "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="galaxy", choices=sorted(WORKLOADS))
    # 0.001 keeps the galaxy's p99 force error below 2e-3 (the metric's bound)
    ap.add_argument("--tol", type=float, default=0.001)
    ap.add_argument("--err-targets", type=int, default=65536)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--ref-sample", type=int, default=16384)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--leaf", type=int, default=8)
    ap.add_argument("--group", type=int, default=32)
    ap.add_argument("--flush", type=int, default=64)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import ggb200

    world, rank, local = multi.world()
    torch.cuda.set_device(local)
    dist = multi.init("nccl")

    name, gen = WORKLOADS[args.workload]
    ic = gen(multi.rank_seed(SEEDS[args.workload], rank))   # independent system per rank
    n = ic["pos"].shape[0]
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)   # every kernel and event of the bench goes on this stream
    torch.cuda.set_stream(stream)
    rec = ggb200.make_records(ic["pos"], ic["mass"], ic["h"])
    d_rec = torch.from_numpy(rec.view(np.uint8)).to(dev)
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    d_pot = torch.empty(n, dtype=torch.float64, device=dev)

    tree = ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush,
                              device=local, blocks_per_sm=args.blocks_per_sm)
    tree.set_stream(stream.cuda_stream)
    tree.load_device(d_rec, [n])
    # start-up Barnes-Hut pass gives OldAcc (accel.c:47-50), left on the device
    tree.build()
    tree.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)

    def step():
        tree.build()
        tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    st0 = tree.last_stats()
    if st0["error_word"]:
        raise RuntimeError("device error word %d" % st0["error_word"])

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ggb200.kernel_launches()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * args.steps + 1)]
    ev[0].record(stream)
    for k in range(args.steps):
        tree.build()
        ev[2 * k + 1].record(stream)
        tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)
        ev[2 * k + 2].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = ggb200.kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = ev[0].elapsed_time(ev[-1])
    walk_ms = sum(ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(args.steps)) / args.steps
    build_ms = (ev[0].elapsed_time(ev[1]) + sum(ev[2 * k].elapsed_time(ev[2 * k + 1])
                                                 for k in range(1, args.steps))) / args.steps
    total_ms = multi.max_over_ranks(dist, total_ms, device=dev)
    n_all = multi.sum_over_ranks(dist, n, device=dev)
    stats = tree.last_stats()
    ms_step = total_ms / args.steps
    value = n_all / (ms_step * 1e-3)
    inter = stats["interactions"]

    # stage breakdown on one extra instrumented step (outside the timed region)
    tprof = ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
                               timing=True, blocks_per_sm=args.blocks_per_sm)
    tprof.set_stream(stream.cuda_stream)
    tprof.load_device(d_rec, [n])
    tprof.build()
    tprof.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)
    tprof.build()
    tprof.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)
    stages = tprof.last_stats()
    tprof.close()

    # force error against the FP64 direct sum on a seeded subsample
    acc = d_acc.cpu().numpy()
    pot = d_pot.cpu().numpy()
    ne = min(args.err_targets, n)
    tg = np.sort(np.random.default_rng(12345).choice(n, ne, replace=False)).astype(np.int32)
    dp = torch.from_numpy(ic["pos"]).to(dev)
    dm = torch.from_numpy(ic["mass"]).to(dev)
    dh = torch.from_numpy(ic["h"]).to(dev)
    dacc = torch.empty((ne, 3), dtype=torch.float64, device=dev)
    dpot = torch.empty(ne, dtype=torch.float64, device=dev)
    ggb200.direct_sum_fp64(dp, dm, dh, n, torch.from_numpy(tg).to(dev), ne, dacc, dpot,
                           stream.cuda_stream)
    torch.cuda.synchronize()
    acc_dir, pot_dir = dacc.cpu().numpy(), dpot.cpu().numpy()
    p50, p99, _ = ics.error_stats(acc[tg], acc_dir)
    wsum = float(np.sum(ic["mass"][tg] * pot[tg]))
    wsum_dir = float(np.sum(ic["mass"][tg] * pot_dir))
    del dp, dm, dh, dacc, dpot

    # FP32 roofline of the walk (measured FMA peak on this GPU)
    peak32 = ggb200.fp32_peak_tflops(stream.cuda_stream)
    walk_tflops = inter * FLOPS_PER_INTERACTION / (stages["ms_walk"] * 1e-3) / 1e12 if stages["ms_walk"] else None
    walk_phase_tflops = inter * FLOPS_PER_INTERACTION / (walk_ms * 1e-3) / 1e12

    # HBM roofline of the sort (200 B per element: 8 passes x 24 B + 8 B histogram read)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    sort_gbs = 200.0 * n / (stages["ms_sort"] * 1e-3) / 1e9 if stages["ms_sort"] else None

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e and rank == 0:
        old = np.linalg.norm(acc, axis=1)
        with ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush,
                                device=local, blocks_per_sm=args.blocks_per_sm) as te:
            def e2e_step():
                te.load(ic["pos"], ic["mass"], ic["h"])
                te.build()
                return te.evaluate(old_acc=old, err_tol_force_acc=args.tol)
            for _ in range(2):
                e2e_step()
            t0 = time.perf_counter()
            ke = max(3, min(args.steps, 5))
            for _ in range(ke):
                e2e_step()
            dt = (time.perf_counter() - t0) / ke
        e2e = {"value": n / dt, "unit": "particles/s", "h2d_bytes_per_step": int(n * (32 + 8)),
               "d2h_bytes_per_step": int(n * (24 + 8)), "ms_per_step": dt * 1e3,
               "path": "gg_load_particles (host FP64 arrays) + gg_build + gg_evaluate (host outputs, OldAcc in)"}

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        ic_cpu = dict(ic)
        ic_cpu["acc_hint"] = acc
        cpu = cpu_reference_rate(ic_cpu, seconds=args.cpu_seconds, tol=args.tol)

    out = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "n": n, "n_total": int(n_all), "err_tol_force_acc": args.tol,
                   "step": "extent+keys+sort+permute+tree+moments+relative walk (OldAcc on device)",
                   "l2": "inputs larger than L2 (32 B/particle records, 134 MB + tree)",
                   "leaf_size": args.leaf, "group_size": args.group, "flush": args.flush,
                   "parallelism": "independent system per GPU" if world > 1 else "1 GPU"},
        "force_error": {"p50": p50, "p99": p99, "targets": ne, "vs": "FP64 direct sum (GPU, same pair rule)",
                        "pot_sum_rel_diff_sample": abs(wsum - wsum_dir) / abs(wsum_dir)},
        "interactions_per_step": inter, "interactions_per_s": inter / (ms_step * 1e-3),
        "interactions_per_particle": inter / n,
        "stage_ms": {"keys": stages["ms_keys"], "sort": stages["ms_sort"], "build": stages["ms_build"],
                     "walk": stages["ms_walk"], "timed_build_phase": build_ms, "timed_walk_phase": walk_ms},
        "roofline": {"bound": "fp32", "kernel": "k_walk", "achieved": walk_tflops, "peak": peak32,
                     "unit": "TFLOP/s", "frac": (walk_tflops / peak32) if walk_tflops else None,
                     "traffic": None, "flops_per_interaction": FLOPS_PER_INTERACTION,
                     "peak_source": "measured FP32 FMA probe (gg_fp32_peak_probe) on this GPU",
                     "timed_phase_achieved": walk_phase_tflops},
        "roofline_sort": {"bound": "hbm", "achieved": sort_gbs, "peak": hbm_peak, "unit": "GB/s",
                          "frac": (sort_gbs / hbm_peak) if sort_gbs else None, "bytes_per_element": 200,
                          "peak_source": hbm_src},
        "clocks": clk, "gpu_launches": int(launches), "e2e": e2e, "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    tree.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
