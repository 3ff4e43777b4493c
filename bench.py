#!/usr/bin/env python3
"""Tree-gravity benchmark: particles/s of one force evaluation step on B200.

A step is one pass of the hot path over one system held in HBM: root cube,
Peano-Hilbert keys, radix sort, permutation, oct-tree build with FP64 moments,
and the relative-criterion walk (ErrTolForceAcc, OldAcc left on the device by
the previous step) -- what every GIZMO step pays when the tree is rebuilt.
The default workload is the 16,777,216-particle clustered system (1,000
Plummer clumps with log-normal masses plus a 20% uniform background), all
particles active; the same run also times a full rebuild plus the walk of a
seeded random 10% of the targets (individual timesteps).  Inputs are larger
than L2 (no flush needed).

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
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gizmo-public_b200"))

import ics  # noqa: E402
import multi  # noqa: E402

FLOPS_PER_INTERACTION = 20   # monopole force convention (3 sub, r^2, rsqrt, m/r^3, 3 fma)
# DRAM bytes (read + write) per particle of one k_walk launch on the galaxy,
# from the ncu capture of the 1,000,000-particle galaxy (114.8 MB read + 39.6 MB
# written); the walk's traffic grows with the particle count, so a launch of
# the 4.2M galaxy is scaled from it
# dram__bytes_read.sum + dram__bytes_write.sum of one k_walk launch: on the
# clustered system measured at full size (16,777,216 particles, groups of 64,
# a 1-pass capture: 4.77 GB read + 1.67 GB written); on the galaxy from the
# capture of the 1,000,000-particle galaxy (114.8 MB read + 39.6 MB written),
# scaled to the 4.2M galaxy by particle count
WALK_DRAM_BYTES_PER_PARTICLE = {"galaxy": 154.4, "galaxy1m": 154.4, "clustered": 6.36e9 / 16777216}
WALK_DRAM_SOURCE = {"galaxy": "ncu dram bytes of one k_walk launch on the 1M galaxy, scaled by N",
                    "galaxy1m": "ncu dram bytes of one k_walk launch on the 1M galaxy",
                    "clustered": "ncu dram bytes of one k_walk launch at full size (groups of 64; 1-pass capture)"}
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
        self.path = os.path.join(tempfile.gettempdir(), "gg_bench_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
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
def cpu_reference_rate(ic, seconds=15.0, seed=1, tol=0.0025, active_n=None):
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
            return ref_runner.rate(ic, seconds=seconds, seed=seed, tol=tol, active_n=active_n)
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


REF_BLOCKS, REF_BLOCK_LEN = 64, 1024   # PH-contiguous sample of the reference timing: 64 runs of 1,024 targets
REF_FULL_MAX = 262144                   # systems up to this size are walked whole by the reference


def reference_sample(ic, seed=1):
    """Targets the reference is timed on, as GIZMO walks them: the whole
    system when it is small, else runs of 1,024 particles consecutive in
    Peano-Hilbert order at seeded places along the curve (64 runs of 1,024)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    n = ic["pos"].shape[0]
    if n <= REF_FULL_MAX:
        return np.arange(n), "all %d targets" % n
    smp = ref_runner.ph_block_sample(ic["pos"], REF_BLOCKS, REF_BLOCK_LEN, seed=seed)
    return smp, "%d runs of %d targets consecutive in Peano-Hilbert order" % (REF_BLOCKS, REF_BLOCK_LEN)


def cpu_reference(ic, ref_tg, args, n_eval):
    """The reference (compiled GIZMO, OpenMP, all host threads) on this
    system, two bounded runs: (1) its forces on the sampled targets `ref_tg`
    (random), with their walk time; (2) its timing on a Peano-Hilbert
    contiguous sample, the order GIZMO's own walk takes.  Each run times one
    rebuild (domain_Decomposition + tree build) and one walk of its sample on
    the resident tree.  Returns (cpu_baseline, reference results on ref_tg);
    the C restatement stands in, without forces, where the compiled reference
    cannot run."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.available():
        return cpu_reference_rate(ic, seconds=args.cpu_seconds, tol=args.tol, active_n=n_eval), None
    n = ic["pos"].shape[0]
    r_rand, i_rand = ref_runner.steps_rate(ic, steps=1, warmup=0, sample=ref_tg, tol=args.tol, active_n=n_eval,
                                           sample_kind="%d seeded random targets" % ref_tg.size)
    smp, kind = reference_sample(ic)
    if smp.size == n:
        r_ph, i_ph = r_rand, i_rand
        if ref_tg.size != n:
            r_ph, i_ph = ref_runner.steps_rate(ic, steps=1, warmup=0, sample=smp, tol=args.tol, active_n=n_eval,
                                               sample_kind=kind)
    else:
        r_ph, i_ph = ref_runner.steps_rate(ic, steps=1, warmup=0, sample=smp, tol=args.tol, active_n=n_eval,
                                           sample_kind=kind)
    v_ph, v_rand = float(np.mean(r_ph)), float(np.mean(r_rand))
    cpu = {"value": v_ph, "unit": "particles/s", "cores": i_ph["cores"], "kind": "reference",
           "sample": i_ph["sample"], "t_domain_s": i_ph["t_domain_s"], "t_build_s": i_ph["t_build_s"],
           "t_walk_per_particle_us": i_ph["t_walk_per_particle_us"], "timed_walk_s": i_ph["step_s"],
           "t_walk_fixed_s": i_ph["t_walk_fixed_s"], "t_empty_walk_s": i_ph["t_empty_walk_s"],
           "model": "n / (t_domain + t_build + t_walk_fixed + t_walk_per_particle x n)",
           "random_sample": {"value": v_rand, "sample": i_rand["sample"],
                             "t_walk_per_particle_us": i_rand["t_walk_per_particle_us"]},
           "random_over_ph_blocks": v_rand / v_ph, "host_cpu": host_cpu()}
    res = {"acc": i_rand["acc"], "pot": i_rand["pot"]}
    if i_rand.get("startup") and ref_tg.size:
        # the reference's own interactions per target (Costtotal of its relative pass over the sample)
        res["interactions_per_target"] = float(i_rand["startup"]["cost_rel"]) / ref_tg.size
    return cpu, res


def subset_reference_rate(cpu, n_sub):
    """The reference's targets/s for a step that rebuilds and walks n_sub
    targets, from the same measured rebuild and per-target walk time."""
    per = cpu["t_walk_per_particle_us"] * 1e-6
    t = cpu["t_domain_s"] + cpu["t_build_s"] + cpu.get("t_walk_fixed_s", 0.0) + per * n_sub
    return {"value": n_sub / t, "unit": "targets/s",
            "cores": cpu["cores"], "kind": cpu["kind"],
            "sample": "the all-active run's measured rebuild and walk time per target (%s)" % cpu["sample"]}


def host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return "%s x %d" % (line.split(":", 1)[1].strip(), os.cpu_count() or 1)
    except OSError:
        pass
    return None


def run_reference_arm(args):
    """Time the reference's own CPU tree gravity (compiled GIZMO, OpenMP, all
    host threads) on this arm's workload.  Small systems: W+K whole steps
    (domain_Decomposition + tree build + relative walk of every particle).
    Large systems: one measured rebuild, then W+K timed walks of a bounded
    Peano-Hilbert contiguous sample of targets on the resident tree; `value` is
    the modelled rate of a whole step from those measured parts, and
    `ms_per_step` the timed sample steps' own mean duration."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload in ("ensemble", "serve"):
        return run_reference_arm_systems(args)
    name, gen = WORKLOADS[args.workload]
    ic = gen(SEEDS[args.workload])
    n = ic["pos"].shape[0]
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    active_n = int(round(args.active_frac * n)) if args.active_frac < 1.0 else None
    if not ref_runner.available():
        vals = [cpu_reference_rate(ic, seconds=args.ref_seconds, seed=1000 + i, tol=args.tol)
                for i in range(args.warmup + args.steps)][args.warmup:]
        v = float(np.mean([x["value"] for x in vals]))
        info = vals[-1]
        step_ms, extra = 1e3 * n / v, {}
    else:
        smp, kind = reference_sample(ic)
        whole = smp.size == n and active_n is None
        rates, info = ref_runner.steps_rate(ic, steps=args.steps, warmup=args.warmup, sample=smp, tol=args.tol,
                                            active_n=active_n, rebuild_steps="all" if whole else 1, sample_kind=kind)
        v = float(np.mean(rates))
        step_ms = 1e3 * float(np.mean(info["step_s"]))
        extra = {"timed_step": "whole step (domain + build + walk of every particle)" if whole else
                 "walk of the sample on the resident tree (the rebuild is timed once and enters the model)",
                 "model": "n / (t_domain + t_build + t_walk_fixed + t_walk_per_particle x n)",
                 "t_domain_s": info["t_domain_s"], "t_build_s": info["t_build_s"],
                 "t_walk_fixed_s": info["t_walk_fixed_s"], "t_empty_walk_s": info["t_empty_walk_s"],
                 "t_walk_per_particle_us": info["t_walk_per_particle_us"],
                 "model_ms_per_full_step": 1e3 * n / v if active_n is None else 1e3 * active_n / v}
        if args.calibrate:
            extra["calibration"] = reference_calibration(ic, args, active_n, v, kind)
    out = {"metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "n": n, "err_tol_force_acc": args.tol,
                      "active": active_n if active_n is not None else n},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "particles/s", "cores": info["cores"], "kind": info["kind"],
                            "sample": info["sample"], "host_cpu": host_cpu()},
           "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    out.update(extra)
    print(json.dumps(out), flush=True)
    return 0


def reference_calibration(ic, args, active_n, v_main, kind_main):
    """The same reference rate from other target samples: seeded random
    targets, and (small systems) a Peano-Hilbert block sample beside the whole
    step, so that the sample model can be checked against a full walk."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    n = ic["pos"].shape[0]
    out = {"main": {"value": v_main, "sample": kind_main}}
    r, i = ref_runner.steps_rate(ic, steps=2, warmup=0, sample=min(16384, n // 4), tol=args.tol, active_n=active_n)
    out["random"] = {"value": float(np.mean(r)), "sample": i["sample"],
                     "t_walk_per_particle_us": i["t_walk_per_particle_us"]}
    if n <= REF_FULL_MAX:
        smp = ref_runner.ph_block_sample(ic["pos"], 4, 1024, seed=3)
        r, i = ref_runner.steps_rate(ic, steps=2, warmup=0, sample=smp, tol=args.tol, active_n=active_n,
                                     sample_kind="4 runs of 1,024 targets consecutive in Peano-Hilbert order")
        out["ph_blocks"] = {"value": float(np.mean(r)), "sample": i["sample"],
                            "t_walk_per_particle_us": i["t_walk_per_particle_us"]}
    for k in list(out):
        if k != "main":
            out[k]["over_main"] = out[k]["value"] / v_main
    return out


# ---------------------------------------------------------------- batched ensemble
ENSEMBLE_NAME = "ensemble_4096_plummer_king_w6_n256_65536"


def ensemble_error_targets(counts, per_system=16, seed=4242):
    """Seeded sample of up to `per_system` targets in every system: (system, global index) pairs."""
    rng = np.random.default_rng(seed)
    off = np.concatenate([[0], np.cumsum(counts)])
    sys_of, idx = [], []
    for s, n in enumerate(counts):
        k = min(per_system, int(n))
        idx.append(off[s] + np.sort(rng.choice(int(n), k, replace=False)))
        sys_of.append(np.full(k, s))
    return np.concatenate(sys_of), np.concatenate(idx)


def ensemble_direct(ic, d_pos, d_mass, d_h, counts, sys_of, idx, stream, dev):
    """FP64 direct sum of every sampled target against the sources of its own system."""
    import torch
    import ggb200
    off = np.concatenate([[0], np.cumsum(counts)])
    acc = np.empty((idx.size, 3))
    d_acc = torch.empty((idx.size, 3), dtype=torch.float64, device=dev)
    d_pot = torch.empty(idx.size, dtype=torch.float64, device=dev)
    d_tg = torch.from_numpy((idx - off[sys_of]).astype(np.int32)).to(dev)
    starts = np.flatnonzero(np.r_[True, sys_of[1:] != sys_of[:-1]])
    ends = np.r_[starts[1:], idx.size]
    for a, b in zip(starts, ends):
        s = int(sys_of[a])
        o, n = int(off[s]), int(counts[s])
        ggb200.direct_sum_fp64(d_pos[o:o + n], d_mass[o:o + n], d_h[o:o + n], n, d_tg[a:b], int(b - a),
                               d_acc[a:b], d_pot[a:b], stream.cuda_stream)
    torch.cuda.synchronize()
    acc[:] = d_acc.cpu().numpy()
    return acc


def systems_reference_rate(systems, tol, what):
    """The reference (compiled GIZMO, all host threads) run on whole systems,
    one process per system as it would run them: particles/s = sum of N / sum
    of (domain + build + walk) step times."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_runner
    if not ref_runner.available():
        return None
    n_tot, t_tot, cores = 0, 0.0, os.cpu_count() or 1
    failed = []
    for sub in systems:
        n = int(sub["pos"].shape[0])
        try:
            rates, info = ref_runner.steps_rate(sub, steps=1, warmup=0, sample=n, tol=tol, rebuild_steps="all")
        except RuntimeError as e:
            # the reference's own limits can end a run (e.g. its top-node
            # allocation in force_create_empty_nodes on a small system): that
            # system is left out of the rate and named in the sample text
            failed.append("%d particles: %s" % (n, str(e).splitlines()[-1][-160:] if str(e) else "failed"))
            continue
        n_tot += n
        t_tot += n / rates[0]
        cores = info["cores"]
    if not n_tot:
        return None
    return {"value": n_tot / t_tot, "unit": "particles/s", "cores": cores, "kind": "reference",
            "sample": "GIZMO's own domain_Decomposition + tree build + relative walk (compiled reference, FP64, "
                      "OpenMP %d threads), all particles active, on %d seeded whole systems of the %s "
                      "(%d particles), one run per system%s" % (
                          cores, len(systems) - len(failed), what, n_tot,
                          "; %d system(s) left out, where the reference itself stopped: %s" % (
                              len(failed), " | ".join(failed)) if failed else "")}


def ensemble_reference_rate(ic, tol, n_sample=16, seed=77):
    counts = ic["counts"]
    off = np.concatenate([[0], np.cumsum(counts)])
    pick = np.sort(np.random.default_rng(seed).choice(counts.size, n_sample, replace=False))
    subs = [{k: ic[k][int(off[s]):int(off[s]) + int(counts[s])] for k in ("pos", "vel", "mass", "h")} for s in pick]
    return systems_reference_rate(subs, tol, "ensemble")


def run_ensemble(args, torch, ggb200, dist, world, rank, local):
    """4,096 independent clusters: one batched build + walk of every system per
    step, autotuned and replayed as one CUDA graph, against the plain form
    (one gg_load/gg_build/gg_evaluate per system) at the same opening tolerance."""
    ic = ics.ensemble(seed=multi.rank_seed(ics.SEED_ENSEMBLE, rank))
    counts = np.asarray(ic["counts"], dtype=np.int64)
    n = int(counts.sum())
    S = counts.size
    off = np.concatenate([[0], np.cumsum(counts)])
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    rec = ggb200.make_records(ic["pos"], ic["mass"], ic["h"])
    d_rec = torch.from_numpy(rec.view(np.uint8)).to(dev)
    d_acc = torch.empty((n, 3), dtype=torch.float64, device=dev)
    d_pot = torch.empty(n, dtype=torch.float64, device=dev)
    tol = args.tol

    tree = ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
                              blocks_per_sm=args.blocks_per_sm, group_order=args.group_order,
                              node_staging=args.node_staging)
    tree.set_stream(stream.cuda_stream)
    tree.load_device(d_rec, counts)
    tree.build()
    tree.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)            # start-up BH pass: OldAcc
    tree.build()
    tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=tol)         # first relative pass
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tuned, tuned_ms = tree.autotune(err_tol_force_acc=tol) if not args.no_autotune else (None, None)
    t_tune = time.perf_counter() - t0

    # uncaptured batched step (also allocates every buffer the capture reuses)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ev[0].record(stream)
    tree.build()
    ev[1].record(stream)
    tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=tol)
    ev[2].record(stream)
    torch.cuda.synchronize()
    plain_batched_ms = ev[0].elapsed_time(ev[2])
    build_ms, walk_ms = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    st = tree.last_stats()
    if st["error_word"]:
        raise RuntimeError("device error word %d" % st["error_word"])
    inter = st["interactions"]

    tree.capture_step(d_acc, d_pot, err_tol_force_acc=tol)
    for _ in range(args.warmup):
        tree.launch_step()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ggb200.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        tree.launch_step()
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = ggb200.kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = multi.max_over_ranks(dist, e0.elapsed_time(e1), device=dev)
    n_all = multi.sum_over_ranks(dist, n, device=dev)
    ms_step = total_ms / args.steps
    value = n_all / (ms_step * 1e-3)
    st = tree.last_stats()
    if st["error_word"]:
        raise RuntimeError("device error word %d after graph replays" % st["error_word"])
    acc_b = d_acc.cpu().numpy()
    old = torch.linalg.norm(d_acc, dim=1).contiguous()

    # plain form: one load + build + evaluate per system, same tolerance and OldAcc
    d_acc_p = torch.empty((n, 3), dtype=torch.float64, device=dev)
    d_pot_p = torch.empty(n, dtype=torch.float64, device=dev)
    plain = ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
                               blocks_per_sm=args.blocks_per_sm, group_order=args.group_order,
                              node_staging=args.node_staging)
    plain.set_stream(stream.cuda_stream)

    def plain_pass():
        for s in range(S):
            o, m = int(off[s]), int(counts[s])
            plain.load_device(d_rec[o * 32:(o + m) * 32], [m])
            plain.build()
            plain.evaluate_device(d_acc_p[o:o + m], d_pot_p[o:o + m], d_old_acc=old[o:o + m],
                                  err_tol_force_acc=tol)
    plain_pass()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    plain_pass()
    p1.record(stream)
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    plain.close()
    acc_p = d_acc_p.cpu().numpy()

    # force errors: FP64 direct sum inside each system, 16 sampled targets per system
    d_pos = torch.from_numpy(ic["pos"]).to(dev)
    d_mass = torch.from_numpy(ic["mass"]).to(dev)
    d_h = torch.from_numpy(ic["h"]).to(dev)
    sys_of, idx = ensemble_error_targets(counts)
    acc_dir = ensemble_direct(ic, d_pos, d_mass, d_h, counts, sys_of, idx, stream, dev)
    del d_pos, d_mass, d_h
    b50, b99, eb = ics.error_stats(acc_b[idx], acc_dir)
    q50, q99, _ = ics.error_stats(acc_p[idx], acc_dir)
    worst_sys = float(max(np.percentile(eb[sys_of == s], 99) for s in np.unique(sys_of)[:64]))

    peak32 = ggb200.fp32_peak_tflops(stream.cuda_stream)
    walk_tflops = inter * FLOPS_PER_INTERACTION / (walk_ms * 1e-3) / 1e12

    e2e = None
    if not args.no_e2e and rank == 0:
        with ggb200.GravityTree(leaf_size=tuned["leaf_size"] if tuned else args.leaf,
                                group_size=tuned["group_size"] if tuned else args.group,
                                flush=tuned["flush"] if tuned else args.flush, device=local,
                                blocks_per_sm=tuned["blocks_per_sm"] if tuned else args.blocks_per_sm,
                                node_staging=tuned["node_staging"] if tuned else args.node_staging) as te:
            old_h = np.linalg.norm(acc_b, axis=1)

            def e2e_step():
                te.load(ic["pos"], ic["mass"], ic["h"], counts=counts)
                te.build()
                return te.evaluate(old_acc=old_h, err_tol_force_acc=tol)
            e2e_step()
            t0 = time.perf_counter()
            ke = 3
            for _ in range(ke):
                e2e_step()
            dt = (time.perf_counter() - t0) / ke
        e2e = {"value": n / dt, "unit": "particles/s", "h2d_bytes_per_step": int(n * (32 + 8)),
               "d2h_bytes_per_step": int(n * (24 + 8)), "ms_per_step": dt * 1e3,
               "path": "gg_load_particles (host FP64 arrays, 4096 systems) + gg_build + gg_evaluate (host outputs)"}

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        cpu = ensemble_reference_rate(ic, tol)

    out = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": ENSEMBLE_NAME, "n_systems": S, "n": n, "n_total": int(n_all),
                   "err_tol_force_acc": tol, "tuned": tuned, "autotune_walk_ms": tuned_ms, "autotune_s": t_tune,
                   "step": "one CUDA graph: extent+keys+sort+record gather+tree+moments+relative walk of every system",
                   "l2": "inputs larger than L2 (1.5 GB of records)",
                   "parallelism": "independent ensemble per GPU" if world > 1 else "1 GPU"},
        "batched_vs_plain": {"graph_ms": ms_step, "batched_uncaptured_ms": plain_batched_ms, "plain_ms": plain_ms,
                             "speedup": plain_ms / ms_step,
                             "plain_form": "per system: gg_load_particles_device + gg_build + gg_evaluate_device, "
                                           "default configuration, same OldAcc and tolerance"},
        "force_error": {"p50": b50, "p99": b99, "plain_p50": q50, "plain_p99": q99, "targets": int(idx.size),
                        "worst_system_p99_first64": worst_sys,
                        "vs": "FP64 direct sum inside each system (GPU, same pair rule)"},
        "interactions_per_step": inter, "interactions_per_s": inter / (ms_step * 1e-3),
        "interactions_per_particle": inter / n,
        "stage_ms": {"build": build_ms, "walk": walk_ms},
        "roofline": {"bound": "fp32", "kernel": "k_walk", "achieved": walk_tflops, "peak": peak32,
                     "unit": "TFLOP/s", "frac": walk_tflops / peak32, "traffic": None,
                     "flops_per_interaction": FLOPS_PER_INTERACTION,
                     "peak_source": "measured FP32 FMA probe (gg_fp32_peak_probe) on this GPU"},
        "clocks": clk, "gpu_launches": int(launches), "e2e": e2e, "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    tree.close()
    if dist:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- serving stream
SERVE_NAME = "serve_poisson_2000rps_plummer_hernquist_clumpy_n1e3_1e6_reeval30"


def _copy_trace(reqs):
    import serve
    return [serve.Request(r.rid, r.kind, r.arrival, system=r.system, target=r.target, dt=r.dt) for r in reqs]


def run_serve(args, torch, ggb200, dist, world, rank, local):
    """Poisson arrivals of force-evaluation solves, served with continuous
    batching against a 120 GB device budget, then the same trace in the plain
    one-request-at-a-time form."""
    import serve
    pool = ics.serving_pool(n_systems=128, seed=multi.rank_seed(ics.SEED_SERVING, rank))
    trace = serve.make_trace(pool, rate=2000.0, window_s=args.serve_window, frac_reeval=0.3, dt=1e-3, recent=64,
                             seed=multi.rank_seed(ics.SEED_SERVING, rank) + 1)
    # warm-up on an offline slice of the trace: the library, the contexts, and
    # the process's cache of pinned staging blocks, which then holds blocks of
    # every size the batches ask for, as a long-running server's would
    # (page-locking them costs host time the first time only)
    warm = serve.Server(budget_bytes=120e9, tol=args.tol, reserve=True)   # maps the 120 GB budget once
    serve.run_trace(warm, _copy_trace(trace[:max(3, args.warmup) * 250]), realtime=False)
    warm.close()
    torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    launches0 = ggb200.kernel_launches()
    srv = serve.Server(budget_bytes=120e9, tol=args.tol, reserve=True)
    reqs = _copy_trace(trace)
    wall = serve.run_trace(srv, reqs, realtime=True)
    launches = ggb200.kernel_launches() - launches0
    clk = clocks.stop()
    st = serve.latency_stats(reqs)
    st.update(batches=srv.n_batches, evictions=srv.evictions, misses=sum(r.miss for r in reqs),
              peak_device_bytes=srv.peak_bytes, wall_s=wall)
    srv.close()

    plain = serve.Server(budget_bytes=120e9, tol=args.tol, batching=False, reserve=True)
    preqs = _copy_trace(trace)
    pwall = serve.run_trace(plain, preqs, realtime=True)
    pst = serve.latency_stats(preqs)
    pst.update(batches=plain.n_batches, evictions=plain.evictions, misses=sum(r.miss for r in preqs),
               peak_device_bytes=plain.peak_bytes, wall_s=pwall)
    plain.close()

    # force error of a seeded sample of served results, FP64 direct sum at the served positions
    dev = torch.device("cuda", local)
    rng = np.random.default_rng(9)
    errs, worst = [], 0.0
    drift_acc = {}
    for r in reqs:
        sid = r.rid if r.kind == "new" else r.target
        drift_acc[r.rid] = sum(q.dt for q in reqs if q.kind == "reeval" and q.target == sid and q.rid <= r.rid)
    pick = rng.choice(len(reqs), min(24, len(reqs)), replace=False)
    same_alone = 0
    for i in pick:
        r = reqs[i]
        s = r.system if r.kind == "new" or r.miss else next(q.system for q in reqs if q.rid == r.target)
        pos = s["pos"] + s["vel"] * drift_acc[r.rid] if drift_acc[r.rid] else s["pos"]
        n = pos.shape[0]
        ne = min(2048, n)
        tg = np.sort(rng.choice(n, ne, replace=False)).astype(np.int32)
        dp, dm, dh = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (pos, s["mass"], s["h"]))
        dacc = torch.empty((ne, 3), dtype=torch.float64, device=dev)
        dpot = torch.empty(ne, dtype=torch.float64, device=dev)
        ggb200.direct_sum_fp64(dp, dm, dh, n, torch.from_numpy(tg).to(dev), ne, dacc, dpot, None)
        torch.cuda.synchronize()
        _, p99, e = ics.error_stats(r.acc[tg], dacc.cpu().numpy())
        errs.append(e)
        worst = max(worst, p99)
        # the same request in the plain form (alone): identical result
        same_alone += int(np.array_equal(r.acc, preqs[i].acc))
    e_all = np.concatenate(errs)

    cpu = None
    if not args.no_cpu and rank == 0 and world == 1:
        small = sorted(pool, key=lambda x: x["pos"].shape[0])
        cpu = systems_reference_rate([small[k] for k in range(0, 64, 8)], args.tol, "serving pool")

    value = st["particles_per_s"]
    n_req = st["requests"]
    bytes_in = sum(r.n * (32 + 24) for r in reqs if r.kind == "new" or r.miss)
    bytes_out = sum(r.n * 32 for r in reqs)
    out = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": n_req,
        "warmup": args.warmup, "ms_per_step": 1e3 * st["makespan_s"] / n_req, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": SERVE_NAME, "rate_per_s": 2000.0, "window_s": args.serve_window, "requests": n_req,
                   "reeval_fraction": 0.3, "drift_dt": 1e-3, "budget_bytes": 120e9, "err_tol_force_acc": args.tol,
                   "pool_systems": len(pool), "step": "one request: arrival to result in host memory",
                   "l2": "inputs streamed from host memory"},
        "serve": st, "plain": pst,
        "batched_vs_plain": {"particles_per_s_ratio": value / pst["particles_per_s"],
                             "p50_ratio": pst["p50_ms"] / st["p50_ms"], "p99_ratio": pst["p99_ms"] / st["p99_ms"]},
        "force_error": {"p50": float(np.median(e_all)), "p99": float(np.percentile(e_all, 99)),
                        "worst_request_p99": worst, "requests_checked": int(pick.size),
                        "same_as_plain": int(same_alone), "vs": "FP64 direct sum at the served positions"},
        "clocks": clk, "gpu_launches": int(launches),
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": int(bytes_in / n_req),
                "d2h_bytes_per_step": int(bytes_out / n_req),
                "path": "serve.Server: gg_load_systems + gg_build + gg_evaluate_async / gg_drift_systems, "
                        "results fetched to host memory"},
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------- one system over the ranks
def run_split(args, torch, ggb200, dist, world, rank, local):
    """Strong scaling: one system of the workload, an equal share per rank;
    a step all-gathers the 32-byte records (NCCL), builds the whole tree on
    every rank and walks the rank's own particles (multi.SplitSystem)."""
    name, gen = WORKLOADS[args.workload]
    ic = gen(SEEDS[args.workload])             # the same system on every rank
    n = ic["pos"].shape[0]
    share = [n // world + (1 if r < n % world else 0) for r in range(world)]
    off = sum(share[:rank])
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    rec = ggb200.make_records(ic["pos"][off:off + share[rank]], ic["mass"][off:off + share[rank]],
                              ic["h"][off:off + share[rank]])
    d_rec = torch.from_numpy(rec.view(np.uint8)).to(dev)
    d_acc = torch.empty((share[rank], 3), dtype=torch.float64, device=dev)
    d_pot = torch.empty(share[rank], dtype=torch.float64, device=dev)
    tree = ggb200.GravityTree(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
                              blocks_per_sm=args.blocks_per_sm, target_order=args.target_order,
                              group_order=args.group_order, node_staging=args.node_staging)
    tree.set_stream(stream.cuda_stream)
    split = multi.SplitSystem(dist, tree, torch, dev)
    split.step(d_rec, d_acc, d_pot, err_tol_theta=0.7)
    for _ in range(args.warmup):
        split.step(d_rec, d_acc, d_pot, err_tol_force_acc=args.tol)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ggb200.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        split.step(d_rec, d_acc, d_pot, err_tol_force_acc=args.tol)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = ggb200.kernel_launches() - launches0
    clk = clocks.stop()
    ms_step = multi.max_over_ranks(dist, e0.elapsed_time(e1), device=dev) / args.steps
    st = tree.last_stats()
    out = {
        "metric": METRIC, "value": n / (ms_step * 1e-3), "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "n": n, "share": share, "err_tol_force_acc": args.tol,
                   "step": "all-gather of 32-byte records + extent+keys+sort+record gather+tree+moments on every rank + "
                           "relative walk of the rank's own particles",
                   "parallelism": "one system over %d GPUs" % world},
        "interactions_per_particle_rank0": st["interactions"] / max(share[rank], 1),
        "clocks": clk, "gpu_launches": int(launches), "e2e": None, "cpu_baseline": None,
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    tree.close()
    if dist:
        dist.destroy_process_group()
    return 0


def run_reference_arm_systems(args):
    """Reference arm of the many-system workloads: the compiled reference run on
    whole systems of the workload, one process per system, W+K samples of
    systems; particles/s = sum of N / sum of step times."""
    if args.workload == "ensemble":
        ic = ics.ensemble(seed=ics.SEED_ENSEMBLE)
        counts = ic["counts"]
        off = np.concatenate([[0], np.cumsum(counts)])
        rng = np.random.default_rng(77)
        systems = []
        for _ in range(args.warmup + args.steps):
            s = int(rng.integers(0, counts.size))
            systems.append({k: ic[k][int(off[s]):int(off[s + 1])] for k in ("pos", "vel", "mass", "h")})
        name, what = ENSEMBLE_NAME, "ensemble"
    else:
        pool = sorted(ics.serving_pool(n_systems=128, seed=ics.SEED_SERVING), key=lambda x: x["pos"].shape[0])
        systems = [pool[k] for k in range(0, 64, max(1, 64 // (args.warmup + args.steps)))][:args.warmup + args.steps]
        name, what = SERVE_NAME, "serving pool"
    info = systems_reference_rate(systems[args.warmup:], args.tol, what)
    if info is None:
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference (oracle/_ref) not built"}))
        return 0
    v = info["value"]
    out = {"metric": METRIC, "value": v, "unit": "particles/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": name, "err_tol_force_acc": args.tol}, "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "particles/s", "cores": info["cores"], "kind": info["kind"],
                            "sample": info["sample"]},
           "e2e": {"value": v, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


# ---------------------------------------------------------------- one system per GPU
def timed_steps(torch, stream, tree, walk, steps, build=None):
    """`steps` steps of build + walk between two CUDA events on the library's
    stream, with an event between build and walk.  Returns (total ms, mean
    build ms, mean walk ms)."""
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps + 1)]
    ev[0].record(stream)
    for k in range(steps):
        (build or tree.build)()
        ev[2 * k + 1].record(stream)
        walk()
        ev[2 * k + 2].record(stream)
    torch.cuda.synchronize()
    total = ev[0].elapsed_time(ev[-1])
    walk_ms = sum(ev[2 * k + 1].elapsed_time(ev[2 * k + 2]) for k in range(steps)) / steps
    build_ms = sum(ev[2 * k].elapsed_time(ev[2 * k + 1]) for k in range(steps)) / steps
    return total, build_ms, walk_ms


def sample_w(mass, pot):
    """1/2 sum m phi over a sample of targets."""
    return 0.5 * float(np.sum(mass * pot))


def reference_errors(ref, acc_dir, pot_dir, mass, acc_gpu, pot_gpu):
    """The reference tree's and this walk's errors on the same targets."""
    r50, r99, _ = ics.error_stats(ref["acc"], acc_dir)
    g50, g99, _ = ics.error_stats(acc_gpu, acc_dir)
    w_dir, w_ref, w_gpu = sample_w(mass, pot_dir), sample_w(mass, ref["pot"]), sample_w(mass, pot_gpu)
    return {"targets": int(acc_dir.shape[0]), "p50": g50, "p99": g99, "ref_p50": r50, "ref_p99": r99,
            "p50_vs_ref": g50 / r50, "p99_vs_ref": g99 / r99,
            "within_1p1_of_reference": bool(g50 <= 1.1 * r50 and g99 <= 1.1 * r99),
            "W_rel_err": abs(w_gpu - w_dir) / abs(w_dir), "ref_W_rel_err": abs(w_ref - w_dir) / abs(w_dir),
            "W_rel_diff_vs_ref": abs(w_gpu - w_ref) / abs(w_ref),
            "W_no_worse_than_ref_or_1e-5": bool(abs(w_gpu - w_dir) <= max(abs(w_ref - w_dir), 1e-5 * abs(w_dir))),
            "W": "1/2 sum m phi over these targets"}


def run_system(args, torch, ggb200, dist, world, rank, local):
    """One system per GPU (independent seeded systems per rank: weak scaling).
    A step = build (extent, keys, sort with the record gather, tree, moments) + relative walk
    of every particle, OldAcc left on the device by the previous step.  With
    --subset-frac (default 0.1 on the clustered system) a second timed loop
    walks a seeded random subset of targets on a full rebuild (individual
    timesteps), reported in the same line."""
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

    kw = dict(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
              blocks_per_sm=args.blocks_per_sm, target_order=args.target_order, group_order=args.group_order,
              node_staging=args.node_staging)
    tree = ggb200.GravityTree(**kw)
    tree.set_stream(stream.cuda_stream)
    tree.load_device(d_rec, [n])
    # start-up Barnes-Hut pass gives OldAcc (accel.c:47-50), then one relative
    # pass over all particles: every later step starts from a relative walk's
    # OldAcc, left on the device
    tree.build()
    tree.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)
    tree.build()
    tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)
    # the project's autotuner picks leaf and group size, flush threshold,
    # blocks per SM and node staging on this system, refusing any candidate
    # less accurate than the default configuration (outside the timed region)
    tuned, tuned_ms, t_tune = None, None, 0.0
    if not args.no_autotune:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tuned, tuned_ms = tree.autotune(err_tol_force_acc=args.tol)
        t_tune = time.perf_counter() - t0
        kw.update(leaf_size=tuned["leaf_size"], group_size=tuned["group_size"], flush=tuned["flush"],
                  blocks_per_sm=tuned["blocks_per_sm"], node_staging=tuned["node_staging"])
        tree.build()
        tree.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)

    act, d_act, na = None, None, n
    if args.active_frac < 1.0:
        act = ics.random_active(n, args.active_frac, seed=multi.rank_seed(77, rank)).astype(np.int32)
        na = int(act.size)
        d_act = torch.from_numpy(act).to(dev)

    def walker(t, d_a, n_a, acc_out, pot_out):
        def walk():
            if args.potential:
                t.evaluate_potential_device(pot_out, d_active=d_a, n_active=n_a, err_tol_force_acc=args.tol,
                                            err_tol_theta=0.0)
            else:
                t.evaluate_device(acc_out, pot_out, d_active=d_a, n_active=n_a, err_tol_force_acc=args.tol,
                                  err_tol_theta=0.0)
        return walk

    walk = walker(tree, d_act, na if act is not None else 0, d_acc, d_pot)
    for _ in range(args.warmup):
        tree.build()
        walk()
    torch.cuda.synchronize()
    if tree.last_stats()["error_word"]:
        raise RuntimeError("device error word %d" % tree.last_stats()["error_word"])
    # a step of every target replays two CUDA graphs, the build's and the
    # walk's launches, with an event between them; the same kernels, without
    # the host issuing some 150 launches per step
    graphs = act is None and not args.potential and not args.no_graph
    if graphs:
        tree.capture_step_parts(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)
        for _ in range(2):
            tree.launch_step_part(0)
            tree.launch_step_part(1)
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ggb200.kernel_launches()
    if graphs:
        total_ms, build_ms, walk_ms = timed_steps(torch, stream, tree, lambda: tree.launch_step_part(1), args.steps,
                                                  build=lambda: tree.launch_step_part(0))
    else:
        total_ms, build_ms, walk_ms = timed_steps(torch, stream, tree, walk, args.steps)
    if dist:
        dist.barrier()
    launches = ggb200.kernel_launches() - launches0
    clk = clocks.stop()
    total_ms = multi.max_over_ranks(dist, total_ms, device=dev)
    n_all = multi.sum_over_ranks(dist, na, device=dev)   # targets evaluated per step
    stats = tree.last_stats()
    if stats["error_word"]:
        raise RuntimeError("device error word %d in the timed steps" % stats["error_word"])
    ms_step = total_ms / args.steps
    value = n_all / (ms_step * 1e-3)
    inter = stats["interactions"]
    acc = d_acc[:na].cpu().numpy()
    pot = d_pot[:na].cpu().numpy()

    # individual timesteps: a random subset of targets walked on a full rebuild,
    # from the all-particle OldAcc the timed steps left (same for every rank)
    subset = None
    if args.subset_frac > 0 and act is None:
        sub = ics.random_active(n, args.subset_frac, seed=multi.rank_seed(77, rank)).astype(np.int32)
        d_sub = torch.from_numpy(sub).to(dev)
        d_acc_s = torch.empty((sub.size, 3), dtype=torch.float64, device=dev)
        d_pot_s = torch.empty(sub.size, dtype=torch.float64, device=dev)
        # a context of its own, from the default configuration, tuned on the
        # subset walk (sparser groups than the all-particle walk's); OldAcc of
        # every particle from the all-particle walk
        kw_s = dict(leaf_size=args.leaf, group_size=args.group, flush=args.flush, device=local,
                    blocks_per_sm=args.blocks_per_sm, target_order=args.target_order, group_order=args.group_order,
                    node_staging=args.node_staging)
        tsub = ggb200.GravityTree(**kw_s)
        tsub.set_stream(stream.cuda_stream)
        tsub.load_device(d_rec, [n])
        tsub.build()
        old_all = torch.linalg.norm(d_acc, dim=1).contiguous() if act is None else None
        tsub.evaluate_device(d_acc_s, d_pot_s, d_active=d_sub, n_active=int(sub.size), d_old_acc=old_all,
                             err_tol_force_acc=args.tol, err_tol_theta=0.0)
        tuned_s = None
        if not args.no_autotune:
            tuned_s, _ = tsub.autotune(err_tol_force_acc=args.tol, d_active=d_sub, n_active=int(sub.size))
        walk_s = walker(tsub, d_sub, int(sub.size), d_acc_s, d_pot_s)
        for _ in range(args.warmup):
            tsub.build()
            walk_s()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clocks_s = ClockSampler(local)
        clocks_s.start()
        time.sleep(0.3)
        tot_s, build_s, walk_s_ms = timed_steps(torch, stream, tsub, walk_s, args.steps)
        clk_s = clocks_s.stop()
        tot_s = multi.max_over_ranks(dist, tot_s, device=dev)
        n_sub_all = multi.sum_over_ranks(dist, int(sub.size), device=dev)
        st_s = tsub.last_stats()
        if st_s["error_word"]:
            raise RuntimeError("device error word %d in the subset steps" % st_s["error_word"])
        subset = {"active": int(sub.size), "fraction": args.subset_frac, "value": n_sub_all / (tot_s / args.steps * 1e-3),
                  "unit": "targets/s", "ms_per_step": tot_s / args.steps, "build_ms": build_s, "walk_ms": walk_s_ms,
                  "interactions_per_target": st_s["interactions"] / sub.size, "clocks": clk_s,
                  "step": "full rebuild + relative walk of a seeded random %g of the particles" % args.subset_frac,
                  "tuned": tuned_s,
                  "_targets": sub, "_acc": d_acc_s.cpu().numpy(), "_pot": d_pot_s.cpu().numpy()}
        del d_acc_s, d_pot_s
        tsub.close()

    # stage breakdown on one extra instrumented step (outside the timed region)
    tprof = ggb200.GravityTree(timing=True, **kw)
    tprof.set_stream(stream.cuda_stream)
    tprof.load_device(d_rec, [n])
    tprof.build()
    tprof.evaluate_device(d_acc, d_pot, err_tol_theta=0.7)
    # one relative walk first, so that the measured step starts, like the timed
    # steps, from a relative walk's OldAcc and group costs
    tprof.build()
    tprof.evaluate_device(d_acc, d_pot, err_tol_force_acc=args.tol, err_tol_theta=0.0)
    tprof.build()
    walker(tprof, d_act, na if act is not None else 0, d_acc, d_pot)()
    stages = tprof.last_stats()
    tprof.close()

    # force errors against the FP64 direct sum: a seeded sample of the outputs,
    # plus the targets the reference tree is run on (a seeded sample of the
    # subset, or of the active set), so that both trees are compared on the
    # same targets
    ne = min(args.err_targets, na)
    rows = np.sort(np.random.default_rng(12345).choice(na, ne, replace=False))   # rows of the outputs
    tg = (rows if act is None else act[rows]).astype(np.int32)                   # their particles
    pool = subset["_targets"] if subset else (act if act is not None else np.arange(n, dtype=np.int32))
    nref = min(args.ref_sample, pool.size)
    ref_pick = np.sort(np.random.default_rng(2468).choice(pool.size, nref, replace=False))
    ref_tg = pool[ref_pick].astype(np.int32)
    all_tg = np.concatenate([tg, ref_tg])
    dp = torch.from_numpy(ic["pos"]).to(dev)
    dm = torch.from_numpy(ic["mass"]).to(dev)
    dh = torch.from_numpy(ic["h"]).to(dev)
    dacc = torch.empty((all_tg.size, 3), dtype=torch.float64, device=dev)
    dpot = torch.empty(all_tg.size, dtype=torch.float64, device=dev)
    ggb200.direct_sum_fp64(dp, dm, dh, n, torch.from_numpy(all_tg).to(dev), all_tg.size, dacc, dpot,
                           stream.cuda_stream)
    torch.cuda.synchronize()
    acc_all_dir, pot_all_dir = dacc.cpu().numpy(), dpot.cpu().numpy()
    del dp, dm, dh, dacc, dpot
    acc_dir, pot_dir = acc_all_dir[:ne], pot_all_dir[:ne]
    acc_rdir, pot_rdir = acc_all_dir[ne:], pot_all_dir[ne:]
    if args.potential:   # the potential walk's own error: |phi - phi_direct| / |phi_direct|
        e = np.abs(pot[rows] - pot_dir) / np.maximum(np.abs(pot_dir), 1e-300)
        p50, p99 = float(np.median(e)), float(np.percentile(e, 99))
    else:
        p50, p99, _ = ics.error_stats(acc[rows], acc_dir)
    force_error = {"p50": p50, "p99": p99, "targets": ne, "vs": "FP64 direct sum (GPU, same pair rule)",
                   "W_rel_err_sample": abs(sample_w(ic["mass"][tg], pot[rows]) - sample_w(ic["mass"][tg], pot_dir))
                   / abs(sample_w(ic["mass"][tg], pot_dir))}

    # FP32 roofline of the walk (measured FMA peak on this GPU): the timed
    # steps' interactions x 20 flops over their walks' mean duration (CUDA
    # events on the walk's stream inside the timed region)
    peak32 = ggb200.fp32_peak_tflops(stream.cuda_stream)
    walk_tflops = inter * FLOPS_PER_INTERACTION / (walk_ms * 1e-3) / 1e12
    instrumented_tflops = (inter * FLOPS_PER_INTERACTION / (stages["ms_walk"] * 1e-3) / 1e12
                           if stages["ms_walk"] else None)

    # HBM roofline of the sort (268 B per element: 8 passes x 24 B + 8 B histogram read,
    # + 68 B of the record gather in the last pass: 32 B read, 32 B written, 4 B rank)
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        hbm_peak, hbm_src = float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except Exception:
        hbm_peak, hbm_src = 6650.0, "fallback 6.65 TB/s"
    sort_gbs = 268.0 * n / (stages["ms_sort"] * 1e-3) / 1e9 if stages["ms_sort"] else None

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e and rank == 0:
        old = np.linalg.norm(acc, axis=1) if act is None else torch.linalg.norm(
            tree_all_acc(tree, torch, dev, n, args.tol), dim=1).cpu().numpy()
        with ggb200.GravityTree(**kw) as te:
            out = (np.empty((na, 3)), np.empty(na))   # the caller's result arrays, reused every step

            def e2e_step():
                te.load(ic["pos"], ic["mass"], ic["h"])
                te.build()
                return te.evaluate(active=act, old_acc=old, err_tol_force_acc=args.tol, out=out)
            for _ in range(2):
                e2e_step()
            t0 = time.perf_counter()
            ke = max(3, min(args.steps, 5))
            for _ in range(ke):
                e2e_step()
            dt = (time.perf_counter() - t0) / ke
        e2e = {"value": na / dt, "unit": "particles/s",
               "h2d_bytes_per_step": int(n * (32 + 8) + (4 * na if act is not None else 0)),
               "d2h_bytes_per_step": int(na * (24 + 8)), "ms_per_step": dt * 1e3,
               "path": "gg_load_particles (host FP64 arrays) + gg_build + gg_evaluate (host outputs, OldAcc in)"}

    # the reference tree (compiled GIZMO, host cores) on the same system: its
    # forces on the sampled targets, and its timing, from two bounded runs
    cpu, ref_cmp, sub_cmp = None, None, None
    if not args.no_cpu and rank == 0 and world == 1 and not args.potential:
        cpu, ref_res = cpu_reference(ic, ref_tg, args, n_eval=na)
        if ref_res is not None:
            ref_rows = np.searchsorted(act, ref_tg) if act is not None else ref_tg
            ref_cmp = reference_errors(ref_res, acc_rdir, pot_rdir, ic["mass"][ref_tg], acc[ref_rows], pot[ref_rows])
            if subset:
                srows = np.searchsorted(subset["_targets"], ref_tg)
                sub_cmp = reference_errors(ref_res, acc_rdir, pot_rdir, ic["mass"][ref_tg], subset["_acc"][srows],
                                           subset["_pot"][srows])
                subset["cpu_baseline"] = subset_reference_rate(cpu, subset["active"])
    if ref_cmp:
        force_error["vs_reference_tree"] = ref_cmp
        if ref_res.get("interactions_per_target"):
            ref_cmp["reference_interactions_per_target"] = ref_res["interactions_per_target"]
    if subset:
        sp50, sp99, _ = ics.error_stats(subset["_acc"][np.searchsorted(subset["_targets"], ref_tg)], acc_rdir)
        subset["force_error"] = sub_cmp or {"p50": sp50, "p99": sp99, "targets": int(ref_tg.size)}
        for k in ("_targets", "_acc", "_pot"):
            subset.pop(k)

    out = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": name, "n": n, "active": na, "n_total": int(n_all), "err_tol_force_acc": args.tol,
                   "walk": "potential only (compute_potential)" if args.potential else "force and potential",
                   "step": "extent+keys+sort+record gather+tree+moments+relative walk (OldAcc on device)" +
                           (", replayed as two CUDA graphs (build, walk)" if graphs else ""),
                   "l2": "inputs larger than L2 (32 B/particle records, %d MB + tree)" % (32 * n // 10 ** 6),
                   "leaf_size": kw["leaf_size"], "group_size": kw["group_size"], "flush": kw["flush"],
                   "blocks_per_sm": kw["blocks_per_sm"] or 2,
                   "group_order": "by previous walk's cost" if args.group_order else "target order",
                   "node_staging": ["cp.async per lane", "bulk copies (TMA) per run"][kw["node_staging"]],
                   "autotuned": tuned is not None, "autotune_walk_ms": tuned_ms, "autotune_s": t_tune,
                   "parallelism": "independent system per GPU" if world > 1 else "1 GPU"},
        "force_error": force_error,
        "interactions_per_step": inter, "interactions_per_s": inter / (ms_step * 1e-3),
        "interactions_per_particle": inter / na,
        "stage_ms": {"keys": stages["ms_keys"], "sort": stages["ms_sort"], "build": stages["ms_build"],
                     "walk": stages["ms_walk"], "timed_build_phase": build_ms, "timed_walk_phase": walk_ms},
        "roofline": {"bound": "fp32", "kernel": "k_walk", "achieved": walk_tflops, "peak": peak32,
                     "unit": "TFLOP/s", "frac": walk_tflops / peak32,
                     "traffic": (WALK_DRAM_BYTES_PER_PARTICLE[args.workload] * n
                                 if args.workload in WALK_DRAM_BYTES_PER_PARTICLE else None),
                     "traffic_source": WALK_DRAM_SOURCE.get(args.workload),
                     "flops_per_interaction": FLOPS_PER_INTERACTION,
                     "peak_source": "measured FP32 FMA probe (gg_fp32_peak_probe) on this GPU",
                     "walk_ms": walk_ms, "instrumented_step_achieved": instrumented_tflops},
        "roofline_sort": {"bound": "hbm", "achieved": sort_gbs, "peak": hbm_peak, "unit": "GB/s",
                          "frac": (sort_gbs / hbm_peak) if sort_gbs else None, "bytes_per_element": 268,
                          "peak_source": hbm_src},
        "clocks": clk, "gpu_launches": int(launches), "e2e": e2e, "cpu_baseline": cpu,
    }
    if ref_cmp and ref_cmp.get("reference_interactions_per_target") and out["roofline"]["frac"]:
        # the same walk time credited with the reference tree's interaction
        # count only: the FP32 fraction of useful work
        ratio = ref_cmp["reference_interactions_per_target"] / (inter / na)
        out["roofline"]["frac_at_reference_interactions"] = out["roofline"]["frac"] * ratio
        out["roofline"]["interactions_vs_reference"] = 1.0 / ratio
    if subset:
        out["active_subset"] = subset
    if rank == 0:
        print(json.dumps(out), flush=True)
    tree.close()
    if dist:
        dist.destroy_process_group()
    return 0


def tree_all_acc(tree, torch, dev, n, tol):
    """|a| of every particle from one relative walk of all of them (OldAcc for
    the end-to-end leg when the timed walk covers a subset only)."""
    d_a = torch.empty((n, 3), dtype=torch.float64, device=dev)
    tree.build()
    tree.evaluate_device(d_a, None, err_tol_force_acc=tol, err_tol_theta=0.0)
    torch.cuda.synchronize()
    return d_a


# ---------------------------------------------------------------- GPU arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="clustered", choices=sorted(WORKLOADS) + ["ensemble", "serve"])
    # ErrTolForceAcc; by default per workload, the largest of 0.001 and 0.0008
    # that keeps the p99 force error below 2e-3 (the metric's bound) with a margin:
    # at 0.001 the galaxy's p99 is 1.77e-3 but the clustered system's 2.0e-3
    ap.add_argument("--tol", type=float, default=None)
    ap.add_argument("--err-targets", type=int, default=65536)
    ap.add_argument("--ref-seconds", type=float, default=8.0)
    ap.add_argument("--ref-sample", type=int, default=16384)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--leaf", type=int, default=8)
    ap.add_argument("--group", type=int, default=32)
    ap.add_argument("--flush", type=int, default=128)
    ap.add_argument("--blocks-per-sm", type=int, default=0)
    ap.add_argument("--target-order", type=int, default=1, choices=[0, 1])
    ap.add_argument("--node-staging", type=int, default=0, choices=[0, 1],
                    help="walk node staging: 0 per-lane cp.async, 1 bulk copies (TMA)")
    ap.add_argument("--group-order", type=int, default=1, choices=[0, 1],
                    help="1: walk groups handed out most expensive first, by the previous walk's costs")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="issue the timed steps' launches one by one")
    ap.add_argument("--serve-window", type=float, default=2.0)
    # individual timesteps: the timed walk evaluates a seeded random fraction of
    # the particles (the tree is still built over all of them)
    ap.add_argument("--active-frac", type=float, default=1.0)
    # a second timed loop in the same run: full rebuild + walk of a seeded
    # random fraction of the targets, reported as "active_subset" (default 0.1
    # on the clustered system, 0 = none elsewhere)
    ap.add_argument("--subset-frac", type=float, default=None)
    # reference arm: also time the reference on other target samples
    ap.add_argument("--calibrate", action="store_true")
    # one system shared by the ranks (strong scaling): each rank holds an equal
    # share, all-gathers the records each step and walks its own particles
    ap.add_argument("--split", action="store_true")
    # time the potential-only walk (compute_potential) instead of the force walk
    ap.add_argument("--potential", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.tol is None:
        args.tol = 0.0008 if args.workload.startswith("clustered") else 0.001
    if args.subset_frac is None:
        args.subset_frac = 0.1 if args.workload == "clustered" else 0.0

    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import ggb200

    world, rank, local = multi.world()
    torch.cuda.set_device(local)
    dist = multi.init("nccl")
    if args.workload == "ensemble":
        return run_ensemble(args, torch, ggb200, dist, world, rank, local)
    if args.workload == "serve":
        return run_serve(args, torch, ggb200, dist, world, rank, local)
    if args.split:
        return run_split(args, torch, ggb200, dist, world, rank, local)

    return run_system(args, torch, ggb200, dist, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
