"""Run the reference code itself (oracle/_ref/gizmo_ref, built by build_ref.sh).

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py to produce
golden vectors, and by bench.py's reference arm / CPU baseline to time the
reference's own OpenMP tree gravity on the host cores.

Initial conditions go to the reference in its unformatted format-1 binary
(read_ic.c:721-730): a 256-byte header block, then POS, VEL, ID and MASS
blocks, each framed by Fortran record markers, positions and masses in FP64
(INPUT_IN_DOUBLEPRECISION).  Particle types carry the per-type softenings
(SofteningHalo = type 1, SofteningDisk = type 2).
"""
import os
import struct
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "gizmo_ref")
# GIZMO driving the B200 library through gizmo-public_b200/host/gravtree_b200.c
BIN_B200 = os.path.join(HERE, "_ref", "gizmo_b200")
BIN_POT = os.path.join(HERE, "_ref", "gizmo_ref_pot")   # variant with compute_potential (no EVALPOTENTIAL)
KERNEL_FAC = 2.8


def available(binary=None):
    binary = binary or BIN
    if not os.path.exists(binary):
        return False
    try:
        r = subprocess.run([binary], stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=30)
        return r.returncode == 2   # usage message: the binary runs on this host
    except Exception:
        return False


def _block(f, payload):
    n = len(payload)
    f.write(struct.pack("<i", n))
    f.write(payload)
    f.write(struct.pack("<i", n))


def write_ic(path, pos, vel, mass, types):
    """Format-1 IC file; particles must be grouped by type in increasing order."""
    types = np.asarray(types)
    assert np.all(np.diff(types) >= 0), "particles must be ordered by type"
    n = pos.shape[0]
    npart = [int(np.count_nonzero(types == t)) for t in range(6)]
    hdr = struct.pack("<6i", *npart)
    hdr += struct.pack("<6d", *([0.0] * 6))           # masses in the MASS block
    hdr += struct.pack("<dd", 0.0, 0.0)               # time, redshift
    hdr += struct.pack("<ii", 0, 0)                   # flag_sfr, flag_feedback
    hdr += struct.pack("<6I", *npart)                 # npartTotal
    hdr += struct.pack("<ii", 0, 1)                   # flag_cooling, num_files
    hdr += struct.pack("<dddd", 0.0, 0.0, 0.0, 1.0)   # BoxSize, OmegaMatter, OmegaLambda, HubbleParam
    hdr += struct.pack("<ii", 0, 0)                   # flag_stellarage, flag_metals
    hdr += struct.pack("<6I", *([0] * 6))             # npartTotalHighWord
    hdr += struct.pack("<iii", 0, 1, 0)               # entropy flag, flag_doubleprecision, flag_ic_info
    hdr += struct.pack("<f", 0.0)
    hdr += b"\0" * (256 - len(hdr))
    assert len(hdr) == 256
    with open(path, "wb") as f:
        _block(f, hdr)
        _block(f, np.ascontiguousarray(pos, dtype="<f8").tobytes())
        _block(f, np.ascontiguousarray(vel, dtype="<f8").tobytes())
        _block(f, np.arange(1, n + 1, dtype="<u4").tobytes())
        _block(f, np.ascontiguousarray(mass, dtype="<f8").tobytes())


PARAMS = """InitCondFile {ic}
OutputDir {out}
SnapshotFileBase snap
RestartFile restart
ResubmitOn 0
ResubmitCommand none
OutputListFilename none
OutputListOn 0
Omega0 0
OmegaBaryon 0
OmegaLambda 0
OmegaRadiation 0
HubbleParam 1
BoxSize 0
MaxMemSize {memmb}
TimeOfFirstSnapshot 1e10
CpuTimeBetRestartFile 1e10
TimeBetStatistics 1e10
TimeBegin 0
TimeMax 1
TimeBetSnapshot 1e10
UnitVelocity_in_cm_per_s 1
UnitLength_in_cm 1
UnitMass_in_g 1
UnitMagneticField_in_gauss 1
GravityConstantInternal 1
TreeDomainUpdateFrequency 0.0
MaxSizeTimestep 0.01
MinSizeTimestep 0
ComovingIntegrationOn 0
ICFormat 1
SnapFormat 1
NumFilesPerSnapshot 1
NumFilesWrittenInParallel 1
TimeLimitCPU 1e9
SofteningGas {eps1}
SofteningHalo {eps1}
SofteningDisk {eps2}
SofteningBulge {eps1}
SofteningStars {eps1}
SofteningBndry {eps1}
SofteningGasMaxPhys {eps1}
SofteningHaloMaxPhys {eps1}
SofteningDiskMaxPhys {eps2}
SofteningBulgeMaxPhys {eps1}
SofteningStarsMaxPhys {eps1}
SofteningBndryMaxPhys {eps1}
BufferSize 200
PartAllocFactor 2.0
InitGasTemp 0
MinGasTemp 0
DesNumNgb 32
MaxHsml 1e10
MinGasHsmlFractional 0
"""


def types_and_eps(h):
    """Map per-particle kernel radii to GIZMO particle types 1 and 2."""
    h = np.asarray(h, dtype=np.float64)
    vals = sorted(np.unique(h).tolist(), reverse=True)
    if len(vals) > 2:
        raise ValueError("the reference harness supports at most two softenings")
    t = np.where(h == vals[0], 1, 2)
    eps1 = vals[0] / KERNEL_FAC
    eps2 = (vals[1] if len(vals) > 1 else vals[0]) / KERNEL_FAC
    return t, eps1, eps2


def run(ic, tol=0.0025, steps=0, sample=None, threads=None, workdir=None, timeout=3600, binary=None,
        sample_only=False, drift_dt=0.0, rebuild_steps=None):
    """Run the reference: start-up evaluation (BH pass, relative pass) and
    optional steady-state steps (the first `rebuild_steps` of them rebuild,
    the others walk the resident tree again; default: all rebuild).  Returns
    dict with acc (pre-G = acc/G with G = 1), pot, oldacc in input order,
    interaction counts and timings."""
    pos, mass, h = ic["pos"], ic["mass"], ic["h"]
    vel = ic.get("vel", np.zeros_like(pos))
    n = pos.shape[0]
    t, eps1, eps2 = types_and_eps(h)
    order = np.argsort(t, kind="stable")   # the file groups particles by type
    own = workdir is None
    d = workdir or tempfile.mkdtemp(prefix="gg_ref_")
    try:
        icp = os.path.join(d, "ics")
        write_ic(icp, pos[order], vel[order], mass[order], t[order])
        os.makedirs(os.path.join(d, "out"), exist_ok=True)
        memmb = int(1000 + n * 3000 / 1e6)
        with open(os.path.join(d, "params"), "w") as f:
            f.write(PARAMS.format(ic=icp, out=os.path.join(d, "out"), memmb=memmb, eps1=repr(eps1), eps2=repr(eps2)))
        args = [binary or BIN, os.path.join(d, "params"), repr(tol), os.path.join(d, "res.bin")]
        if steps or sample is not None or drift_dt > 0 or rebuild_steps is not None:
            sp = "-"
            if sample is not None:
                sp = os.path.join(d, "sample.bin")
                # IDs in the file are positions in the type-ordered file, plus one
                inv = np.empty(n, np.int64)
                inv[order] = np.arange(n)
                (inv[np.asarray(sample)] + 1).astype("<i8").tofile(sp)
            args += [str(steps), sp, "1" if sample_only else "0", repr(float(drift_dt)),
                     str(steps if rebuild_steps is None else int(rebuild_steps))]
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        t0 = time.perf_counter()
        r = subprocess.run(args, cwd=d, stdout=subprocess.PIPE, stderr=subprocess.PIPE, env=env, timeout=timeout)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError("reference run failed (%d): %s" % (r.returncode, r.stdout.decode()[-2000:] +
                                                                  r.stderr.decode()[-2000:]))
        rec = np.fromfile(os.path.join(d, "res.bin"), dtype=np.dtype([("id", "<u8"), ("v", "<f8", 5)]))
        ids = rec["id"].astype(np.int64) - 1
        out = np.empty((n, 5))
        out[order[ids]] = rec["v"]
        info = {"wall_s": wall, "steps": []}
        bh = np.fromfile(os.path.join(d, "res.bin.bh"), dtype=rec.dtype)
        out_bh = np.empty((n, 5))
        out_bh[order[bh["id"].astype(np.int64) - 1]] = bh["v"]
        kr = np.fromfile(os.path.join(d, "res.bin.keys"), dtype=np.dtype([("id", "<u8"), ("hi", "<u8"), ("lo", "<u8")]))
        keys_hi = np.empty(n, np.uint64)
        keys_lo = np.empty(n, np.uint64)
        kidx = order[kr["id"].astype(np.int64) - 1]
        keys_hi[kidx], keys_lo[kidx] = kr["hi"], kr["lo"]
        res_extra = {}
        pot_path = os.path.join(d, "res.bin.pot")
        if os.path.exists(pot_path):
            pr = np.fromfile(pot_path, dtype=np.dtype([("id", "<u8"), ("v", "<f8")]))
            pot_only = np.empty(n)
            pot_only[order[pr["id"].astype(np.int64) - 1]] = pr["v"]
            res_extra["pot_only"] = pot_only
        if drift_dt > 0:
            dr = np.fromfile(os.path.join(d, "res.bin.drift"), dtype=rec.dtype)
            out_dr = np.empty((n, 5))
            out_dr[order[dr["id"].astype(np.int64) - 1]] = dr["v"]
            pr = np.fromfile(os.path.join(d, "res.bin.pos"), dtype=np.dtype([("id", "<u8"), ("v", "<f8", 3)]))
            pos_dr = np.empty((n, 3))
            pos_dr[order[pr["id"].astype(np.int64) - 1]] = pr["v"]
            res_extra = {"acc_drift": out_dr[:, :3], "pot_drift": out_dr[:, 3], "oldacc_drift": out_dr[:, 4],
                         "pos_drift": pos_dr}
        for line in r.stdout.decode().splitlines():
            if line.startswith("phorder"):
                info["phorder"] = {k: int(v) for k, v in (p.split("=", 1) for p in line.split()[1:])}
            if line.startswith("drift"):
                kv = dict(p.split("=", 1) for p in line.split()[1:])
                info["drift"] = {k: float(v) for k, v in kv.items()}
            if line.startswith("domain"):
                kv = dict(p.split("=", 1) for p in line.split()[1:])
                info["domain"] = {"corner": [float(x) for x in kv["corner"].split(",")], "len": float(kv["len"])}
            if line.startswith("empty"):
                info["empty_walk_s"] = float(line.split("=", 1)[1])
            if line.startswith("startup") or line.startswith("step"):
                kv = dict(p.split("=", 1) for p in line.split()[1 if line.startswith("startup") else 2:] if "=" in p)
                kv = {k: float(v) for k, v in kv.items()}
                if line.startswith("startup"):
                    info["startup"] = kv
                else:
                    info["steps"].append(kv)
        return {"acc": out[:, :3], "pot": out[:, 3], "oldacc": out[:, 4], "acc_bh": out_bh[:, :3],
                "pot_bh": out_bh[:, 3], "key_hi": keys_hi, "key_lo": keys_lo, "info": info, **res_extra}
    finally:
        if own:
            import shutil
            shutil.rmtree(d, ignore_errors=True)


def ph_block_sample(pos, n_blocks, block_len, seed=1):
    """A sample of targets as GIZMO walks them: `n_blocks` runs of `block_len`
    particles that are consecutive in Peano-Hilbert order (the order of P[]
    after domain_Decomposition, in which the OpenMP walk hands out its active
    particles), one run at a seeded random place in each of n_blocks equal
    stretches of the curve.  Returns sorted particle indices."""
    import oracle
    n = pos.shape[0]
    if n_blocks * block_len >= n:
        return np.arange(n)
    _, lo = oracle.ph_keys(pos, oracle.find_extent(pos), bits=21)
    order = np.argsort(lo, kind="stable")
    rng = np.random.default_rng(seed)
    stretch = n // n_blocks
    starts = np.arange(n_blocks) * stretch + rng.integers(0, max(stretch - block_len, 0) + 1, size=n_blocks)
    return np.sort(np.concatenate([order[a:a + block_len] for a in starts]))


def steps_rate(ic, steps=3, warmup=1, sample=16384, seed=1, tol=0.0025, threads=None, active_n=None,
               rebuild_steps=1, sample_kind=None):
    """The reference's particles/s per steady-state step, from a bounded sample.

    One run of GIZMO's own code with only the sampled targets active: the
    start-up passes (Barnes-Hut, then relative), then `rebuild_steps` steps of
    domain_Decomposition (keys, sort, reorder) + tree build + relative walk,
    then warmup + steps walks of the sample on the resident tree
    (rebuild_steps="all": warmup + steps steps that each rebuild).  `sample` is
    a count (seeded random targets) or an index array.  A step's cost for n_eval
    targets is modelled as the measured rebuild (domain + build) plus the
    measured walk time per sampled target times n_eval.  Returns (model rates
    of the timed steps, info); info["step_s"] holds the timed steps' own
    durations and info["acc"] the sample's start-up relative-pass forces."""
    n = ic["pos"].shape[0]
    cores = threads or os.cpu_count() or 1
    if np.ndim(sample) == 0:
        ns = min(n, int(sample))
        sample = np.sort(np.random.default_rng(seed).choice(n, ns, replace=False))
        sample_kind = sample_kind or "%d seeded random targets" % ns
    sample = np.asarray(sample)
    ns = sample.size
    n_eval = n if active_n is None else int(active_n)   # targets a step evaluates
    fixed = 0.0
    if rebuild_steps == "all":   # every step rebuilds: each timed step is a whole step
        res = run(ic, tol=tol, steps=warmup + steps, sample=sample, threads=cores, sample_only=True)
        rb = res["info"]["steps"][warmup:]
        rebuild_steps = len(rb)
        step_s = [x["t_domain"] + x["t_gravity"] for x in rb]
        per_list = [max(x["t_gravity"] - x["t_build"], 1e-12) / ns for x in rb]
    else:
        rebuild_steps = max(1, int(rebuild_steps))
        res = run(ic, tol=tol, steps=rebuild_steps + warmup + steps, sample=sample, threads=cores, sample_only=True,
                  rebuild_steps=rebuild_steps)
        st = res["info"]["steps"]
        rb = st[:rebuild_steps]
        timed = st[rebuild_steps + warmup:] or [dict(x, t_gravity=x["t_gravity"] - x["t_build"]) for x in rb]
        step_s = [x["t_gravity"] for x in timed]
        # a walk's time = a part paid once per call (loops over every
        # particle, buffers; measured by a call with no target) + a time per
        # target; the per-target part is what scales to n_eval
        fixed = min(res["info"].get("empty_walk_s", 0.0), 0.9 * min(step_s))
        per_list = [max(t - fixed, 1e-12) / ns for t in step_s]
    t_domain = float(np.mean([x["t_domain"] for x in rb]))
    t_build = float(np.mean([x["t_build"] for x in rb]))
    rates = [n_eval / (t_domain + t_build + fixed + per * n_eval) for per in per_list]
    info = {"unit": "particles/s", "cores": cores, "kind": "reference",
            "sample": "GIZMO's own domain_Decomposition + tree build (timed in %d rebuild step(s)) and relative "
                      "gravity walk (compiled reference, FP64, OpenMP %d threads) of %s of %d, walked %d times on "
                      "the resident tree; a step of %d targets is modelled as rebuild + the walk's fixed part + "
                      "walk time per sampled target x %d" % (rebuild_steps, cores, sample_kind or "%d targets" % ns, n, len(step_s),
                                       n_eval, n_eval),
            "t_domain_s": t_domain, "t_build_s": t_build, "t_walk_fixed_s": fixed,
            "t_empty_walk_s": res["info"].get("empty_walk_s"),
            "t_walk_per_particle_us": float(np.mean(per_list)) * 1e6, "step_s": step_s, "sample_n": int(ns),
            "startup": res["info"].get("startup"), "targets": sample, "acc": res["acc"][sample],
            "pot": res["pot"][sample]}
    return rates, info


def rate(ic, seconds=15.0, seed=1, tol=0.0025, threads=None, active_n=None):
    """One bounded measurement of the reference's step rate (about `seconds` of walk)."""
    n = ic["pos"].shape[0]
    probe, pinfo = steps_rate(ic, steps=1, warmup=0, sample=512, seed=seed, tol=tol, threads=threads)
    per = pinfo["t_walk_per_particle_us"] * 1e-6
    ns = int(min(n, max(512, seconds / max(per, 1e-9))))
    rates, info = steps_rate(ic, steps=1, warmup=0, sample=ns, seed=seed + 1, tol=tol, threads=threads,
                             active_n=active_n)
    info["value"] = float(np.mean(rates))
    return info
