"""Seeded synthetic initial conditions for the tree-gravity workloads.

Every generator returns a dict with float64 arrays ``pos`` (N,3), ``vel``
(N,3), ``mass`` (N,), ``h`` (N,) -- the softening kernel radius, i.e. 2.8 times
the Plummer-equivalent softening (GIZMO's ForceSoftening_KernelRadius,
proto.h:134-155 with KERNEL_FAC_FROM_FORCESOFT_TO_PLUMMER = 1/2.8, kernel.h:709)
-- plus a ``meta`` dict recording every constant that was chosen.

Units: G = 1.  Workloads (N, seeds and shapes):
  plummer      isolated Plummer sphere, M = a = 1, radii truncated at 20a,
               isotropic velocities from the distribution function
               (Aarseth, Henon & Wielen 1974 rejection method)
  galaxy       Hernquist halo (M=1, a=1, truncated at 100a) + exponential disk
               (M=0.05, R_d=0.05, sech^2 z_0=0.005); softening 0.01 / 0.005
  clustered    1000 Plummer clumps with log-normal masses (sigma = 1 dex),
               a_k = 0.01 (M_k/<M>)^(1/3), centres uniform in the unit sphere,
               plus a 20% uniform background; equal-mass particles, eps = 1e-4
  ensemble     many independent Plummer or King (W0 = 6) clusters of
               log-uniform size, per-system eps = 0.01 r_half
"""
import math

import numpy as np

KERNEL_FAC = 2.8  # kernel radius / Plummer-equivalent softening (cubic spline)

SEED_PLUMMER = 20261201
SEED_GALAXY = 20261202
SEED_CLUSTERED = 20261203
SEED_ENSEMBLE = 20261204
SEED_SERVING = 20261205


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def _iso_dirs(rng, n):
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)


def _plummer_unit(rng, n, rmax=20.0):
    """Positions/velocities of an M = a = G = 1 Plummer sphere, r <= rmax."""
    r = np.empty(n)
    filled = 0
    while filled < n:
        m = n - filled
        x = rng.uniform(0.0, 1.0, 2 * m + 16)
        x = x[x > 0]
        rr = 1.0 / np.sqrt(x ** (-2.0 / 3.0) - 1.0)
        rr = rr[rr <= rmax][:m]
        r[filled:filled + rr.size] = rr
        filled += rr.size
    pos = _iso_dirs(rng, n) * r[:, None]
    # speed: q = v/v_esc with density g(q) = q^2 (1-q^2)^(7/2), rejection in [0,1]x[0,0.1]
    q = np.empty(n)
    filled = 0
    while filled < n:
        m = n - filled
        qq = rng.uniform(0.0, 1.0, 2 * m + 16)
        yy = rng.uniform(0.0, 0.1, 2 * m + 16)
        ok = qq[yy < qq * qq * (1.0 - qq * qq) ** 3.5][:m]
        q[filled:filled + ok.size] = ok
        filled += ok.size
    vesc = np.sqrt(2.0) * (1.0 + r * r) ** -0.25
    vel = _iso_dirs(rng, n) * (q * vesc)[:, None]
    return pos, vel


def plummer(n=65536, seed=SEED_PLUMMER, eps=0.01, rmax=20.0):
    rng = _rng(seed)
    pos, vel = _plummer_unit(rng, n, rmax)
    mass = np.full(n, 1.0 / n)
    h = np.full(n, KERNEL_FAC * eps)
    return dict(pos=pos, vel=vel, mass=mass, h=h,
                meta=dict(model="plummer", n=n, seed=seed, eps=eps, rmax=rmax, M=1.0, a=1.0))


def _hernquist(rng, n, a=1.0, rmax=100.0):
    mmax = (rmax / (rmax + a)) ** 2
    x = rng.uniform(0.0, mmax, n)
    s = np.sqrt(x)
    r = a * s / (1.0 - s)
    pos = _iso_dirs(rng, n) * r[:, None]
    return pos, r


def galaxy(n_halo=3_000_000, n_disk=1_194_304, seed=SEED_GALAXY, eps_halo=0.01, eps_disk=0.005,
           m_halo=1.0, m_disk=0.05, rd=0.05, z0=0.005):
    from scipy.special import lambertw

    rng = _rng(seed)
    hpos, hr = _hernquist(rng, n_halo)
    # exponential disk: cumulative mass 1-(1+R/Rd)exp(-R/Rd) inverted with Lambert W_{-1}
    u = rng.uniform(0.0, 1.0, n_disk) * (1.0 - 1e-12)
    R = -rd * (np.real(lambertw((u - 1.0) / np.e, -1)) + 1.0)
    phi = rng.uniform(0.0, 2.0 * np.pi, n_disk)
    z = z0 * np.arctanh(2.0 * rng.uniform(0.0, 1.0, n_disk) * (1 - 2e-12) - 1.0 + 1e-12)
    dpos = np.stack([R * np.cos(phi), R * np.sin(phi), z], axis=1)
    # approximate velocities: halo isotropic at the local circular speed, disk circular
    mh_enc = m_halo * (hr / (hr + 1.0)) ** 2 / ((100.0 / 101.0) ** 2)
    vh = np.sqrt(mh_enc / np.maximum(hr, 1e-6))
    hvel = _iso_dirs(rng, n_halo) * (vh / np.sqrt(3.0))[:, None]
    md_enc = m_disk * (1.0 - (1.0 + R / rd) * np.exp(-R / rd))
    mh_R = m_halo * (R / (R + 1.0)) ** 2 / ((100.0 / 101.0) ** 2)
    vc = np.sqrt((md_enc + mh_R) / np.maximum(R, 1e-6))
    dvel = np.stack([-vc * np.sin(phi), vc * np.cos(phi), np.zeros(n_disk)], axis=1)
    pos = np.concatenate([hpos, dpos])
    vel = np.concatenate([hvel, dvel])
    mass = np.concatenate([np.full(n_halo, m_halo / n_halo), np.full(n_disk, m_disk / max(n_disk, 1))])
    h = np.concatenate([np.full(n_halo, KERNEL_FAC * eps_halo), np.full(n_disk, KERNEL_FAC * eps_disk)])
    ratio = (m_disk / n_disk) / (m_halo / n_halo) if n_disk else None
    return dict(pos=pos, vel=vel, mass=mass, h=h,
                meta=dict(model="galaxy", n=n_halo + n_disk, n_halo=n_halo, n_disk=n_disk, seed=seed,
                          eps_halo=eps_halo, eps_disk=eps_disk, halo_rmax=100.0, rd=rd, z0=z0,
                          disk_to_halo_particle_mass=ratio))


def clustered(n=16_777_216, seed=SEED_CLUSTERED, n_clumps=1000, sigma_dex=1.0, f_clumps=0.8, eps=1e-4,
              a_scale=0.01, rmax_clump=20.0):
    rng = _rng(seed)
    lm = rng.normal(0.0, sigma_dex, n_clumps)
    mk = 10.0 ** lm
    mk = mk / mk.sum()
    want = f_clumps * n * mk
    nk = np.floor(want).astype(np.int64)
    short = int(round(f_clumps * n)) - int(nk.sum())
    if short > 0:
        order = np.argsort(-(want - nk))
        nk[order[:short]] += 1
    ak = a_scale * (mk / mk.mean()) ** (1.0 / 3.0)
    # clump centres uniform in the unit sphere
    cr = rng.uniform(0.0, 1.0, n_clumps) ** (1.0 / 3.0)
    centres = _iso_dirs(rng, n_clumps) * cr[:, None]
    parts_p, parts_v = [], []
    for k in range(n_clumps):
        if nk[k] == 0:
            continue
        p, v = _plummer_unit(rng, int(nk[k]), rmax_clump)
        mtot = nk[k] / n
        parts_p.append(centres[k] + p * ak[k])
        parts_v.append(v * math.sqrt(mtot / ak[k]))
    nb = n - int(nk.sum())
    br = rng.uniform(0.0, 1.0, nb) ** (1.0 / 3.0)
    parts_p.append(_iso_dirs(rng, nb) * br[:, None])
    parts_v.append(np.zeros((nb, 3)))
    pos = np.concatenate(parts_p)
    vel = np.concatenate(parts_v)
    mass = np.full(n, 1.0 / n)
    h = np.full(n, KERNEL_FAC * eps)
    return dict(pos=pos, vel=vel, mass=mass, h=h,
                meta=dict(model="clustered", n=n, seed=seed, n_clumps=n_clumps, sigma_dex=sigma_dex,
                          f_clumps=f_clumps, eps=eps, clump_a="0.01*(M_k/<M>)^(1/3)", clump_rmax=rmax_clump,
                          n_background=nb))


def random_active(n, frac, seed):
    """Sorted seeded random subset of size round(frac*n) (individual timesteps)."""
    rng = _rng(seed)
    k = int(round(frac * n))
    return np.sort(rng.choice(n, size=k, replace=False)).astype(np.int32)


# ---------------------------------------------------------------- King models

def _king_profile(W0, npts=4000):
    """Integrate the King (1966) model in King units (r0 = 1): returns r, W(r), M(<r).

    Density of a lowered isothermal sphere as a function of the dimensionless
    potential W: rho(W) ~ exp(W) erf(sqrt W) - sqrt(4W/pi) (1 + 2W/3); Poisson:
    W'' + 2 W'/r = -9 rho(W)/rho(W0).
    """
    from scipy.integrate import solve_ivp
    from scipy.special import erf

    def rho(W):
        W = np.maximum(W, 0.0)
        return np.exp(W) * erf(np.sqrt(W)) - np.sqrt(4.0 * W / np.pi) * (1.0 + 2.0 * W / 3.0)

    rho0 = rho(W0)

    def rhs(r, y):
        W, dW = y
        return [dW, -9.0 * rho(W) / rho0 - 2.0 * dW / r]

    def hit(r, y):
        return y[0]
    hit.terminal = True
    r0 = 1e-6
    y0 = [W0 - 1.5 * r0 * r0, -3.0 * r0]
    sol = solve_ivp(rhs, [r0, 1e3], y0, events=hit, dense_output=True, rtol=1e-9, atol=1e-12, max_step=0.05)
    rt = sol.t_events[0][0] if sol.t_events[0].size else sol.t[-1]
    r = np.linspace(r0, rt, npts)
    W = np.maximum(sol.sol(r)[0], 0.0)
    dens = rho(W) / rho0
    m = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] * r[1:] ** 2 + dens[:-1] * r[:-1] ** 2) * np.diff(r))])
    return r, W, m / m[-1]


_KING_CACHE = {}


def _king_unit(rng, n, W0=6.0):
    """King model positions/velocities scaled to total mass 1 and r_half = 1."""
    if W0 not in _KING_CACHE:
        _KING_CACHE[W0] = _king_profile(W0)
    r_tab, W_tab, m_tab = _KING_CACHE[W0]
    rh = np.interp(0.5, m_tab, r_tab)
    r = np.interp(rng.uniform(0.0, 1.0, n), m_tab, r_tab)
    W = np.interp(r, r_tab, W_tab)
    # speeds from f(E) ~ exp(W - v^2/2) - 1 (sigma = 1), v <= sqrt(2W): rejection
    v = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        vmax = np.sqrt(2.0 * W[todo])
        cand = rng.uniform(0.0, 1.0, todo.size) * vmax
        fmax = np.maximum(np.exp(W[todo]) - 1.0, 1e-300) * vmax * vmax
        f = (np.exp(W[todo] - 0.5 * cand * cand) - 1.0) * cand * cand
        ok = rng.uniform(0.0, 1.0, todo.size) * fmax < f
        v[todo[ok]] = cand[ok]
        todo = todo[~ok]
    pos = _iso_dirs(rng, n) * (r / rh)[:, None]
    vel = _iso_dirs(rng, n) * v[:, None]
    # virial-ish velocity scale for M = 1, r_half = 1 (only used for drifts)
    vel *= 1.0 / max(np.sqrt(np.mean(np.sum(vel ** 2, axis=1))), 1e-12) * np.sqrt(0.4)
    return pos, vel


def ensemble(n_systems=4096, nmin=256, nmax=65536, seed=SEED_ENSEMBLE):
    """Independent clusters: log-uniform sizes, Plummer or King W0=6 by seed."""
    rng = _rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_systems)).astype(np.int64)
    kinds = rng.integers(0, 2, n_systems)   # 0 Plummer, 1 King
    pos_l, vel_l, m_l, h_l = [], [], [], []
    for s in range(n_systems):
        n = int(sizes[s])
        if kinds[s] == 0:
            p, v = _plummer_unit(rng, n, 20.0)
            rhalf = 1.0 / np.sqrt(2.0 ** (2.0 / 3.0) - 1.0)   # Plummer half-mass radius, a = 1
        else:
            p, v = _king_unit(rng, n, 6.0)
            rhalf = 1.0
        pos_l.append(p + 100.0 * s)   # systems are independent; offsets only keep the arrays apart
        vel_l.append(v)
        m_l.append(np.full(n, 1.0 / n))
        h_l.append(np.full(n, KERNEL_FAC * 0.01 * rhalf))
    return dict(pos=np.concatenate(pos_l), vel=np.concatenate(vel_l), mass=np.concatenate(m_l),
                h=np.concatenate(h_l), counts=sizes, kinds=kinds,
                meta=dict(model="ensemble", n_systems=n_systems, nmin=nmin, nmax=nmax, seed=seed,
                          total=int(sizes.sum()), eps="0.01 r_half"))


def serving_system(kind, n, seed):
    """One system of a serving stream: 0 Plummer (eps 0.01), 1 Hernquist halo
    (eps 0.01), 2 clumpy mixture (Plummer clumps plus background, eps 1e-4)."""
    if kind == 0:
        return plummer(n, seed=seed)
    if kind == 1:
        return galaxy(n_halo=n, n_disk=0, seed=seed)
    return clustered(n, seed=seed, n_clumps=int(max(4, min(100, n // 1000))))


def serving_pool(n_systems=64, nmin=1000, nmax=1_000_000, seed=SEED_SERVING):
    """Systems for a serving stream: sizes log-uniform in [nmin, nmax], kinds
    Plummer / Hernquist / clumpy in equal shares, each from its own seed."""
    rng = _rng(seed)
    sizes = np.exp(rng.uniform(np.log(nmin), np.log(nmax), n_systems)).astype(np.int64)
    kinds = rng.integers(0, 3, n_systems)
    pool = []
    for i in range(n_systems):
        s = serving_system(int(kinds[i]), int(sizes[i]), seed + 1 + i)
        s["kind"] = int(kinds[i])
        pool.append(s)
    return pool


def error_stats(acc, acc_ref):
    """Median and 99th percentile of |a - a_ref| / |a_ref| (per target)."""
    acc = np.asarray(acc, dtype=np.float64).reshape(-1, 3)
    ref = np.asarray(acc_ref, dtype=np.float64).reshape(-1, 3)
    e = np.linalg.norm(acc - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
    return float(np.median(e)), float(np.percentile(e, 99)), e
