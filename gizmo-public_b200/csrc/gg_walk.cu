// gg_walk.cu -- warp-cooperative tree walk (force_treeevaluate, forcetree.c:1633-2807).
//
// A warp serves one group of up to 32*TPL targets that are consecutive in
// Peano-Hilbert order (TPL targets per lane).  The warp walks the tree once
// for the whole group with an explicit node stack: each round pops up to 32
// nodes, one per lane, and tests them against the group's bounding box with
// the reference's opening rules made conservative over the group
// (distance = from the node's centre of mass to the box, the smallest
// ErrTolForceAcc*OldAcc of the group, the largest target softening):
//   - massless nodes are skipped                         (forcetree.c:2038)
//   - one-particle nodes are always opened               (:2043-2050)
//   - h < maxsoft and r^2 < maxsoft^2 opens              (:2099-2102)
//   - Barnes-Hut pass: len^2 > r^2 theta^2 opens         (:2104-2111)
//   - relative pass: r^2 < (soft+0.6 len)^2 or
//     r^2 < (maxsoft+0.6 len)^2, m len^2 > r^4 aold, or
//     the target inside the 1.2*len box opens           (:2119-2147)
// For a group of one target these are exactly the reference's tests, run in
// FP64 on the FP64 centre of mass (exact mode).  Larger groups run the same
// tests in FP32 on offsets from the group centre, with the box half-widths
// rounded up; a test within FP32 rounding of its threshold may go either way,
// which is far below the margin the group's conservative box adds.  Used nodes and particles are
// appended (ballot + popc compaction) to per-warp shared-memory lists as
// FP32 offsets from the group centre; a "far" list holds entries that are
// Newtonian for every target of the group (no softening branch, no self
// term) and a "near" list holds the rest.  When a list reaches the flush
// threshold every lane evaluates it for its targets in FP32 (cubic-spline
// softening, kernel.h:452-470, with h = max(h_target, h_source),
// forcetree.c:2263-2283); each flush's partial sums are added to the
// per-target totals with Kahan compensation.  Interactions are counted like
// the reference (forcetree.c:2258, :2488): one per used node or particle with
// r^2 > 0 and m > 0.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define WALK_THREADS 256
#define WALK_WARPS (WALK_THREADS / 32)
#define FULL 0xffffffffu

int gg_walk_threads() { return WALK_THREADS; }

// Per-warp shared memory, in float4 units:
//   far list float4[cap] | near list float4[cap] | near softening float4[cap] |
//   node stack int[WALK_SSTACK] | node slots GGNode[32]
// with cap = flush + 32.  The stack spills to the warp's global stack area
// when it overflows (deep or wide traversals only).
#define WALK_SSTACK 512
__host__ __device__ __forceinline__ int walk_warp_float4s(int flush)
{
    const int cap = flush + 32;
    return 3 * cap + WALK_SSTACK / 4 + 32 * 4;
}

int gg_walk_smem_bytes(int flush, int tpl)
{
    (void)tpl;
    return WALK_WARPS * walk_warp_float4s(flush) * 16;
}

// The next round's node records are staged in shared memory with cp.async, one
// 64-byte slot per lane, so no registers are held while the loads are in
// flight (the walk then fits 3 blocks per SM).  A lane refills its slot only
// after its test of the node in it is complete.
__device__ __forceinline__ void stage_node(int4 *slot, const GGNode *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(slot);
    const int4 *s = reinterpret_cast<const int4 *>(src);
#pragma unroll
    for (int i = 0; i < 4; i++)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d + 16 * i), "l"(s + i) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ GGNode staged_node(const int4 *slot)
{
    asm volatile("cp.async.wait_all;" ::: "memory");
    GGNode r;
    int4 *d = reinterpret_cast<int4 *>(&r);
#pragma unroll
    for (int i = 0; i < 4; i++) d[i] = slot[i];
    return r;
}

__device__ __forceinline__ GGPart load_part(const GGPart *p)
{
    GGPart r;
    const int4 *src = reinterpret_cast<const int4 *>(p);
    int4 *dst = reinterpret_cast<int4 *>(&r);
    dst[0] = __ldg(src);
    dst[1] = __ldg(src + 1);
    return r;
}

struct Kahan {
    float s, c;
    __device__ __forceinline__ void add(float x)
    {
        float y = x - c;
        float t = s + y;
        c = (t - s) - y;
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// This file is compiled with denormals flushed to zero (-ftz=true): rsqrtf and
// the reciprocals are then single hardware approximations without range
// fix-ups.  An entry goes to the far list only when its squared distance from
// the group's box exceeds FAR_MIN_R2, so every far pair has a normal r^2; near
// pairs are selected, not multiplied, out of the sums when r^2 is zero (and
// r^2 below the smallest normal float is zero here).
#define FAR_MIN_R2 1e-36f

// Cubic-spline softened force and potential factors for u = r/h < 1
// (kernel.h:452-470), without a branch or a per-piece coefficient choice.  The
// outer piece (0.5 <= u < 1) equals the inner polynomial plus a correction
// that vanishes below u = 0.5, written in t = max(u - 0.5, 0):
//   w_force = 32/3 + u^2 (32 u - 38.4)  -  256 t^4 (t^2/6 + t/5 + 1/16) / u^3
//   w_pot   = -2.8 + u^2 (16/3 + u^2 (6.4 u - 9.6))  +  t^5 (-6.4 - 128/15 t) / u
// (the force correction is the mass the outer piece of the density removes,
// divided by u^3; the potential correction integrates u times it from 0.5).
// iu = 1/u is passed in (the caller has it from r^-1).  The corrections are
// multiplied out starting from t, so a zero t stays zero however large iu is.
// Returns w_force, writes w_pot; they are still to be scaled by h^-3 and h^-1.
__device__ __forceinline__ float spline_wf(float u, float iu, float *wp)
{
    const float u2 = u * u;
    const float t = fmaxf(u - 0.5f, 0.f);
    const float t2 = t * t, t4 = t2 * t2;
    const float fin = fmaf(u2, fmaf(u, 32.f, -38.4f), 10.666666666667f);
    const float q = t4 * fmaf(t, fmaf(t, 0.166666666667f, 0.2f), 0.0625f);
    const float pin = fmaf(u2, fmaf(u2, fmaf(u, 6.4f, -9.6f), 5.333333333333f), -2.8f);
    *wp = fmaf((t4 * t) * fmaf(t, -8.533333333333f, -6.4f), iu, pin);
    return fmaf(-256.f, ((q * iu) * iu) * iu, fin);
}

template <int TPL>
struct Targets {
    float x[TPL], y[TPL], z[TPL], h[TPL], hinv[TPL];
    bool valid[TPL];
    Kahan ax[TPL], ay[TPL], az[TPL], pot[TPL];
    int nint[TPL];
};

// POT: the potential-only walk (force_treeevaluate_potential, forcetree.c:3169-3474)
template <int TPL, bool POT>
__device__ __forceinline__ void flush_far(const float4 *__restrict__ far, int nf, Targets<TPL> &T)
{
    __syncwarp();
    float px[TPL], py[TPL], pz[TPL], pp[TPL];
#pragma unroll
    for (int s = 0; s < TPL; s++) { px[s] = 0.f; py[s] = 0.f; pz[s] = 0.f; pp[s] = 0.f; }
#pragma unroll 4
    for (int j = 0; j < nf; j++) {
        const float4 e = far[j];
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            float dx = e.x - T.x[s], dy = e.y - T.y[s], dz = e.z - T.z[s];
            float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float rinv = rsqrtf(r2);
            float mr = e.w * rinv;
            if (!POT) {
                float fac = mr * rinv * rinv;
                px[s] = fmaf(dx, fac, px[s]);
                py[s] = fmaf(dy, fac, py[s]);
                pz[s] = fmaf(dz, fac, pz[s]);
            }
            pp[s] -= mr;
        }
    }
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        if (!POT) { T.ax[s].add(px[s]); T.ay[s].add(py[s]); T.az[s].add(pz[s]); }
        T.pot[s].add(pp[s]);
        T.nint[s] += nf;
    }
    __syncwarp();
}

// Near list: entries within the softening of some target of the group.  Most
// of them need the spline for some lanes and the Newtonian form for others
// (both for 85% of entries on the galaxy), so every lane evaluates both
// branch-free and selects; without a branch the loop unrolls over entries and
// independent entries overlap their dependency chains.  r^2 = 0 (the target
// itself, or a coincident particle) contributes nothing and is not counted.
// POT: the potential-only walk, which has no r^2 > 0 condition: an r = 0 pair
// adds m w_pot(0) / h like any other (the caller removes the self term).
// HOMOG: every target of the group has the same kernel radius h_t, so the
// pair's softening h_g = max(h_t, h_source) and its products are per entry,
// formed when the entry was listed: nearH = {h_g, 1/h_g, m/h_g, m/h_g^3}.
// Otherwise nearH = {h_source, 1/h_source} and h_g is formed per pair.
template <int TPL, bool POT, bool HOMOG>
__device__ __forceinline__ void flush_near(const float4 *__restrict__ nearE, const float4 *__restrict__ nearH, int nn,
                                           Targets<TPL> &T)
{
    __syncwarp();
    float px[TPL], py[TPL], pz[TPL], pp[TPL];
    int self[TPL];
#pragma unroll
    for (int s = 0; s < TPL; s++) { px[s] = 0.f; py[s] = 0.f; pz[s] = 0.f; pp[s] = 0.f; self[s] = 0; }
#pragma unroll 2
    for (int j = 0; j < nn; j++) {
        const float4 e = nearE[j];
        const float4 hh = nearH[j];
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            const float dx = e.x - T.x[s], dy = e.y - T.y[s], dz = e.z - T.z[s];
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            const float hg = HOMOG ? hh.x : fmaxf(T.h[s], hh.x);
            const float hinv = HOMOG ? hh.y : fminf(T.hinv[s], hh.y);   // 1/h_g: the inverses are rounded alike
            const float rinv = rsqrtf(POT ? fmaxf(r2, 1e-30f) : r2);   // finite at r = 0 when it counts
            // spline for u = r/h_g < 1 (kernel.h:452-470), Newtonian beyond (:391-398);
            // the two meet at u = 1, where the spline's force factor is 1/u^3
            const float u = r2 * rinv * hinv, iu = hg * rinv;
            float wp;
            const float wf = spline_wf(u, iu, &wp);
            const bool soft = u < 1.f;
            float fpot, fac = 0.f;
            if (HOMOG) {   // Newtonian as m/h_g^3 (1/u)^3 and -m/h_g (1/u), on the entry's products
                fpot = hh.z * (soft ? wp : -iu);
                if (!POT) fac = hh.w * (soft ? wf : iu * iu * iu);
            } else {
                const float mr = e.w * rinv;
                fpot = soft ? e.w * wp * hinv : -mr;
                if (!POT) fac = soft ? e.w * wf * (hinv * hinv * hinv) : mr * rinv * rinv;
            }
            if (POT) {
                pp[s] += fpot;
            } else {
                const bool use = r2 > 0.f;
                fac = use ? fac : 0.f;
                fpot = use ? fpot : 0.f;
                self[s] += use ? 0 : 1;
                px[s] = fmaf(dx, fac, px[s]);
                py[s] = fmaf(dy, fac, py[s]);
                pz[s] = fmaf(dz, fac, pz[s]);
                pp[s] += fpot;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        if (!POT) { T.ax[s].add(px[s]); T.ay[s].add(py[s]); T.az[s].add(pz[s]); }
        T.pot[s].add(pp[s]);
        T.nint[s] += nn - self[s];
    }
    __syncwarp();
}

template <int TPL, bool POT>
__device__ __forceinline__ void flush_near_sel(bool homog, const float4 *__restrict__ nearE,
                                               const float4 *__restrict__ nearH, int nn, Targets<TPL> &T)
{
    if (homog) flush_near<TPL, POT, true>(nearE, nearH, nn, T);
    else flush_near<TPL, POT, false>(nearE, nearH, nn, T);
}

// softening record of a near-list entry with kernel radius hsrc and mass m (see flush_near)
__device__ __forceinline__ float4 near_soft(float hsrc, float m, bool homog, float hgroup)
{
    if (homog) {
        const float hg = fmaxf(hgroup, hsrc);
        const float hinv = hg > 0.f ? __frcp_rn(hg) : INFINITY;
        return make_float4(hg, hinv, m * hinv, m * (hinv * hinv * hinv));
    }
    return make_float4(hsrc, hsrc > 0.f ? __frcp_rn(hsrc) : INFINITY, 0.f, 0.f);
}

__device__ __forceinline__ double warp_min_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
__device__ __forceinline__ double warp_max_d(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
    return v;
}
__device__ __forceinline__ int warp_incl_scan(int v, int lane)
{
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(FULL, v, o);
        if (lane >= o) v += y;
    }
    return v;
}

// MINB: resident blocks per SM the register allocation must allow (1..3): a
// tuning knob trading registers (spills) against warps in flight.
// F64T: opening tests in FP64 (used for one-target groups, where the tests are
// exactly the reference's); otherwise the tests run in FP32 on FP64-formed
// offsets from the group centre, against a bounding box rounded outwards.
template <int TPL, int MINB, bool F64T, bool POT>
__global__ void __launch_bounds__(WALK_THREADS, MINB) k_walk(WalkParams p)
{
    extern __shared__ float4 walk_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int FL = p.flush, cap = FL + 32;
    float4 *far = walk_smem + (size_t)warp * walk_warp_float4s(FL);
    float4 *nearE = far + cap;
    float4 *nearH = nearE + cap;
    int *sstack = reinterpret_cast<int *>(far + 3 * cap);
    int4 *nslot = reinterpret_cast<int4 *>(far + 3 * cap + WALK_SSTACK / 4) + 4 * lane;
    int *gstack = p.stack + (size_t)(blockIdx.x * WALK_WARPS + warp) * p.stack_cap;
    const int ngroups = *p.ngroups;
    const double theta = p.theta;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(p.group_counter, 1);
        g = __shfl_sync(FULL, g, 0);
        if (g >= ngroups) break;
        const GGGroup grp = p.groups[p.gorder ? (int)p.gorder[g] : g];
        const long long t_start = clock64();

        // ---- targets of the group
        Targets<TPL> T;
        double tx[TPL], ty[TPL], tz[TPL];
        int tpi[TPL];
        double bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
        double aold_min = INFINITY;
        float hmin = INFINITY, hmax = 0.f;
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            int k = s * 32 + lane;
            bool v = k < grp.count;
            T.valid[s] = v;
            T.nint[s] = 0;
            T.ax[s] = {0.f, 0.f}; T.ay[s] = {0.f, 0.f}; T.az[s] = {0.f, 0.f}; T.pot[s] = {0.f, 0.f};
            tpi[s] = -1;
            tx[s] = ty[s] = tz[s] = 0.0;
            T.h[s] = 0.f;
            T.hinv[s] = INFINITY;
            if (v) {
                int t = grp.first + k;
                int pi = p.tlist ? p.tlist[t] : t;
                tpi[s] = pi;
                GGPart q = load_part(p.parts + pi);
                tx[s] = q.x; ty[s] = q.y; tz[s] = q.z;
                T.h[s] = q.h;
                T.hinv[s] = q.h > 0.f ? __frcp_rn(q.h) : INFINITY;
                double oa = p.oldacc_in ? p.oldacc_in[p.perm[pi]] : 0.0;
                aold_min = fmin(aold_min, p.tol * oa);
                hmin = fminf(hmin, q.h);
                hmax = fmaxf(hmax, q.h);
                bmin[0] = fmin(bmin[0], q.x); bmax[0] = fmax(bmax[0], q.x);
                bmin[1] = fmin(bmin[1], q.y); bmax[1] = fmax(bmax[1], q.y);
                bmin[2] = fmin(bmin[2], q.z); bmax[2] = fmax(bmax[2], q.z);
            }
        }
        double cg[3], hw[3];
#pragma unroll
        for (int q = 0; q < 3; q++) {
            bmin[q] = warp_min_d(bmin[q]);
            bmax[q] = warp_max_d(bmax[q]);
            cg[q] = 0.5 * (bmin[q] + bmax[q]);
            hw[q] = fmax(0.5 * (bmax[q] - bmin[q]), fmax(bmax[q] - cg[q], cg[q] - bmin[q]));
        }
        aold_min = warp_min_d(aold_min);
        hmin = (float)warp_min_d((double)hmin);
        hmax = (float)warp_max_d((double)hmax);
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            T.x[s] = (float)(tx[s] - cg[0]);
            T.y[s] = (float)(ty[s] - cg[1]);
            T.z[s] = (float)(tz[s] - cg[2]);
        }
        const double hmaxd = (double)hmax, hmind = (double)hmin;
        const float hwf[3] = {__double2float_ru(hw[0]), __double2float_ru(hw[1]), __double2float_ru(hw[2])};
        const float aoldf = (float)aold_min, thetaf = (float)theta;
        const bool homog = hmin == hmax;   // one kernel radius in the group (warp-uniform)

        // ---- traversal
        // The node stack lives in shared memory (sp entries) on top of a spill
        // area in global memory (gsp entries).  Each round pops up to 32 nodes;
        // the next round's node records are staged (cp.async) before this
        // round's leaf particles and list flushes are processed, which hides
        // their latency.
        int sp = 1, gsp = 0, nf = 0, nn = 0;
        int list_far = 0, list_near = 0, tested = 0;   // warp-uniform statistics of this group
        bool overflow = false;
        if (lane == 0) sstack[0] = grp.root;
        __syncwarp();
        // pop up to 32 nodes (one per lane); returns the count (warp-uniform)
        auto pop_nodes = [&](int &node) -> int {
            if (sp == 0 && gsp > 0) {   // refill from the spill area, keeping stack order
                const int m = min(gsp, WALK_SSTACK / 2);
                for (int i = lane; i < m; i += 32) sstack[i] = gstack[gsp - m + i];
                gsp -= m;
                sp = m;
                __syncwarp();
            }
            const int k = min(sp, 32);
            node = -1;
            if (lane < k) node = sstack[sp - k + lane];
            sp -= k;
            __syncwarp();
            return k;
        };
        int node = -1;
        int k = pop_nodes(node);
        if (lane < k) stage_node(nslot, p.nodes + node);
        while (k > 0) {
            tested += k;

            int act = 0, na = 0, nb = 0;
            bool isfar = false;
            float4 ent = make_float4(0.f, 0.f, 0.f, 0.f);
            float hp = 0.f;
            if (lane < k) {
                const GGNode nd = staged_node(nslot);
                na = nd.a;
                nb = nd.b;
                if (nd.mass > 0.f) {
                    if (nb == -1) {
                        act = 3;
                    } else if (!F64T) {
                        const float dx = (float)(nd.cx - cg[0]), dy = (float)(nd.cy - cg[1]), dz = (float)(nd.cz - cg[2]);
                        const float ex = fmaxf(fabsf(dx) - hwf[0], 0.f), ey = fmaxf(fabsf(dy) - hwf[1], 0.f),
                                    ez = fmaxf(fabsf(dz) - hwf[2], 0.f);
                        const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                        const float ms = nd.maxsoft, L = nd.len;
                        bool open = (hmin < ms) && (r2 < ms * ms);
                        if (!open) {
                            if (thetaf > 0.f) {
                                open = L * L > r2 * thetaf * thetaf;
                            } else {
                                const float a1 = fmaf(0.6f, L, hmax), a2 = fmaf(0.6f, L, ms);
                                open = (r2 < a1 * a1) || (r2 < a2 * a2) || (nd.mass * L * L > r2 * r2 * aoldf);
                                if (!open)
                                    open = (fabsf(dx + nd.gx) < fmaf(0.6f, L, hwf[0])) &&
                                           (fabsf(dy + nd.gy) < fmaf(0.6f, L, hwf[1])) &&
                                           (fabsf(dz + nd.gz) < fmaf(0.6f, L, hwf[2]));
                            }
                        }
                        if (open) {
                            act = (nb > 0) ? 2 : 3;
                        } else {
                            act = 1;
                            ent = make_float4(dx, dy, dz, nd.mass);
                            hp = ms;
                            const float hh = fmaxf(hmax, ms);
                            isfar = (r2 >= hh * hh) && (r2 > FAR_MIN_R2);
                        }
                    } else {
                        double dx = nd.cx - cg[0], dy = nd.cy - cg[1], dz = nd.cz - cg[2];
                        double ex = fmax(fabs(dx) - hw[0], 0.0), ey = fmax(fabs(dy) - hw[1], 0.0),
                               ez = fmax(fabs(dz) - hw[2], 0.0);
                        double r2 = ex * ex + ey * ey + ez * ez;
                        double ms = (double)nd.maxsoft, L = (double)nd.len;
                        bool open = (hmind < ms) && (r2 < ms * ms);
                        if (!open) {
                            if (theta > 0.0) {
                                open = L * L > r2 * theta * theta;
                            } else {
                                double a1 = hmaxd + 0.6 * L, a2 = ms + 0.6 * L;
                                open = (r2 < a1 * a1) || (r2 < a2 * a2) || ((double)nd.mass * L * L > r2 * r2 * aold_min);
                                if (!open) {
                                    double gx = fabs(dx + (double)nd.gx), gy = fabs(dy + (double)nd.gy),
                                           gz = fabs(dz + (double)nd.gz);
                                    open = (gx < 0.6 * L + hw[0]) && (gy < 0.6 * L + hw[1]) && (gz < 0.6 * L + hw[2]);
                                }
                            }
                        }
                        if (open) {
                            act = (nb > 0) ? 2 : 3;
                        } else {
                            act = 1;
                            ent = make_float4((float)dx, (float)dy, (float)dz, nd.mass);
                            hp = nd.maxsoft;
                            double hh = fmax(hmaxd, ms);
                            isfar = (r2 >= hh * hh) && (r2 > (double)FAR_MIN_R2);
                        }
                    }
                }
            }
            // used nodes -> lists
            {
                unsigned mf = __ballot_sync(FULL, act == 1 && isfar);
                unsigned mn = __ballot_sync(FULL, act == 1 && !isfar);
                if (act == 1) {
                    if (isfar) far[nf + __popc(mf & lt_mask)] = ent;
                    else {
                        int pos = nn + __popc(mn & lt_mask);
                        nearE[pos] = ent;
                        nearH[pos] = near_soft(hp, ent.w, homog, hmax);
                    }
                }
                nf += __popc(mf);
                nn += __popc(mn);
                list_far += __popc(mf);
                list_near += __popc(mn);
            }
            // opened internal nodes -> children on the stack (spilling its
            // bottom half to global memory when it would overflow)
            {
                int nch = (act == 2) ? nb : 0;
                int incl = warp_incl_scan(nch, lane);
                int total = __shfl_sync(FULL, incl, 31);
                if (sp + total > WALK_SSTACK) {
                    const int m = WALK_SSTACK / 2;
                    if (gsp + m > p.stack_cap) {
                        overflow = true;
                        break;
                    }
                    for (int i = lane; i < m; i += 32) gstack[gsp + i] = sstack[i];
                    __syncwarp();
                    for (int i = lane; i < sp - m; i += 32) sstack[i] = sstack[m + i];   // sp - m <= m: no overlap
                    __syncwarp();
                    gsp += m;
                    sp -= m;
                }
                int o = sp + incl - nch;
                for (int c = 0; c < nch; c++) sstack[o + c] = na + c;
                sp += total;
                __syncwarp();
            }
            // next round's node records are staged now; the copies complete behind
            // this round's flushes and leaf particles
            int next_node = -1;
            const int next_k = pop_nodes(next_node);
            if (lane < next_k) stage_node(nslot, p.nodes + next_node);
            if (nf >= FL) { flush_far<TPL, POT>(far, nf, T); nf = 0; }
            if (nn >= FL) { flush_near_sel<TPL, POT>(homog, nearE, nearH, nn, T); nn = 0; }
            // opened leaves -> particles, 32 at a time
            {
                int cnt = (act == 3) ? -nb : 0;
                int incl = warp_incl_scan(cnt, lane);
                int P = __shfl_sync(FULL, incl, 31);
                int excl = incl - cnt;
                for (int pb = 0; pb < P; pb += 32) {
                    int q = pb + lane;
                    int src = 0;
#pragma unroll
                    for (int step = 16; step > 0; step >>= 1) {
                        int v = __shfl_sync(FULL, incl, src + step - 1);
                        if (v <= q) src += step;
                    }
                    src = min(src, 31);
                    int a_src = __shfl_sync(FULL, na, src);
                    int e_src = __shfl_sync(FULL, excl, src);
                    bool use = false, pfar = false;
                    float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
                    float ph = 0.f;
                    if (q < P) {
                        int pi = a_src + (q - e_src);
                        GGPart pp = load_part(p.parts + pi);
                        if (pp.m > 0.f) {
                            const float dx = (float)(pp.x - cg[0]), dy = (float)(pp.y - cg[1]), dz = (float)(pp.z - cg[2]);
                            const float ex = fmaxf(fabsf(dx) - hwf[0], 0.f), ey = fmaxf(fabsf(dy) - hwf[1], 0.f),
                                        ez = fmaxf(fabsf(dz) - hwf[2], 0.f);
                            const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                            const float hh = fmaxf(hmax, pp.h);
                            pe = make_float4(dx, dy, dz, pp.m);
                            ph = pp.h;
                            use = true;
                            pfar = (r2 >= hh * hh) && (r2 > FAR_MIN_R2);
                        }
                    }
                    unsigned mf = __ballot_sync(FULL, use && pfar);
                    unsigned mn = __ballot_sync(FULL, use && !pfar);
                    if (use) {
                        if (pfar) far[nf + __popc(mf & lt_mask)] = pe;
                        else {
                            int pos = nn + __popc(mn & lt_mask);
                            nearE[pos] = pe;
                            nearH[pos] = near_soft(ph, pe.w, homog, hmax);
                        }
                    }
                    nf += __popc(mf);
                    nn += __popc(mn);
                    list_far += __popc(mf);
                    list_near += __popc(mn);
                    if (nf >= FL) { flush_far<TPL, POT>(far, nf, T); nf = 0; }
                    if (nn >= FL) { flush_near_sel<TPL, POT>(homog, nearE, nearH, nn, T); nn = 0; }
                }
            }
            k = next_k;
            node = next_node;
        }
        if (overflow) {
            if (lane == 0) atomicOr(p.err, GG_EBIT_STACK_OVERFLOW);
            continue;
        }
        if (nf > 0) flush_far<TPL, POT>(far, nf, T);
        if (nn > 0) flush_near_sel<TPL, POT>(homog, nearE, nearH, nn, T);

        // ---- results
        // this group's device cycles per target: the cost the next walk orders its groups by
        const float tcost = (float)(clock64() - t_start) / (float)grp.count;
        int mycount = 0;
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            if (!T.valid[s]) continue;
            int t = grp.first + s * 32 + lane;
            int pi = tpi[s];
            unsigned li = p.perm[pi];
            int o = p.tout ? p.tout[t] : (int)li;
            if (POT) {
                // compute_potential removes the self term m_i kernel(0) / h_i
                // (potential.c:137-145); subtract the FP32 value the walk added
                const float mi = p.parts[pi].m;
                p.pot[o] = T.pot[s].value() - (double)((mi * -2.8f) * T.hinv[s]);
            } else {
                double ax = T.ax[s].value(), ay = T.ay[s].value(), az = T.az[s].value();
                p.acc[3 * (size_t)o] = ax;
                p.acc[3 * (size_t)o + 1] = ay;
                p.acc[3 * (size_t)o + 2] = az;
                if (p.pot) p.pot[o] = T.pot[s].value();
                if (p.oldacc_out) p.oldacc_out[li] = sqrt(ax * ax + ay * ay + az * az);
            }
            if (p.ninter) p.ninter[o] = T.nint[s];
            if (p.cost_out) p.cost_out[li] = tcost;
            mycount += T.nint[s];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mycount += __shfl_xor_sync(FULL, mycount, o);
        if (lane == 0) {
            atomicAdd(p.interactions, (unsigned long long)mycount);
            atomicAdd(p.interactions + 1, (unsigned long long)list_far);
            atomicAdd(p.interactions + 2, (unsigned long long)list_near);
            atomicAdd(p.interactions + 3, (unsigned long long)tested);
        }
    }
}

template <int TPL, int MINB, bool F64T, bool POT = false>
static void launch_walk_t(const WalkParams &p, int blocks, int smem, cudaStream_t st)
{
    cudaFuncSetAttribute(k_walk<TPL, MINB, F64T, POT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_walk<TPL, MINB, F64T, POT><<<blocks, WALK_THREADS, smem, st>>>(p);
}

// blocks_per_sm selects the register budget of the instantiation (1..3) and
// the persistent grid is that many blocks per SM
void gg_launch_walk(const WalkParams &p, int tpl, int blocks_per_sm, cudaStream_t st)
{
    int smem = gg_walk_smem_bytes(p.flush, tpl);
    int minb = blocks_per_sm < 1 ? 1 : (blocks_per_sm > 3 ? 3 : blocks_per_sm);
    int blocks = gg_num_sms() * blocks_per_sm;
    if (p.pot_only) {   // the potential-only walk: one register budget per mode
        if (p.group_size == 1) launch_walk_t<1, 2, true, true>(p, blocks, smem, st);
        else if (tpl == 2) launch_walk_t<2, 2, false, true>(p, blocks, smem, st);
        else launch_walk_t<1, 2, false, true>(p, blocks, smem, st);
    } else if (p.group_size == 1) {
        launch_walk_t<1, 2, true>(p, blocks, smem, st);   // exact mode: the reference's tests
    } else if (tpl == 2) {
        if (minb == 1) launch_walk_t<2, 1, false>(p, blocks, smem, st);
        else if (minb == 2) launch_walk_t<2, 2, false>(p, blocks, smem, st);
        else launch_walk_t<2, 3, false>(p, blocks, smem, st);
    } else {
        if (minb == 1) launch_walk_t<1, 1, false>(p, blocks, smem, st);
        else if (minb == 2) launch_walk_t<1, 2, false>(p, blocks, smem, st);
        else launch_walk_t<1, 3, false>(p, blocks, smem, st);
    }
    gg_note_launches(1);
}
