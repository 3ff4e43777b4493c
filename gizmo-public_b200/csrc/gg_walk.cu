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
//
// How the work is arranged on the SM (each part is described where it is):
//   - the next round's node records are staged in shared memory while this
//     round's leaves and flushes run (per-lane cp.async, or bulk copies of
//     runs of consecutive records on an mbarrier);
//   - stack pushes use prefix counts from bit ballots; the particles of opened
//     leaves go through a per-warp queue and are classified 32 at a time;
//   - the lists are pair-interleaved and evaluated two entries per packed
//     FP32x2 instruction;
//   - the persistent warps take groups in the order the host side planned
//     (most expensive first, from the previous walk's measured cost), and each
//     group records its own cost for the next walk.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define WALK_THREADS 256
#define WALK_WARPS (WALK_THREADS / 32)
#define FULL 0xffffffffu

int gg_walk_threads() { return WALK_THREADS; }

// Per-warp shared memory, in float4 units:
//   far list float4[cap] | near list float4[cap] | near softening float4[cap] |
//   node stack int[WALK_SSTACK] | node slots GGNode[32] | particle queue int[PQ_CAP] |
//   mbarrier of the node copies (16 bytes)
// with cap = list_cap(flush) entries of 4 floats.  The stack spills to the warp's global stack area
// when it overflows (deep or wide traversals only).
#define WALK_SSTACK 512
// particle queue: indices of the particles of opened leaves, evaluated 32 at a time
#define PQ_CAP 224
// list capacity in entries: a flush threshold plus one ballot's worth, even
// (the lists are stored in pairs)
__host__ __device__ __forceinline__ int list_cap(int flush) { return (flush + 33) & ~1; }
__host__ __device__ __forceinline__ int walk_warp_float4s(int flush)
{
    const int cap = list_cap(flush);
    return 3 * cap + WALK_SSTACK / 4 + 32 * 4 + PQ_CAP / 4 + 1;
}

int gg_walk_smem_bytes(int flush, int tpl)
{
    (void)tpl;
    return WALK_WARPS * walk_warp_float4s(flush) * 16;
}

// ---- staging of node records
// The next round's node records are copied into shared memory, one 64-byte slot
// per lane, while this round's leaves and flushes are processed; no registers
// are held while the copies are in flight.  A lane's slot is refilled only
// after its test of the node in it is complete.  Two ways (gg_config
// .node_staging), measured close to each other:
//  0: each lane copies its own record with cp.async (16-byte pieces through
//     L1, where the top levels of the tree, which every group visits, hit);
//  1: the bulk-copy (TMA) engine, one copy per run of consecutive records.
// (Staging two rounds ahead, in two slots, measured no faster.)
__device__ __forceinline__ void stage_node(int4 *slot, const GGNode *src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(slot);
    const int4 *s = reinterpret_cast<const int4 *>(src);
#pragma unroll
    for (int i = 0; i < 4; i++)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d + 16 * i), "l"(s + i) : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Bulk copies: the nodes a round pops sit in
// consecutive lanes, and the children of one node are consecutive records, so
// they form a few runs of consecutive records: the first lane of each run
// issues one cp.async.bulk for the whole run.  The copies complete on the
// warp's mbarrier, which lane 0 arms with the round's byte count; the test
// waits on the barrier's phase.  Every wait is bounded: after WALK_WAIT_LIMIT
// polls the warp records GG_EBIT_WALK_TIMEOUT, waits once more (bounded) for
// its copies and leaves the kernel.
#define WALK_WAIT_LIMIT (1 << 20)

__device__ __forceinline__ void stage_nodes(unsigned bar, unsigned slot0, const GGNode *nodes, int node, int k,
                                            int lane)
{
    const int prev = __shfl_up_sync(FULL, node, 1);
    const bool start = lane < k && (lane == 0 || node != prev + 1);
    const unsigned starts = __ballot_sync(FULL, start);
    // the slots were read by this round's tests, whose values were consumed
    // before the pop above (warp-synchronous): the copies may overwrite them
    if (lane == 0)
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(k * 64) : "memory");
    __syncwarp();
    if (start) {
        const unsigned later = starts & ~((2u << lane) - 1u);   // run starts after this lane
        const int end = later ? __ffs(later) - 1 : k;
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(slot0 + 64u * lane), "l"(nodes + node), "r"(64u * (end - lane)), "r"(bar)
                     : "memory");
    }
}

// true once the phase of the given parity has completed; false if the bounded
// wait gave up
__device__ __forceinline__ bool bar_wait(unsigned bar, unsigned parity)
{
    for (int i = 0; i < WALK_WAIT_LIMIT; i++) {
        unsigned done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(bar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
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

// ---- packed FP32x2 arithmetic (sm_100): one instruction, two IEEE FP32
// operations with round-to-nearest, each exactly the scalar operation
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 sel2(bool px, bool py, float2 a, float2 b)
{
    return make_float2(px ? a.x : b.x, py ? a.y : b.y);
}

// Interaction lists are stored pair-interleaved: entries 2p and 2p+1 occupy
// the eight floats {x0, x1, y0, y1, z0, z1, w0, w1} (w: mass), so that one
// 128-bit shared-memory load gives the register pairs the packed instructions
// take.  The softening records of the near list use the same layout.
__device__ __forceinline__ void list_put(float *list, int j, float4 v)
{
    float *b = list + ((j >> 1) << 3) + (j & 1);
    b[0] = v.x;
    b[2] = v.y;
    b[4] = v.z;
    b[6] = v.w;
}
// A list of odd length is evaluated with one more entry: massless and 1e18 away
// (its r^2 is finite and its terms are exactly zero).  The lists have room.
#define PAD_ENTRY make_float4(1e18f, 1e18f, 1e18f, 0.f)

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
// Two pairs at a time, in packed FP32x2.
__device__ __forceinline__ float2 spline_wf2(float2 u, float2 iu, float2 *wp)
{
    const float2 u2 = mul2(u, u);
    const float2 um = add2(u, dup2(-0.5f));
    const float2 t = make_float2(fmaxf(um.x, 0.f), fmaxf(um.y, 0.f));
    const float2 t2 = mul2(t, t), t4 = mul2(t2, t2);
    const float2 fin = fma2(u2, fma2(u, dup2(32.f), dup2(-38.4f)), dup2(10.666666666667f));
    const float2 q = mul2(t4, fma2(t, fma2(t, dup2(0.166666666667f), dup2(0.2f)), dup2(0.0625f)));
    const float2 pin = fma2(u2, fma2(u2, fma2(u, dup2(6.4f), dup2(-9.6f)), dup2(5.333333333333f)), dup2(-2.8f));
    *wp = fma2(mul2(mul2(t4, t), fma2(t, dup2(-8.533333333333f), dup2(-6.4f))), iu, pin);
    return fma2(dup2(-256.f), mul2(mul2(mul2(q, iu), iu), iu), fin);
}

template <int TPL>
struct Targets {
    float x[TPL], y[TPL], z[TPL], h[TPL], hinv[TPL];
    bool valid[TPL];
    Kahan ax[TPL], ay[TPL], az[TPL], pot[TPL];
    int nint[TPL];
};

// Far list: Newtonian for every target of the group, two entries per packed
// instruction.  Each flush keeps one partial sum per entry parity and adds
// both into the Kahan totals.
// POT: the potential-only walk (force_treeevaluate_potential, forcetree.c:3169-3474)
template <int TPL, bool POT>
__device__ __forceinline__ void flush_far(float *__restrict__ far, int nf, Targets<TPL> &T)
{
    if ((nf & 1) && (threadIdx.x & 31) == 0) list_put(far, nf, PAD_ENTRY);
    __syncwarp();
    const float4 *L = reinterpret_cast<const float4 *>(far);
    float2 px[TPL], py[TPL], pz[TPL], pp[TPL], nx[TPL], ny[TPL], nz[TPL];
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        px[s] = py[s] = pz[s] = pp[s] = dup2(0.f);
        nx[s] = dup2(-T.x[s]); ny[s] = dup2(-T.y[s]); nz[s] = dup2(-T.z[s]);
    }
    const int np = (nf + 1) >> 1;
#pragma unroll 2
    for (int q = 0; q < np; q++) {
        const float4 A = L[2 * q], B = L[2 * q + 1];
        const float2 ex = make_float2(A.x, A.y), ey = make_float2(A.z, A.w);
        const float2 ez = make_float2(B.x, B.y), em = make_float2(B.z, B.w);
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            const float2 dx = add2(ex, nx[s]), dy = add2(ey, ny[s]), dz = add2(ez, nz[s]);
            const float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
            const float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
            const float2 mr = mul2(em, rinv);
            if (!POT) {
                const float2 fac = mul2(mul2(mr, rinv), rinv);
                px[s] = fma2(dx, fac, px[s]);
                py[s] = fma2(dy, fac, py[s]);
                pz[s] = fma2(dz, fac, pz[s]);
            }
            pp[s] = fma2(mr, dup2(-1.f), pp[s]);
        }
    }
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        if (!POT) {
            T.ax[s].add(px[s].x + px[s].y);
            T.ay[s].add(py[s].x + py[s].y);
            T.az[s].add(pz[s].x + pz[s].y);
        }
        T.pot[s].add(pp[s].x + pp[s].y);
        T.nint[s] += nf;
    }
    __syncwarp();
}

// Near list: entries within the softening of some target of the group.  Most
// of them need the spline for some lanes and the Newtonian form for others
// (both for 85% of entries on the galaxy), so every lane evaluates both
// branch-free and selects, two entries per packed instruction.  r^2 = 0 (the
// target itself, or a coincident particle) contributes nothing and is not
// counted.
// POT: the potential-only walk, which has no r^2 > 0 condition: an r = 0 pair
// adds m w_pot(0) / h like any other (the caller removes the self term).
// HOMOG: every target of the group has the same kernel radius h_t, so the
// pair's softening h_g = max(h_t, h_source) and its products are per entry,
// formed when the entry was listed: nearH = {h_g, 1/h_g, m/h_g, m/h_g^3}.
// Otherwise nearH = {h_source, 1/h_source} and h_g is formed per pair.
template <int TPL, bool POT, bool HOMOG>
__device__ __forceinline__ void flush_near(float *__restrict__ nearE, float *__restrict__ nearH, int nn,
                                           Targets<TPL> &T)
{
    if ((nn & 1) && (threadIdx.x & 31) == 0) {
        list_put(nearE, nn, PAD_ENTRY);
        list_put(nearH, nn, make_float4(1.f, 1.f, 0.f, 0.f));
    }
    __syncwarp();
    const float4 *LE = reinterpret_cast<const float4 *>(nearE);
    const float4 *LH = reinterpret_cast<const float4 *>(nearH);
    float2 px[TPL], py[TPL], pz[TPL], pp[TPL], nx[TPL], ny[TPL], nz[TPL];
    int self[TPL];
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        px[s] = py[s] = pz[s] = pp[s] = dup2(0.f);
        nx[s] = dup2(-T.x[s]); ny[s] = dup2(-T.y[s]); nz[s] = dup2(-T.z[s]);
        self[s] = 0;
    }
    const int np = (nn + 1) >> 1;
#pragma unroll 2
    for (int q = 0; q < np; q++) {
        const float4 A = LE[2 * q], B = LE[2 * q + 1], C = LH[2 * q], D = LH[2 * q + 1];
        const float2 ex = make_float2(A.x, A.y), ey = make_float2(A.z, A.w);
        const float2 ez = make_float2(B.x, B.y), em = make_float2(B.z, B.w);
        const float2 hs = make_float2(C.x, C.y), hsinv = make_float2(C.z, C.w);
        const float2 mh = make_float2(D.x, D.y), mh3 = make_float2(D.z, D.w);
#pragma unroll
        for (int s = 0; s < TPL; s++) {
            const float2 dx = add2(ex, nx[s]), dy = add2(ey, ny[s]), dz = add2(ez, nz[s]);
            const float2 r2 = fma2(dx, dx, fma2(dy, dy, mul2(dz, dz)));
            const float2 hg = HOMOG ? hs : make_float2(fmaxf(T.h[s], hs.x), fmaxf(T.h[s], hs.y));
            // 1/h_g: the inverses are rounded alike
            const float2 hinv = HOMOG ? hsinv : make_float2(fminf(T.hinv[s], hsinv.x), fminf(T.hinv[s], hsinv.y));
            // finite at r = 0 when it counts
            const float2 rinv = make_float2(rsqrtf(POT ? fmaxf(r2.x, 1e-30f) : r2.x),
                                            rsqrtf(POT ? fmaxf(r2.y, 1e-30f) : r2.y));
            // spline for u = r/h_g < 1 (kernel.h:452-470), Newtonian beyond (:391-398);
            // the two meet at u = 1, where the spline's force factor is 1/u^3
            const float2 u = mul2(mul2(r2, rinv), hinv), iu = mul2(hg, rinv);
            float2 wp;
            const float2 wf = spline_wf2(u, iu, &wp);
            const bool sx = u.x < 1.f, sy = u.y < 1.f;
            float2 fpot, fac = dup2(0.f);
            if (HOMOG) {   // Newtonian as m/h_g^3 (1/u)^3 and -m/h_g (1/u), on the entry's products
                fpot = mul2(mh, sel2(sx, sy, wp, make_float2(-iu.x, -iu.y)));
                if (!POT) fac = mul2(mh3, sel2(sx, sy, wf, mul2(mul2(iu, iu), iu)));
            } else {
                const float2 mr = mul2(em, rinv);
                fpot = sel2(sx, sy, mul2(mul2(em, wp), hinv), make_float2(-mr.x, -mr.y));
                if (!POT)
                    fac = sel2(sx, sy, mul2(mul2(em, wf), mul2(mul2(hinv, hinv), hinv)), mul2(mul2(mr, rinv), rinv));
            }
            if (POT) {
                pp[s] = add2(pp[s], fpot);
            } else {
                const bool ux = r2.x > 0.f, uy = r2.y > 0.f;
                fac = sel2(ux, uy, fac, dup2(0.f));
                fpot = sel2(ux, uy, fpot, dup2(0.f));
                self[s] += (ux ? 0 : 1) + (uy ? 0 : 1);
                px[s] = fma2(dx, fac, px[s]);
                py[s] = fma2(dy, fac, py[s]);
                pz[s] = fma2(dz, fac, pz[s]);
                pp[s] = add2(pp[s], fpot);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < TPL; s++) {
        if (!POT) {
            T.ax[s].add(px[s].x + px[s].y);
            T.ay[s].add(py[s].x + py[s].y);
            T.az[s].add(pz[s].x + pz[s].y);
        }
        T.pot[s].add(pp[s].x + pp[s].y);
        T.nint[s] += nn - self[s];
    }
    __syncwarp();
}

template <int TPL, bool POT>
__device__ __forceinline__ void flush_near_sel(bool homog, float *__restrict__ nearE, float *__restrict__ nearH,
                                               int nn, Targets<TPL> &T)
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
// exclusive prefix sum over the warp of v in [0, 2^BITS) from one ballot per
// bit, and the total from one reduction: the votes are independent, so the
// latency is that of one vote, not of a chain of shuffles
template <int BITS>
__device__ __forceinline__ int warp_excl_bits(int v, unsigned lt_mask, int *total)
{
    int ex = 0;
#pragma unroll
    for (int b = 0; b < BITS; b++) ex += __popc(__ballot_sync(FULL, (v >> b) & 1) & lt_mask) << b;
    *total = (int)__reduce_add_sync(FULL, (unsigned)v);
    return ex;
}

// MINB: resident blocks per SM the register allocation must allow (1..3): a
// tuning knob trading registers (spills) against warps in flight.
// F64T: opening tests in FP64 (used for one-target groups, where the tests are
// exactly the reference's); otherwise the tests run in FP32 on FP64-formed
// offsets from the group centre, against a bounding box rounded outwards.
template <int TPL, int MINB, bool F64T, bool POT, bool TMA = false>
__global__ void __launch_bounds__(WALK_THREADS, MINB) k_walk(WalkParams p)
{
    extern __shared__ float4 walk_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int FL = p.flush, cap = list_cap(FL);
    float *far = reinterpret_cast<float *>(walk_smem + (size_t)warp * walk_warp_float4s(FL));
    float *nearE = far + 4 * cap;
    float *nearH = nearE + 4 * cap;
    int *sstack = reinterpret_cast<int *>(far + 12 * cap);
    int4 *const nslot = reinterpret_cast<int4 *>(far + 12 * cap + WALK_SSTACK) + 4 * lane;
    const unsigned slot0 = (unsigned)__cvta_generic_to_shared(far + 12 * cap + WALK_SSTACK);
    int *pq = reinterpret_cast<int *>(far + 12 * cap + WALK_SSTACK + 32 * 16);
    const unsigned bar = (unsigned)__cvta_generic_to_shared(far + 12 * cap + WALK_SSTACK + 32 * 16 + PQ_CAP);
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    unsigned phase = 0;   // parity of the barrier phase the next wait is for
    constexpr bool tma = TMA;   // node staging by bulk copies (else per-lane cp.async)
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
        // evaluate the top m (<= 32) particles of the queue, one per lane:
        // classify them against the group box and append them to the lists
        int qn = 0;
        auto take_particles = [&](int m) {
            bool use = false, pfar = false;
            float4 pe = make_float4(0.f, 0.f, 0.f, 0.f);
            float ph = 0.f;
            if (lane < m) {
                const GGPart pp = load_part(p.parts + pq[qn - m + lane]);
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
            qn -= m;
            const unsigned mf = __ballot_sync(FULL, use && pfar);   // also orders the queue reads before reuse
            const unsigned mn = __ballot_sync(FULL, use && !pfar);
            if (use) {
                if (pfar) list_put(far, nf + __popc(mf & lt_mask), pe);
                else {
                    const int pos = nn + __popc(mn & lt_mask);
                    list_put(nearE, pos, pe);
                    list_put(nearH, pos, near_soft(ph, pe.w, homog, hmax));
                }
            }
            nf += __popc(mf);
            nn += __popc(mn);
            list_far += __popc(mf);
            list_near += __popc(mn);
            if (nf >= FL) { flush_far<TPL, POT>(far, nf, T); nf = 0; }
            if (nn >= FL) { flush_near_sel<TPL, POT>(homog, nearE, nearH, nn, T); nn = 0; }
            __syncwarp();
        };
        int node = -1;
        int k = pop_nodes(node);
        if (tma) {
            if (k > 0) stage_nodes(bar, slot0, p.nodes, node, k, lane);   // one barrier phase per staged round
        } else if (lane < k) {
            stage_node(nslot, p.nodes + node);
        }
        bool timed_out = false;
        while (k > 0) {
            tested += k;
            if (tma) {
                if (!bar_wait(bar, phase)) {
                    timed_out = true;
                    break;
                }
                phase ^= 1u;
            } else {
                asm volatile("cp.async.wait_all;" ::: "memory");
            }

            int act = 0, na = 0, nb = 0;
            bool isfar = false;
            float4 ent = make_float4(0.f, 0.f, 0.f, 0.f);
            float hp = 0.f;
            if (lane < k) {
                GGNode nd;
#pragma unroll
                for (int i = 0; i < 4; i++) reinterpret_cast<int4 *>(&nd)[i] = nslot[i];
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
                    if (isfar) list_put(far, nf + __popc(mf & lt_mask), ent);
                    else {
                        int pos = nn + __popc(mn & lt_mask);
                        list_put(nearE, pos, ent);
                        list_put(nearH, pos, near_soft(hp, ent.w, homog, hmax));
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
                const int nch = (act == 2) ? nb : 0;   // 1..8 children
                int total;
                const int ex = warp_excl_bits<4>(nch, lt_mask, &total);
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
                const int o = sp + ex;
                for (int c = 0; c < nch; c++) sstack[o + c] = na + c;
                sp += total;
                __syncwarp();
            }
            // next round's node records are staged now; the copies complete behind
            // this round's flushes and leaf particles
            int next_node = -1;
            const int next_k = pop_nodes(next_node);
            if (tma) {
                if (next_k > 0) stage_nodes(bar, slot0, p.nodes, next_node, next_k, lane);
            } else if (lane < next_k) {
                stage_node(nslot, p.nodes + next_node);
            }
            if (nf >= FL) { flush_far<TPL, POT>(far, nf, T); nf = 0; }
            if (nn >= FL) { flush_near_sel<TPL, POT>(homog, nearE, nearH, nn, T); nn = 0; }
            // opened leaves -> their particles onto the particle queue, which
            // is evaluated 32 particles at a time (leftovers wait for later
            // rounds).  A push that does not fit is taken in parts, the queue
            // drained between them.
            {
                int first = na, rem = (act == 3) ? -nb : 0;
                while (__any_sync(FULL, rem > 0)) {
                    int P, ex;
                    const unsigned big = __ballot_sync(FULL, rem >= 16);
                    if (!big) {
                        ex = warp_excl_bits<4>(rem, lt_mask, &P);   // leaves of up to 15 particles
                    } else if (!__any_sync(FULL, rem >= 64)) {
                        ex = warp_excl_bits<6>(rem, lt_mask, &P);
                    } else {
                        const int incl = warp_incl_scan(rem, lane);
                        P = __shfl_sync(FULL, incl, 31);
                        ex = incl - rem;
                    }
                    const int room = PQ_CAP - qn;
                    const int take = min(max(room - ex, 0), rem);
                    for (int c = 0; c < take; c++) pq[qn + ex + c] = first + c;
                    qn += min(P, room);
                    first += take;
                    rem -= take;
                    __syncwarp();
                    while (qn >= 32) take_particles(32);
                }
            }
            k = next_k;
            node = next_node;
        }
        if (!tma) asm volatile("cp.async.wait_all;" ::: "memory");   // no copy into the slot outlives its group
        if (timed_out) {   // copies may still be in flight: wait once more, then leave
            if (lane == 0) atomicOr(p.err, GG_EBIT_WALK_TIMEOUT);
            bar_wait(bar, phase);
            return;
        }
        if (overflow) {
            if (lane == 0) atomicOr(p.err, GG_EBIT_STACK_OVERFLOW);
            continue;
        }
        if (qn > 0) take_particles(qn);
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

template <int TPL, int MINB, bool F64T, bool POT = false, bool TMA = false>
static void launch_walk_t(const WalkParams &p, int blocks, int smem, cudaStream_t st)
{
    cudaFuncSetAttribute(k_walk<TPL, MINB, F64T, POT, TMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    k_walk<TPL, MINB, F64T, POT, TMA><<<blocks, WALK_THREADS, smem, st>>>(p);
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
    } else if (p.node_staging == 1) {   // bulk-copy node staging (the force walk's tuned forms)
        if (tpl == 2) {
            if (minb == 3) launch_walk_t<2, 3, false, false, true>(p, blocks, smem, st);
            else launch_walk_t<2, 2, false, false, true>(p, blocks, smem, st);
        } else {
            if (minb == 3) launch_walk_t<1, 3, false, false, true>(p, blocks, smem, st);
            else launch_walk_t<1, 2, false, false, true>(p, blocks, smem, st);
        }
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
