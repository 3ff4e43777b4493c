// gg_util.cu -- scans, walk-group tables, active-target compaction and the
// FP64 direct summation used to measure force errors.
#include <algorithm>
#include <climits>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define SC_THREADS 256
#define SC_ITEMS 8   // consecutive elements per thread: one block-wide scan per 2048

static int scan_blocks() { return gg_num_sms() * 4; }
int gg_scan_scratch_ints() { return scan_blocks() + 64; }

// ---- exclusive scan of n ints into out[0..n] (out[n] = total); in may be
// read as 0/1 flags (nonzero_mode) -------------------------------------------
__device__ __forceinline__ int block_excl_scan(int v, int *ws, int *total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < nw ? ws[lane] : 0, u = t;
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, u, o);
            if (lane >= o) u += y;
        }
        if (lane < nw) ws[lane] = u - t;
        if (lane == nw - 1) ws[32] = u;
    }
    __syncthreads();
    int r = x - v + ws[w];
    *total = ws[32];
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(const int *__restrict__ in, int n, int nonzero, int *bsum)
{
    __shared__ int ws[33];
    const int G = gridDim.x, chunk = (n + G - 1) / G;
    const int cb = blockIdx.x * chunk, ce = min(n, cb + chunk);
    int acc = 0;
    int i = cb + threadIdx.x;
    for (; i + 3 * SC_THREADS < ce; i += 4 * SC_THREADS) {   // four loads in flight per thread
        const int a = in[i], b = in[i + SC_THREADS], c = in[i + 2 * SC_THREADS], d = in[i + 3 * SC_THREADS];
        acc += nonzero ? (a != 0) + (b != 0) + (c != 0) + (d != 0) : a + b + c + d;
    }
    for (; i < ce; i += SC_THREADS) {
        const int v = in[i];
        acc += nonzero ? (v != 0) : v;
    }
    int tot;
    block_excl_scan(acc, ws, &tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_top(int *bsum, int G)
{
    __shared__ int ws[33];
    int carry = 0;
    for (int base = 0; base < G; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < G ? bsum[i] : 0, tot;
        int e = block_excl_scan(v, ws, &tot);
        if (i < G) bsum[i] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) bsum[G] = carry;
}

// each thread scans SC_ITEMS consecutive elements of a 2048-element tile in
// registers; one block-wide scan of the threads' sums per tile
__global__ void k_scan_down(const int *__restrict__ in, int n, int nonzero, const int *__restrict__ bsum, int *out)
{
    __shared__ int ws[33];
    const int G = gridDim.x, chunk = (n + G - 1) / G;
    const int cb = blockIdx.x * chunk, ce = min(n, cb + chunk);
    int run = bsum[blockIdx.x];
    for (int base = cb; base < ce; base += SC_THREADS * SC_ITEMS) {
        const int i0 = base + threadIdx.x * SC_ITEMS;
        int v[SC_ITEMS], sum = 0;
#pragma unroll
        for (int j = 0; j < SC_ITEMS; j++) {
            int x = i0 + j < ce ? in[i0 + j] : 0;
            if (nonzero) x = (x != 0);
            v[j] = x;
            sum += x;
        }
        int tot;
        int r = run + block_excl_scan(sum, ws, &tot);
#pragma unroll
        for (int j = 0; j < SC_ITEMS; j++) {
            if (i0 + j < ce) out[i0 + j] = r;
            r += v[j];
        }
        run += tot;
    }
    if (blockIdx.x == G - 1 && threadIdx.x == 0) out[n] = bsum[G];
}

static void scan_run(const int *in, int *out, int n, int nonzero, int *scratch, cudaStream_t st)
{
    int G = scan_blocks();
    k_scan_reduce<<<G, SC_THREADS, 0, st>>>(in, n, nonzero, scratch);
    k_scan_top<<<1, 1024, 0, st>>>(scratch, G);
    k_scan_down<<<G, SC_THREADS, 0, st>>>(in, n, nonzero, scratch, out);
    gg_note_launches(3);
}

void gg_launch_scan(const int *in, int *out, int n, int *scratch, cudaStream_t st)
{
    scan_run(in, out, n, 0, scratch, st);
}

#define GG_ORDER_MAX_LEVEL 14

// cell level of the target order of system s: the deepest level whose cells
// are still as large as the system's largest kernel radius, at most lmax
__device__ __forceinline__ int target_order_level(const GGDomainDev *__restrict__ dom,
                                                  const unsigned *__restrict__ hmm, int s, int lmax)
{
    const float hmax = __uint_as_float(hmm[2 * s + 1]);
    const double len = dom[s].len;
    int L = 0;
    if (hmax > 0.f && isfinite(hmax))
        while (L < lmax && ldexp(len, -(L + 1)) >= (double)hmax) L++;
    else
        L = lmax;
    return L;
}

// ---- groups: ceil(n_s / gs) groups per system -------------------------------
__global__ void k_groups_count(const int *__restrict__ toff, int S, int gs, int *gscan, int *ngroups)
{
    __shared__ int ws[33];
    int carry = 0;
    for (int base = 0; base < S; base += blockDim.x) {
        int s = base + threadIdx.x;
        int v = 0;
        if (s < S) v = (toff[s + 1] - toff[s] + gs - 1) / gs;
        int tot;
        int e = block_excl_scan(v, ws, &tot);
        if (s < S) gscan[s] = carry + e;
        carry += tot;
    }
    if (threadIdx.x == 0) {
        gscan[S] = carry;
        *ngroups = carry;
    }
}

__global__ void k_groups_write(const int *__restrict__ toff, const int *__restrict__ gscan, int S, int gs,
                               const int *__restrict__ ngroups, GGGroup *groups)
{
    const int ng = *ngroups;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
        int lo = 0, hi = S - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (gscan[mid] <= g) lo = mid; else hi = mid - 1;
        }
        int s = lo;
        int k = g - gscan[s];
        int first = toff[s] + k * gs;
        GGGroup gr;
        gr.first = first;
        gr.count = min(gs, toff[s + 1] - first);
        gr.root = s;
        gr.sys = s;
        groups[g] = gr;
    }
}

void gg_launch_groups(const int *toff, int S, int gs, GGGroup *groups, int *ngroups, int *gscan, cudaStream_t st)
{
    k_groups_count<<<1, 1024, 0, st>>>(toff, S, gs, gscan, ngroups);
    k_groups_write<<<gg_num_sms() * 8, 256, 0, st>>>(toff, gscan, S, gs, ngroups, groups);
    gg_note_launches(2);
}

// ---- groups bounded by tree nodes ------------------------------------------------
// A group opens every node that reaches into the bounding box of its targets,
// down to the particles for nodes inside the box.  Consecutive targets in key
// order can still be far apart (the curve crosses sparse regions in long
// strides), and then the box of a run of gs of them encloses dense regions none
// of them belong to, which every target of the group opens to the particles: on
// the 16.8M clustered system single groups of 64 outskirt targets, whose boxes
// held 160,000-260,000 particles, ran longer than the rest of the walk together.
// So a group never spans two "group nodes": the shallowest tree nodes holding at
// most gs * GG_GROUP_NODE_GROUPS of the walk's targets, or lying at or below the
// cell level the target order sorts by (targets ordered by softening class are
// contiguous only per cell).  Within a group node the targets are cut into runs
// of gs as before.  The rule depends on the system's own tree and targets only,
// so a system's groups do not depend on the systems batched with it.
#define GG_GROUP_NODE_GROUPS 64

__device__ __forceinline__ bool group_node_pred(const TreeBuf &tb, const int *__restrict__ tscan, int k, int cap,
                                                int lo)
{
    const int b = tb.start[k], e = tb.end[k];
    const int targets = tscan ? tscan[e] - tscan[b] : e - b;
    return targets <= cap || tb.level[k] >= lo;
}

// gnode[i] = the group node of sorted particle i.  tscan: exclusive count of
// the walk's targets before each sorted particle (NULL: every particle is a
// target).  A warp takes 32 nodes at a time and writes each group node's
// particle range with all its lanes.
__global__ void k_group_nodes(TreeBuf tb, const int *__restrict__ tscan, int gs, const GGDomainDev *__restrict__ dom,
                              const unsigned *__restrict__ hmm, int lmax, int *__restrict__ gnode)
{
    const int nn = *tb.nnodes;
    const int lane = threadIdx.x & 31;
    const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const int cap = GG_GROUP_NODE_GROUPS * gs;
    for (int base = wg * 32; base < nn; base += nw * 32) {
        const int k = base + lane;
        bool is_gn = false;
        if (k < nn) {
            const int lo = dom ? target_order_level(dom, hmm, tb.sys[k], lmax) : INT_MAX;
            const int par = tb.parent[k];
            is_gn = group_node_pred(tb, tscan, k, cap, lo) && (par < 0 || !group_node_pred(tb, tscan, par, cap, lo));
        }
        unsigned m = __ballot_sync(0xffffffffu, is_gn);
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const int kk = base + j;
            const int b = tb.start[kk], e = tb.end[kk];
            for (int i = b + lane; i < e; i += 32) gnode[i] = kk;
        }
    }
}

// flag[t] = 1 where target t starts a new group node
__global__ void k_group_seg_flags(int nt, const int *__restrict__ tlist, const int *__restrict__ gnode,
                                  int *__restrict__ flag)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        const int pi = tlist ? tlist[t] : t;
        flag[t] = (t == 0 || gnode[pi] != gnode[tlist ? tlist[t - 1] : t - 1]) ? 1 : 0;
    }
}

// segstart[j] = first target of segment j; segstart[nseg] = nt
__global__ void k_group_seg_starts(int nt, const int *__restrict__ flag, const int *__restrict__ segidx,
                                   int *__restrict__ segstart)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        if (flag[t]) segstart[segidx[t]] = t;
        if (t == 0) segstart[segidx[nt]] = nt;
    }
}

// seg[t] becomes the segment holding target t, flag[t] 1 where t starts a
// group: every gs-th target of its segment (both in place, one thread per t)
__global__ void k_group_start_flags(int nt, int *__restrict__ flag, int *__restrict__ seg,
                                    const int *__restrict__ segstart, int gs)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        const int j = seg[t] + flag[t] - 1;
        seg[t] = j;
        flag[t] = ((t - segstart[j]) % gs) == 0 ? 1 : 0;
    }
}

__global__ void k_group_write_tree(int nt, const int *__restrict__ flag, const int *__restrict__ seg,
                                   const int *__restrict__ segstart, const int *__restrict__ gidx,
                                   const int *__restrict__ toff, int S, int gs, int maxg, GGGroup *__restrict__ groups,
                                   int *__restrict__ ngroups, int *__restrict__ err)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        if (t == 0) *ngroups = min(gidx[nt], maxg);
        if (!flag[t]) continue;
        const int g = gidx[t];
        if (g >= maxg) {   // cannot happen: the table is sized for the bound on group nodes
            atomicOr(err, GG_EBIT_NODE_OVERFLOW);
            continue;
        }
        const int j = seg[t];
        int lo = 0, hi = S - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (toff[mid] <= t) lo = mid; else hi = mid - 1;
        }
        GGGroup gr;
        gr.first = t;
        gr.count = min(gs, segstart[j + 1] - t);
        gr.root = lo;
        gr.sys = lo;
        groups[g] = gr;
    }
}

// Upper bound of the number of groups: every group node is a root or a child
// of a node holding more than gs * GG_GROUP_NODE_GROUPS targets (fewer than
// n / (gs * GG_GROUP_NODE_GROUPS) per depth, at most 8 children each); each
// adds at most one partial group to the n / gs full ones.
long long gg_max_groups(long long n, int S, int gs)
{
    if (gs <= 1) return n + S + 1;
    const long long per_depth = n / ((long long)gs * GG_GROUP_NODE_GROUPS) + 1;
    return n / gs + 2LL * S + 1 + 8LL * GG_MAX_DEPTH * per_depth;
}

// Scratch: gnode n_particles + 1 ints (reused for the group index scan),
// flag nt, seg and segstart nt + 1 each.
void gg_launch_groups_tree(int nt, const int *tlist, const int *tscan, const int *toff, int S, int gs,
                           const TreeBuf &tb, const GGDomainDev *order_dom, const unsigned *hmm, int lmax, int *gnode,
                           int *flag, int *seg, int *segstart, int maxg, GGGroup *groups, int *ngroups,
                           int *scan_scratch, int *err, cudaStream_t st)
{
    const int threads = 256, blocks = gg_num_sms() * 8;
    if (nt <= 0) {
        cudaMemsetAsync(ngroups, 0, sizeof(int), st);
        return;
    }
    k_group_nodes<<<blocks, threads, 0, st>>>(tb, tscan, gs, order_dom, hmm, lmax, gnode);
    k_group_seg_flags<<<blocks, threads, 0, st>>>(nt, tlist, gnode, flag);
    scan_run(flag, seg, nt, 0, scan_scratch, st);
    k_group_seg_starts<<<blocks, threads, 0, st>>>(nt, flag, seg, segstart);
    k_group_start_flags<<<blocks, threads, 0, st>>>(nt, flag, seg, segstart, gs);
    int *gidx = gnode;   // the group nodes are no longer needed
    scan_run(flag, gidx, nt, 0, scan_scratch, st);
    k_group_write_tree<<<blocks, threads, 0, st>>>(nt, flag, seg, segstart, gidx, toff, S, gs, maxg, groups, ngroups,
                                                   err);
    gg_note_launches(5);
}

int gg_target_order_lmax(int S)
{
    int sbits = 0;
    while ((1 << sbits) < S) sbits++;
    return std::min(GG_ORDER_MAX_LEVEL, (64 - 8 - sbits) / 3);
}

// ---- group order by measured cost -----------------------------------------------
// Groups are handed to the persistent walk warps by an atomic counter.  In
// target order the dearest groups (dense centres, sparse outskirts) may come
// last and leave a tail in which few warps still work.  Each walk records per
// target its group's device cycles divided by the group's size; the next walk
// sums these over each of its own groups and hands the groups out most
// expensive first (longest-processing-time-first list scheduling), by whole
// octaves of cost: that ends the walk as early as a full sort by cost would
// on the measured galaxy, clustered and Plummer costs, and keeps most groups
// in target order.  A group's result does not depend on when it runs, so the
// order changes no output.
__global__ void k_group_cost(const GGGroup *__restrict__ groups, const int *__restrict__ ngroups, int maxg,
                             const int *__restrict__ tlist, const unsigned *__restrict__ perm,
                             const float *__restrict__ cost, unsigned long long *key, unsigned *val)
{
    const int ng = *ngroups;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < maxg; g += gridDim.x * blockDim.x) {
        unsigned k = 255u;   // past the device count: last
        if (g < ng) {
            const GGGroup G = groups[g];
            float c = 0.f;
            for (int t = G.first; t < G.first + G.count; t++) c += cost[perm[tlist ? tlist[t] : t]];
            // descending octave of the cost (the float's exponent field); a
            // valid group never takes the last key
            k = 255u - max(__float_as_uint(fmaxf(c, 0.f)) >> 23, 1u);
        }
        key[g] = k;
        val[g] = (unsigned)g;
    }
}

gg_status gg_order_groups_by_cost(const GGGroup *groups, const int *ngroups, int maxg, const int *tlist,
                                  const unsigned *perm, const float *cost, unsigned long long *key,
                                  unsigned *gorder, void *sort_scratch, int *err, cudaStream_t st)
{
    if (maxg <= 0) return GG_OK;
    const int blocks = std::max(1, std::min(gg_num_sms() * 4, (maxg + 255) / 256));
    k_group_cost<<<blocks, 256, 0, st>>>(groups, ngroups, maxg, tlist, perm, cost, key, gorder);
    gg_note_launches(1);
    // one pass over the 8-bit key; the sort is stable, so the groups of one cost octave keep
    // target order and neighbouring warps still walk neighbouring regions
    return gg_sort_pairs_run(key, gorder, maxg, 8, 0, nullptr, 1, sort_scratch, err, st);
}

// ---- active targets ------------------------------------------------------------
__global__ void k_mark_active(const int *__restrict__ active, int n_active, const unsigned *__restrict__ rank, int n,
                              int *flag, int *err)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n_active; j += gridDim.x * blockDim.x) {
        int a = active[j];
        if (a < 0 || a >= n) { atomicOr(err, GG_EBIT_BAD_INPUT); continue; }
        flag[rank[a]] = j + 1;
    }
}

__global__ void k_compact_active(const int *__restrict__ flag, const int *__restrict__ scan, int n, int *tlist,
                                 int *tout, const int *__restrict__ poff, int S, int *toff)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int f = flag[i];
        if (f) {
            int t = scan[i];
            tlist[t] = i;
            tout[t] = f - 1;
        }
    }
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= S; s += gridDim.x * blockDim.x) toff[s] = scan[poff[s]];
}

void gg_launch_active(const int *active, int n_active, const unsigned *rank, int n, int *flag, int *flagscan,
                      int *tlist, int *tout, const int *poff, int S, int *toff, int *scratch, int *err,
                      cudaStream_t st)
{
    cudaMemsetAsync(flag, 0, (size_t)n * sizeof(int), st);
    k_mark_active<<<gg_num_sms() * 4, 256, 0, st>>>(active, n_active, rank, n, flag, err);
    scan_run(flag, flagscan, n, 1, scratch, st);
    k_compact_active<<<gg_num_sms() * 8, 256, 0, st>>>(flag, flagscan, n, tlist, tout, poff, S, toff);
    gg_note_launches(2);
}

// ---- FP64 direct summation ---------------------------------------------------
// Same pair rule as the walk (forcetree.c:2258-2283): Newtonian when r >= h_i
// and r >= h_j, otherwise the cubic spline with h = max(h_i, h_j).
__device__ __forceinline__ void spline64(double u, double hinv, double *wf, double *wp)
{
    if (u < 0.5) {
        *wf = (10.666666666667 + u * u * (32.0 * u - 38.4)) * hinv * hinv * hinv;
        *wp = (-2.8 + u * u * (5.333333333333 + u * u * (6.4 * u - 9.6))) * hinv;
    } else {
        *wf = (21.333333333333 - 48.0 * u + 38.4 * u * u - 10.666666666667 * u * u * u - 0.066666666667 / (u * u * u)) *
              hinv * hinv * hinv;
        *wp = (-3.2 + 0.066666666667 / u + u * u * (10.666666666667 + u * (-16.0 + u * (9.6 - 2.133333333333 * u)))) *
              hinv;
    }
}

#define DS_TILE 256
__global__ void __launch_bounds__(DS_TILE) k_direct(long long nsrc, const double *__restrict__ pos,
                                                    const double *__restrict__ mass, const double *__restrict__ h,
                                                    long long ntgt, const int *__restrict__ targets, double *acc,
                                                    double *pot)
{
    __shared__ double sx[DS_TILE], sy[DS_TILE], sz[DS_TILE], sm[DS_TILE], sh[DS_TILE];
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool valid = t < ntgt;
    long long i = valid ? (targets ? targets[t] : t) : 0;
    double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2], hi = h[i];
    double ax = 0, ay = 0, az = 0, pp = 0;
    for (long long base = 0; base < nsrc; base += DS_TILE) {
        long long j = base + threadIdx.x;
        __syncthreads();
        if (j < nsrc) {
            sx[threadIdx.x] = pos[3 * j]; sy[threadIdx.x] = pos[3 * j + 1]; sz[threadIdx.x] = pos[3 * j + 2];
            sm[threadIdx.x] = mass[j]; sh[threadIdx.x] = h[j];
        } else {
            sm[threadIdx.x] = 0; sx[threadIdx.x] = sy[threadIdx.x] = sz[threadIdx.x] = 0; sh[threadIdx.x] = 0;
        }
        __syncthreads();
        int m = (int)min((long long)DS_TILE, nsrc - base);
        for (int k = 0; k < m; k++) {
            double dx = sx[k] - xi, dy = sy[k] - yi, dz = sz[k] - zi;
            double r2 = dx * dx + dy * dy + dz * dz;
            double mj = sm[k];
            if (r2 > 0 && mj > 0) {
                double r = sqrt(r2), hj = sh[k], fac, fp;
                if (r >= hi && r >= hj) {
                    fac = mj / (r2 * r);
                    fp = -mj / r;
                } else {
                    double hg = hi > hj ? hi : hj, hinv = 1.0 / hg, wf, wp;
                    spline64(r * hinv, hinv, &wf, &wp);
                    fac = mj * wf;
                    fp = mj * wp;
                }
                ax += dx * fac; ay += dy * fac; az += dz * fac; pp += fp;
            }
        }
    }
    if (valid) {
        acc[3 * t] = ax; acc[3 * t + 1] = ay; acc[3 * t + 2] = az;
        if (pot) pot[t] = pp;
    }
}

void gg_launch_direct(long long n_src, const double *pos, const double *mass, const double *h, long long n_tgt,
                      const int *targets, double *acc, double *pot, cudaStream_t st)
{
    long long blocks = (n_tgt + DS_TILE - 1) / DS_TILE;
    if (blocks < 1) return;
    k_direct<<<(unsigned)blocks, DS_TILE, 0, st>>>(n_src, pos, mass, h, n_tgt, targets, acc, pot);
    gg_note_launches(1);
}

// FP64 direct sum of sampled targets against the sources of their own system,
// read from the load-order records (masses and softenings as stored, FP32):
// the force and potential a sampled target would have with every node opened,
// and its stored mass.
// One block per target, the sources strided over the block and the sums
// reduced in a fixed order, so the result does not depend on scheduling.
// Used by the autotuner to measure a configuration's force errors.
#define DR_THREADS 256
__global__ void __launch_bounds__(DR_THREADS) k_direct_records(const GGPart *__restrict__ rec,
                                                               const int *__restrict__ poff,
                                                               const int2 *__restrict__ tg, int ntg,
                                                               double *__restrict__ acc, double *__restrict__ pot,
                                                               double *__restrict__ mass)
{
    __shared__ double red[4][DR_THREADS];
    for (int t = blockIdx.x; t < ntg; t += gridDim.x) {
        const int i = tg[t].x, s = tg[t].y;
        const GGPart q = rec[i];
        const double hi = (double)q.h;
        double ax = 0, ay = 0, az = 0, pp = 0;
        for (int j = poff[s] + threadIdx.x; j < poff[s + 1]; j += DR_THREADS) {
            const GGPart r = rec[j];
            const double dx = r.x - q.x, dy = r.y - q.y, dz = r.z - q.z;
            const double r2 = dx * dx + dy * dy + dz * dz, mj = (double)r.m;
            if (r2 > 0 && mj > 0) {
                const double rr = sqrt(r2), hj = (double)r.h;
                double fac, fp;
                if (rr >= hi && rr >= hj) {
                    fac = mj / (r2 * rr);
                    fp = -mj / rr;
                } else {
                    const double hg = hi > hj ? hi : hj, hinv = 1.0 / hg;
                    double wf, wp;
                    spline64(rr * hinv, hinv, &wf, &wp);
                    fac = mj * wf;
                    fp = mj * wp;
                }
                ax += dx * fac; ay += dy * fac; az += dz * fac; pp += fp;
            }
        }
        red[0][threadIdx.x] = ax; red[1][threadIdx.x] = ay; red[2][threadIdx.x] = az; red[3][threadIdx.x] = pp;
        __syncthreads();
        for (int w = DR_THREADS / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w)
                for (int k = 0; k < 4; k++) red[k][threadIdx.x] += red[k][threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            acc[3 * (size_t)t] = red[0][0]; acc[3 * (size_t)t + 1] = red[1][0]; acc[3 * (size_t)t + 2] = red[2][0];
            pot[t] = red[3][0];
            mass[t] = (double)q.m;
        }
        __syncthreads();
    }
}

// rows of an output (acc n*3, pot n; load order, or active order) gathered
// for the sampled targets (tg[t].x = the row)
__global__ void k_gather_rows(const double *__restrict__ acc, const double *__restrict__ pot,
                              const int2 *__restrict__ tg, int ntg, double *__restrict__ acc_out,
                              double *__restrict__ pot_out)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntg; t += gridDim.x * blockDim.x) {
        const size_t i = (size_t)tg[t].x;
        acc_out[3 * (size_t)t] = acc[3 * i];
        acc_out[3 * (size_t)t + 1] = acc[3 * i + 1];
        acc_out[3 * (size_t)t + 2] = acc[3 * i + 2];
        pot_out[t] = pot ? pot[i] : 0.0;
    }
}

void gg_launch_direct_records(const GGPart *rec, const int *poff, const int2 *tg, int ntg, double *acc, double *pot,
                              double *mass, cudaStream_t st)
{
    if (ntg < 1) return;
    const int blocks = std::min(ntg, gg_num_sms() * 8);
    k_direct_records<<<blocks, DR_THREADS, 0, st>>>(rec, poff, tg, ntg, acc, pot, mass);
    gg_note_launches(1);
}

void gg_launch_gather_rows(const double *acc, const double *pot, const int2 *tg, int ntg, double *acc_out,
                           double *pot_out, cudaStream_t st)
{
    if (ntg < 1) return;
    const int blocks = std::min((ntg + 255) / 256, gg_num_sms() * 4);
    k_gather_rows<<<blocks, 256, 0, st>>>(acc, pot, tg, ntg, acc_out, pot_out);
    gg_note_launches(1);
}

// ---- FP32 FMA throughput probe ---------------------------------------------
// Independent FMA chains per thread, enough warps to fill every SM: the
// CUDA-core FP32 roofline that the walk is measured against.
#define PEAK_CHAINS 8
__global__ void k_fma_peak(float *out, int iters, float a, float b)
{
    float x[PEAK_CHAINS];
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) x[c] = threadIdx.x * 1e-7f + c;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int c = 0; c < PEAK_CHAINS; c++) x[c] = fmaf(x[c], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < PEAK_CHAINS; c++) s += x[c];
    if (s == 1234.5f) out[0] = s;   // keeps the chains live
}

extern "C" gg_status gg_fp32_peak_probe(double *tflops, void *stream)
{
    if (!tflops) return GG_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    float *out = nullptr;
    GG_CUDA_TRY(cudaMallocAsync((void **)&out, 64, st));
    const int threads = 512, blocks = gg_num_sms() * 4, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0, st);
        k_fma_peak<<<blocks, threads, 0, st>>>(out, iters, 0.999999f, 1e-7f);
        gg_note_launches(1);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        double fl = 2.0 * PEAK_CHAINS * (double)iters * threads * blocks;
        if (ms > 0 && rep > 0) best = fl / (ms * 1e-3) / 1e12 > best ? fl / (ms * 1e-3) / 1e12 : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    GG_CUDA_TRY(cudaStreamSynchronize(st));
    *tflops = best;
    return GG_OK;
}

// ---- walk targets ordered by (system, cell, softening class) ------------------
// A walk group opens nodes for the largest softening among its targets, so in a
// halo + disk system a group that mixes the two gives its disk targets the
// halo's larger near zone.  Ordering the targets of a system by softening alone
// keeps groups homogeneous but stretches the rarer class thin across dense
// regions, and such groups then cost more than a warp's share of the whole
// walk.  So the order is: Peano-Hilbert cell at the softening scale (the
// deepest level whose cells are still as large as the system's largest kernel
// radius, at most GG_ORDER_MAX_LEVEL), then softening class (quarter octaves of
// h above the system's smallest), then key order.  Groups stay compact and are
// homogeneous wherever a cell holds enough targets of one class.
__global__ void k_target_keys(int nt, const int *__restrict__ tlist, const GGPart *__restrict__ parts,
                              const unsigned long long *__restrict__ pkeys, const int *__restrict__ poff, int S,
                              const GGDomainDev *__restrict__ dom, const unsigned *__restrict__ hmm, int lmax,
                              unsigned long long *key, unsigned *val)
{
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
        const int pi = tlist ? tlist[t] : t;
        int lo = 0, hi = S - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (__ldg(poff + mid) <= pi) lo = mid; else hi = mid - 1;
        }
        const unsigned hmin_bits = hmm[2 * lo];
        const int L = target_order_level(dom, hmm, lo, lmax);
        const unsigned long long cell = (pkeys[pi] >> (3 * (GG_MAX_LEVEL - L))) << (3 * (lmax - L));
        const unsigned hb = __float_as_uint(fmaxf(parts[pi].h, 0.f));
        const unsigned cls = hb > hmin_bits ? min((hb - hmin_bits) >> 21, 255u) : 0u;
        key[t] = ((unsigned long long)lo << (3 * lmax + 8)) | (cell << 8) | cls;
        val[t] = (unsigned)t;
    }
}

__global__ void k_target_apply(int nt, const unsigned *__restrict__ val, const int *__restrict__ tlist_in,
                               const int *__restrict__ tout_in, int *tlist_out, int *tout_out)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
        int t = (int)val[k];
        tlist_out[k] = tlist_in ? tlist_in[t] : t;
        if (tout_out) tout_out[k] = tout_in[t];
    }
}

gg_status gg_order_targets_by_softening(int nt, const int *tlist_in, const int *tout_in, const GGPart *parts,
                                        const unsigned long long *pkeys, const int *poff, int S,
                                        const GGDomainDev *dom, const unsigned *hmm, unsigned long long *key,
                                        unsigned *val, int *tlist_out, int *tout_out, void *sort_scratch, int *err,
                                        cudaStream_t st)
{
    if (nt <= 0) return GG_OK;
    int sbits = 0;
    while ((1 << sbits) < S) sbits++;
    const int lmax = gg_target_order_lmax(S);
    const int key_bits = sbits + 3 * lmax + 8;
    int blocks = gg_num_sms() * 4;
    k_target_keys<<<blocks, 256, 0, st>>>(nt, tlist_in, parts, pkeys, poff, S, dom, hmm, lmax, key, val);
    gg_note_launches(1);
    gg_status s = gg_sort_pairs_run(key, val, nt, key_bits, 0, nullptr, 1, sort_scratch, err, st);
    if (s) return s;
    k_target_apply<<<blocks, 256, 0, st>>>(nt, val, tlist_in, tout_in, tlist_out, tout_out);
    gg_note_launches(1);
    return GG_OK;
}

// ---- FP64 energy and momentum checks (global.c:54 potential energy) ----------
// One block per chunk of one system sums m*phi/2 and m*a over its particles
// (load order) in a fixed order; a second kernel adds each system's chunk
// partials in chunk order, so the result does not depend on scheduling.
__global__ void k_energy_chunks(const int4 *__restrict__ chunks, const GGPart *__restrict__ rec,
                                const double *__restrict__ acc, const double *__restrict__ pot, double *part)
{
    const int4 ch = chunks[blockIdx.x];   // {system, first, end, unused}
    double w = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
    for (int i = ch.y + (int)threadIdx.x; i < ch.z; i += blockDim.x) {
        const double m = (double)rec[i].m;
        if (pot) w += 0.5 * m * pot[i];
        if (acc) {
            fx += m * acc[3 * (size_t)i];
            fy += m * acc[3 * (size_t)i + 1];
            fz += m * acc[3 * (size_t)i + 2];
        }
    }
    __shared__ double sh[4][256];
    sh[0][threadIdx.x] = w; sh[1][threadIdx.x] = fx; sh[2][threadIdx.x] = fy; sh[3][threadIdx.x] = fz;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o)
            for (int q = 0; q < 4; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 4) part[4 * (size_t)blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

__global__ void k_energy_systems(const int *__restrict__ sys_first_chunk, int S, const double *__restrict__ part,
                                 double *out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = sys_first_chunk[s]; c < sys_first_chunk[s + 1]; c++)
        for (int q = 0; q < 4; q++) v[q] += part[4 * (size_t)c + q];
    for (int q = 0; q < 4; q++) out[4 * (size_t)s + q] = v[q];
}

void gg_launch_energy(const int4 *chunks, int nchunks, const int *sys_first_chunk, int S, const GGPart *rec,
                      const double *acc, const double *pot, double *part, double *out, cudaStream_t st)
{
    if (nchunks > 0) {
        k_energy_chunks<<<nchunks, 256, 0, st>>>(chunks, rec, acc, pot, part);
        gg_note_launches(1);
    }
    k_energy_systems<<<(S + 127) / 128, 128, 0, st>>>(sys_first_chunk, S, part, out);
    gg_note_launches(1);
}
