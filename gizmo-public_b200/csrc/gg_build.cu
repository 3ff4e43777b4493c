// gg_build.cu -- particle permutation, oct-tree construction and moments.
//
// The reference builds its oct-tree by inserting particles one at a time
// (force_treebuild_single, gravity/forcetree.c:152-342) and then computes
// moments with a recursive depth-first pass (force_update_node_recursive,
// forcetree.c:434-942).  Here the tree comes straight from the sorted keys:
// a node is a run of particles sharing a key prefix, so a level-by-level pass
// finds each node's children by binary search on the next 3-bit key digit,
// and children are stored contiguously (first child + count).
//
// Two departures from the reference's node set, neither of which changes a
// force or the interaction count of a target:
//   * chains of single-child nodes are collapsed: a node is stored at the
//     deepest cell that still holds all its particles.  Every node in such a
//     chain has the same mass and centre of mass, and a deeper cell is never
//     opened where a shallower one is not (its len is smaller and its 1.2*len
//     box lies inside the parent's), so the walk uses the same monopole;
//   * a cell with at most `leaf_size` particles is a leaf bucket.  Opening it
//     yields its particles; leaf_size = 1 gives the reference's one-particle
//     leaves.  Cells at the 21-bit key depth with more particles are split
//     into chunks of leaf_size (the reference splits such near-coincident
//     particles at random, forcetree.c:219-231).
// Moments are FP64 sums (mass, mass-weighted position), children summed in
// key order, one depth per launch from the deepest up, with the centre of mass
// falling back to the geometric centre for empty cells (forcetree.c:764-781).
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define TB_THREADS 256
#define TB_GROUP 8                      // threads per node in the count/write kernels
#define TB_NODES (TB_THREADS / TB_GROUP)

__global__ void k_permute(const unsigned *__restrict__ perm, const GGPart *__restrict__ in, GGPart *__restrict__ out,
                          unsigned *__restrict__ rank, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned src = perm[i];
        if (src >= (unsigned)n) src = 0;   // only after a failed sort, which is reported
        out[i] = in[src];
        rank[src] = (unsigned)i;
    }
}

// roots: one per system, geometric level 0 (the domain cube), depth 0
__global__ void k_tree_roots(int S, const int *__restrict__ poff, TreeBuf tb)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0) {
        tb.depth_beg[0] = 0;
        tb.depth_beg[1] = S;
        tb.nnodes[0] = S;
    }
    if (s >= S) return;
    tb.start[s] = poff[s];
    tb.end[s] = poff[s + 1];
    tb.level[s] = 0;
    tb.parent[s] = -1;
    tb.sys[s] = s;
}

// deepest common level of two keys (0..21)
__device__ __forceinline__ int common_level(unsigned long long a, unsigned long long b)
{
    unsigned long long x = a ^ b;
    if (x == 0) return GG_MAX_LEVEL;
    int p = 63 - __clzll((long long)x);   // highest differing bit, 0..62
    return GG_MAX_LEVEL - 1 - p / 3;
}

// first index in [lo,hi) with key >= v
__device__ __forceinline__ int lower_bound_key(const unsigned long long *__restrict__ keys, int lo, int hi,
                                               unsigned long long v)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// A full-depth cell with more than `leaf` particles is split into at most 8
// equal chunks (which split again at the next depth if still too large), so no
// node ever has more than 8 children.
__device__ __forceinline__ int chunk_size(int cnt, int leaf)
{
    const int n8 = min(8, (cnt + leaf - 1) / leaf);
    return (cnt + n8 - 1) / n8;
}
// every chunk non-empty: ceil(cnt / size) <= 8 chunks of `size` particles (the last may be shorter)
__device__ __forceinline__ int chunk_children(int cnt, int leaf)
{
    const int sz = chunk_size(cnt, leaf);
    return (cnt + sz - 1) / sz;
}

__device__ __forceinline__ unsigned tb_ld_status(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void tb_st_status(unsigned *p, unsigned v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
#define TB_PUBLISHED 0x80000000u
#define TB_SPIN_LIMIT (1 << 22)

// One depth of the build in one launch.  Blocks take their chunk of the
// depth's nodes in ticket order (an atomic counter, so that every block a
// block waits for has already started).  Count: 8 threads per node find the
// 7 digit boundaries (or the chunk split of a full-depth cell) and the child
// count; the block publishes its children total.  Then each block adds up the
// totals of the blocks before it -- they publish before they wait on anyone,
// so the bounded wait ends -- and writes its nodes' children at contiguous
// indices from there; the last block also sets the next depth's range.  A
// child index at or past the node capacity is not written and sets
// GG_EBIT_NODE_OVERFLOW (the capacity is sized so that it cannot happen).
__global__ void __launch_bounds__(TB_THREADS) k_tree_depth(int depth, const unsigned long long *__restrict__ keys,
                                                           TreeBuf tb, int leaf)
{
    __shared__ int s_sum, s_ticket, s_off, s_tot;
    __shared__ int s_red[TB_THREADS / 32];
    __shared__ int s_nch[TB_NODES];
    __shared__ int s_excl[TB_NODES];
    const int lb = tb.depth_beg[depth], le = tb.depth_beg[depth + 1];
    const int nl = le - lb;
    const int G = gridDim.x;
    if (threadIdx.x == 0) {
        s_ticket = (int)atomicAdd(tb.ticket + depth, 1u);
        s_sum = 0;
    }
    __syncthreads();
    const int blk = s_ticket;
    if (nl == 0) {   // nothing at this depth: the next one is empty too
        if (blk == G - 1 && threadIdx.x == 0) {
            tb.depth_beg[depth + 2] = le;
            tb.nnodes[0] = le;
        }
        return;
    }
    const int chunk = (nl + G - 1) / G;
    const int cb = lb + blk * chunk, ce = min(le, cb + chunk);
    const int g = threadIdx.x / TB_GROUP, j = threadIdx.x % TB_GROUP;
    const int gbase = (threadIdx.x & 31) & ~(TB_GROUP - 1);

    // ---- count
    int my = 0;
    for (int base = cb; base < ce; base += TB_NODES) {
        const int k = base + g;
        const bool valid = k < ce;
        int s = 0, e = 0, lev = 0;
        if (valid) { s = tb.start[k]; e = tb.end[k]; lev = tb.level[k]; }
        const int cnt = e - s;
        const bool split = valid && cnt > leaf && depth < GG_MAX_DEPTH - 1;
        const bool digit_mode = split && lev < GG_MAX_LEVEL;
        const bool chunk_mode = split && lev >= GG_MAX_LEVEL;
        int b = s;
        if (digit_mode && j > 0) {
            int shift = 3 * (GG_MAX_LEVEL - (lev + 1));
            unsigned long long prefix = keys[s] >> (shift + 3);
            b = lower_bound_key(keys, s, e, ((prefix << 3) | (unsigned long long)j) << shift);
        }
        if (digit_mode) tb.bnd[(size_t)k * 8 + j] = b;
        const int nb = __shfl_down_sync(0xffffffffu, b, 1, TB_GROUP);
        const int bn = (j < 7) ? nb : e;
        const unsigned m = __ballot_sync(0xffffffffu, digit_mode && bn > b);
        int nch = 0;
        if (digit_mode) nch = __popc((m >> gbase) & 0xFFu);
        else if (chunk_mode) nch = chunk_children(cnt, leaf);
        if (valid && j == 0) {
            tb.nch[k] = nch;
            tb.child[k] = -1;
            my += nch;
        }
    }
    if (my) atomicAdd(&s_sum, my);
    __syncthreads();
    if (threadIdx.x == 0) tb_st_status(tb.bstat + (size_t)depth * G + blk, TB_PUBLISHED | (unsigned)s_sum);

    // ---- this block's first child index: the totals of the blocks before it
    int before = 0;
    for (int i = threadIdx.x; i < blk; i += TB_THREADS) {
        const unsigned *w = tb.bstat + (size_t)depth * G + i;
        unsigned v = tb_ld_status(w);
        int spins = 0;
        while (!(v & TB_PUBLISHED)) {
            if (++spins > TB_SPIN_LIMIT) {
                atomicOr(tb.err, GG_EBIT_SORT_TIMEOUT);
                break;
            }
            __nanosleep(64);
            v = tb_ld_status(w);
        }
        before += (int)(v & ~TB_PUBLISHED);
    }
    before = __reduce_add_sync(0xffffffffu, before);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = before;
    __syncthreads();
    if (threadIdx.x == 0) {
        int off = 0;
        for (int w = 0; w < TB_THREADS / 32; w++) off += s_red[w];
        s_off = off;
        if (blk == G - 1) {   // the last chunk: the depth's total is known
            long long nxt = (long long)le + off + s_sum;
            if (nxt > tb.cap) {
                atomicOr(tb.err, GG_EBIT_NODE_OVERFLOW);
                nxt = tb.cap;
            }
            tb.depth_beg[depth + 2] = (int)nxt;
            tb.nnodes[0] = (int)nxt;
        }
    }
    __syncthreads();   // also orders this block's count-phase stores before the reads below
    if (s_sum == 0) return;

    // ---- write
    int run = le + s_off;
    for (int base = cb; base < ce; base += TB_NODES) {
        int k = base + g;
        bool valid = k < ce;
        if (j == 0) s_nch[g] = valid ? tb.nch[k] : 0;
        __syncthreads();
        if (threadIdx.x < 32) {
            int v = threadIdx.x < TB_NODES ? s_nch[threadIdx.x] : 0, x = v;
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if ((int)threadIdx.x >= o) x += y;
            }
            if (threadIdx.x < TB_NODES) s_excl[threadIdx.x] = x - v;
            if (threadIdx.x == 31) s_tot = x;
        }
        __syncthreads();
        if (valid) {
            int nch = s_nch[g];
            int first = run + s_excl[g];
            if (j == 0) tb.child[k] = nch ? first : -1;
            if (nch) {
                int s = tb.start[k], e = tb.end[k], lev = tb.level[k], sys = tb.sys[k];
                if (lev >= GG_MAX_LEVEL) {
                    const int csz = chunk_size(e - s, leaf);
                    for (int c = j; c < nch; c += TB_GROUP) {
                        int idx = first + c;
                        if (idx >= tb.cap) { atomicOr(tb.err, GG_EBIT_NODE_OVERFLOW); continue; }
                        int cs = s + c * csz, ce2 = min(e, cs + csz);
                        tb.start[idx] = cs; tb.end[idx] = ce2; tb.level[idx] = GG_CHUNK_LEVEL;
                        tb.parent[idx] = k; tb.sys[idx] = sys;
                    }
                } else {
                    int b = tb.bnd[(size_t)k * 8 + j];
                    int bn = (j < 7) ? tb.bnd[(size_t)k * 8 + j + 1] : e;
                    int rank = 0;
                    for (int jj = 0; jj < j; jj++) {
                        int b0 = tb.bnd[(size_t)k * 8 + jj];
                        int b1 = (jj < 7) ? tb.bnd[(size_t)k * 8 + jj + 1] : e;
                        rank += b1 > b0;
                    }
                    if (bn > b) {
                        int idx = first + rank;
                        if (idx >= tb.cap) {
                            atomicOr(tb.err, GG_EBIT_NODE_OVERFLOW);
                        } else {
                            tb.start[idx] = b; tb.end[idx] = bn;
                            tb.level[idx] = common_level(keys[b], keys[bn - 1]);
                            tb.parent[idx] = k; tb.sys[idx] = sys;
                        }
                    }
                }
            }
        }
        int tot = s_tot;
        __syncthreads();
        run += tot;
    }
}

// Bottom-up moments, one depth per launch from the deepest up: a leaf sums its
// particles, an internal node its children (one depth deeper, computed by the
// previous launch), each in index order in FP64.  Nodes are numbered depth by
// depth with the children of consecutive nodes consecutive, so the lanes of a
// warp read one contiguous stretch of child records (or of particles).
__global__ void k_tree_moments_depth(int depth, const GGPart *__restrict__ parts,
                                     const GGDomainDev *__restrict__ dom, TreeBuf tb, GGNode *__restrict__ nodes)
{
    const int lb = tb.depth_beg[depth], le = tb.depth_beg[depth + 1];
    for (int k = lb + blockIdx.x * blockDim.x + threadIdx.x; k < le; k += gridDim.x * blockDim.x) {
        const int lev = tb.level[k], sys = tb.sys[k];
        const GGDomainDev d = dom[sys];
        double M = 0, sx = 0, sy = 0, sz = 0;
        float maxsoft = 0;
        int a, b;
        const int s = tb.start[k];
        const int c0 = tb.child[k];
        if (c0 < 0) {   // leaf: its particles
            const int e = tb.end[k];
            for (int i = s; i < e; i++) {
                const GGPart p = parts[i];
                const double m = (double)p.m;
                M += m;
                sx += m * p.x; sy += m * p.y; sz += m * p.z;
                maxsoft = fmaxf(maxsoft, p.h);
            }
            a = s;
            b = -(e - s);
        } else {        // internal: its children
            const int nc = tb.nch[k];
            for (int c = c0; c < c0 + nc; c++) {
                const double m = tb.mass64[c];
                M += m;
                sx += m * nodes[c].cx;
                sy += m * nodes[c].cy;
                sz += m * nodes[c].cz;
                maxsoft = fmaxf(maxsoft, nodes[c].maxsoft);
            }
            a = c0;
            b = nc;
        }
        // geometric cell: level `lev` cell containing the node's first particle
        const int gl = lev > GG_MAX_LEVEL ? GG_MAX_LEVEL : lev;
        const double len = ldexp(d.len, -gl);
        double cen[3];
        if (gl == 0) {
            cen[0] = d.center[0]; cen[1] = d.center[1]; cen[2] = d.center[2];
        } else {
            const GGPart p0 = parts[s];
            const double pv[3] = {p0.x, p0.y, p0.z};
            for (int q = 0; q < 3; q++) {
                const unsigned cell = gg_quantize(pv[q], d.corner[q], d.len) >> (GG_MAX_LEVEL - gl);
                cen[q] = d.corner[q] + ((double)cell + 0.5) * len;
            }
        }
        double cx, cy, cz;
        if (M > 0) { cx = sx / M; cy = sy / M; cz = sz / M; }
        else { cx = cen[0]; cy = cen[1]; cz = cen[2]; }
        GGNode nd;
        nd.cx = cx; nd.cy = cy; nd.cz = cz;
        nd.mass = (float)M; nd.len = (float)len; nd.maxsoft = maxsoft;
        nd.gx = (float)(cen[0] - cx); nd.gy = (float)(cen[1] - cy); nd.gz = (float)(cen[2] - cz);
        nd.a = a; nd.b = b; nd.level = lev; nd.parent = tb.parent[k];
        nodes[k] = nd;
        tb.mass64[k] = M;
    }
}

void gg_launch_permute(const unsigned *perm, const GGPart *in, GGPart *out, unsigned *rank, int n, cudaStream_t st)
{
    int threads = 256, blocks = gg_num_sms() * 8;
    if ((long long)blocks * threads > n) blocks = (n + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    k_permute<<<blocks, threads, 0, st>>>(perm, in, out, rank, n);
    gg_note_launches(1);
}

// blocks of the per-depth count and write kernels: 8 per SM keeps enough binary
// searches in flight to hide their dependent loads
int gg_tree_grid() { return gg_num_sms() * 8; }

void gg_launch_tree(const unsigned long long *keys, const int *poff, int S, int leaf, int cap, TreeBuf tb,
                    const GGPart *parts, const GGDomainDev *dom, GGNode *nodes, cudaStream_t st)
{
    const int G = gg_tree_grid();
    k_tree_roots<<<(S + 127) / 128, 128, 0, st>>>(S, poff, tb);
    tb.cap = cap;
    cudaMemsetAsync(tb.ticket, 0, GG_MAX_DEPTH * sizeof(unsigned), st);
    cudaMemsetAsync(tb.bstat, 0, (size_t)GG_MAX_DEPTH * G * sizeof(unsigned), st);
    for (int depth = 0; depth < GG_MAX_DEPTH; depth++) k_tree_depth<<<G, TB_THREADS, 0, st>>>(depth, keys, tb, leaf);
    const int threads = 256, blocks = gg_num_sms() * 8;
    for (int depth = GG_MAX_DEPTH - 1; depth >= 0; depth--)
        k_tree_moments_depth<<<blocks, threads, 0, st>>>(depth, parts, dom, tb, nodes);
    gg_note_launches(1 + 2 * GG_MAX_DEPTH);
}
