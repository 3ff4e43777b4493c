// gg_sort.cu -- stable LSD radix sort of (64-bit key, 32-bit value) pairs.
//
// Replaces the reference's stable mergesort of {peanokey, index} records
// (mysort_peano, system/peano.c:414-462; mysort_domain, domain.c:2674-2723).
// Design (one-sweep): one up-front pass builds the digit histograms of every
// pass; each pass is then a single kernel in which a CTA ranks a tile of
// SORT_TILE keys in shared memory, publishes its per-digit counts, sums its
// predecessors' counts with a decoupled look-back, and writes the tile out
// digit-sorted so that global stores are contiguous runs.  SORT_BITS-bit
// digits (8: the 63-bit Peano-Hilbert keys take 8 passes).  For several
// systems further passes sort stably by system id (taken from the value, an
// index into the concatenated particle array), so the final order is
// (system, key).
//
// The look-back status words of a pass live in one of two arrays: pass p
// reads and writes array p % 2 and clears its own tile's words of the other
// array for pass p + 1 (whose tiles only start once every tile of pass p has
// finished), so one memset before the first pass serves every pass.
//
// Every wait in the look-back is bounded: after GG_SORT_SPIN_LIMIT polls the
// CTA records GG_EBIT_SORT_TIMEOUT in the error word and carries on, so a
// failure returns an error instead of hanging the device.
#include <algorithm>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#ifndef GG_SORT_BITS
#define GG_SORT_BITS 8
#endif
// 8-bit digits (8 passes for the 63-bit keys), 2560-key tiles, 4 blocks per
// SM: measured best on the 16.8M clustered system's keys with the vote-based
// ranking, early counts and windowed look-back (ms per sort):
//   9 bits x 2048 x 4: 2.11   9 x 3072 x 3: 1.90   9 x 4096 x 2: 1.98
//   8 bits x 2048 x 4: 1.78   8 x 2560 x 4: 1.69   8 x 3072 x 3: 1.73   8 x 4096 x 2: 1.89
// With match.any ranking 9 x 2048 x 4 had been best, at 2.46.
#ifndef GG_SORT_ITEMS
#define GG_SORT_ITEMS 10
#endif
#ifndef GG_SORT_MINB
#define GG_SORT_MINB 4    // blocks per SM the pass kernel's registers must allow
#endif

#define SORT_THREADS 256
#define SORT_ITEMS GG_SORT_ITEMS
#define SORT_TILE (SORT_THREADS * SORT_ITEMS)
#define SORT_WARPS (SORT_THREADS / 32)
#define SORT_BITS GG_SORT_BITS
#define RADIX (1 << SORT_BITS)
#define DPT (RADIX / SORT_THREADS)          // digits per thread in the per-digit phases
#define ST_AGG (1u << 30)
#define ST_INC (2u << 30)
#define ST_FLAGS (3u << 30)
#define ST_VALUE 0x3FFFFFFFu
#define GG_SORT_SPIN_LIMIT (1 << 22)
#ifndef GG_SORT_LB_WINDOW
#define GG_SORT_LB_WINDOW 4   // predecessors read per look-back round trip
#endif

static_assert(RADIX >= SORT_THREADS && RADIX % SORT_THREADS == 0, "each thread owns whole digits");
static_assert(SORT_BITS * GG_SORT_MAX_PASSES >= 64 + 32, "enough passes for a 64-bit key and a system id");

int gg_sort_bits() { return SORT_BITS; }

__device__ __forceinline__ int sort_sys_of(const int *__restrict__ poff, int S, unsigned v)
{
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if ((unsigned)__ldg(poff + mid) <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// histograms of all passes: passes [0, nkey) take key digits, passes
// [nkey, nkey+nsys) take system-id digits
__global__ void k_sort_hist(const unsigned long long *__restrict__ keys, const unsigned *__restrict__ vals, int n,
                            int nkey, int nsys, const int *__restrict__ poff, int S, unsigned *g_hist)
{
    extern __shared__ unsigned sh[];   // (nkey + nsys) * RADIX
    const int np = nkey + nsys;
    for (int i = threadIdx.x; i < np * RADIX; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long k = keys[i];
        for (int p = 0; p < nkey; p++) atomicAdd(&sh[p * RADIX + ((k >> (SORT_BITS * p)) & (RADIX - 1))], 1u);
        if (nsys) {
            const unsigned s = (unsigned)sort_sys_of(poff, S, vals[i]);
            for (int p = 0; p < nsys; p++)
                atomicAdd(&sh[(nkey + p) * RADIX + ((s >> (SORT_BITS * p)) & (RADIX - 1))], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np * RADIX; i += blockDim.x)
        if (sh[i]) atomicAdd(&g_hist[i], sh[i]);
}

// block-wide exclusive scan of DPT consecutive values per thread (digits
// DPT*tid .. DPT*tid+DPT-1); returns the thread's exclusive base and writes
// each digit's exclusive prefix into excl[]
__device__ __forceinline__ void block_excl_scan(const unsigned (&v)[DPT], unsigned (&excl)[DPT], unsigned *s_wsum)
{
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    unsigned t = 0;
#pragma unroll
    for (int q = 0; q < DPT; q++) { excl[q] = t; t += v[q]; }
    unsigned x = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[w] = x;
    __syncthreads();
    unsigned wo = 0;
    for (int ww = 0; ww < w; ww++) wo += s_wsum[ww];
    const unsigned base = x - t + wo;
#pragma unroll
    for (int q = 0; q < DPT; q++) excl[q] += base;
}

// exclusive scan of each pass's RADIX counts (one block of SORT_THREADS per pass)
__global__ void __launch_bounds__(SORT_THREADS) k_sort_hist_scan(const unsigned *g_hist, unsigned *g_off)
{
    __shared__ unsigned s_wsum[SORT_WARPS];
    const int p = blockIdx.x;
    unsigned v[DPT], e[DPT];
#pragma unroll
    for (int q = 0; q < DPT; q++) v[q] = g_hist[p * RADIX + DPT * threadIdx.x + q];
    block_excl_scan(v, e, s_wsum);
#pragma unroll
    for (int q = 0; q < DPT; q++) g_off[p * RADIX + DPT * threadIdx.x + q] = e[q];
}

__device__ __forceinline__ unsigned ld_status(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(unsigned *p, unsigned v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct SortSmem {
    unsigned long long keys[SORT_TILE];
    unsigned vals[SORT_TILE];
    unsigned short dig[SORT_TILE];
    unsigned whist[SORT_WARPS][RADIX];
    unsigned bhist[RADIX];   // the tile's digit counts, published before the ranking
    unsigned texcl[RADIX];
    unsigned gbase[RADIX];
    unsigned wsum[SORT_WARPS];
    int tile;
};

// one pass: digit = (key >> shift) & (RADIX-1), or of the system id when sys_mode.
// status: this pass's look-back words; status_next: the next pass's, of which
// this tile clears its own (nullptr for the last pass).  GATHER (the last pass
// of a build's sort): each pair's value is a record index, and the pass also
// moves that record to the pair's sorted position and records the position.
template <bool GATHER>
__global__ void __launch_bounds__(SORT_THREADS, GG_SORT_MINB) k_sort_pass(
    const unsigned long long *__restrict__ kin, const unsigned *__restrict__ vin, unsigned long long *__restrict__ kout,
    unsigned *__restrict__ vout, int n, int shift, int sys_mode, const int *__restrict__ poff, int S,
    const unsigned *__restrict__ g_off, unsigned *status, unsigned *status_next, unsigned *tile_counter, int *err,
    SortGather gather)
{
    extern __shared__ __align__(16) unsigned char sort_smem_raw[];
    SortSmem &sm = *reinterpret_cast<SortSmem *>(sort_smem_raw);

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) sm.tile = (int)atomicAdd(tile_counter, 1u);
    for (int i = tid; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&sm.whist[0][0])[i] = 0;
    for (int i = tid; i < RADIX; i += SORT_THREADS) sm.bhist[i] = 0;
    __syncthreads();
    const int tile = sm.tile;
    const long long tile_base = (long long)tile * SORT_TILE;
    const long long wbase = tile_base + (long long)w * 32 * SORT_ITEMS;
    const unsigned lt_mask = (1u << lane) - 1u;

    unsigned long long k[SORT_ITEMS];
    unsigned v[SORT_ITEMS], rank[SORT_ITEMS], dg[SORT_ITEMS];
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        const long long idx = wbase + j * 32 + lane;
        const bool valid = idx < n;
        k[j] = valid ? kin[idx] : ~0ull;
        v[j] = valid ? vin[idx] : 0u;
    }
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        const long long idx = wbase + j * 32 + lane;
        unsigned d;
        if (idx >= n) d = RADIX - 1;
        else if (sys_mode) d = ((unsigned)sort_sys_of(poff, S, v[j]) >> shift) & (RADIX - 1);
        else d = (unsigned)(k[j] >> shift) & (RADIX - 1);
        dg[j] = d;
        atomicAdd(&sm.bhist[d], 1u);
    }
    // Early counts: the tile's per-digit counts (items past n counted under the
    // last digit, as the ranking counts them) are published before the
    // ranking, so that successors looking back find them sooner.
    __syncthreads();
    unsigned *st = status + (size_t)tile * RADIX;
#pragma unroll
    for (int q = 0; q < DPT; q++) {
        const int d = DPT * tid + q;
        st_status(&st[d], (tile == 0 ? ST_INC : ST_AGG) | (sm.bhist[d] & ST_VALUE));
    }
    // stable warp-level ranking in (item, lane) order == index order
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        const unsigned d = dg[j];
        // lanes holding the same digit: one vote per digit bit (independent
        // votes, cheaper here than match.any)
        unsigned peers = 0xffffffffu;
#pragma unroll
        for (int b = 0; b < SORT_BITS; b++) {
            const unsigned m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
            peers &= ((d >> b) & 1u) ? m : ~m;
        }
        const int leader = __ffs(peers) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(&sm.whist[w][d], (unsigned)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        rank[j] = base + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();

    // per digit (thread tid owns digits DPT*tid ..): warp-exclusive offsets and the tile's count
    unsigned sum[DPT];
#pragma unroll
    for (int q = 0; q < DPT; q++) {
        const int d = DPT * tid + q;
        unsigned acc = 0;
#pragma unroll
        for (int ww = 0; ww < SORT_WARPS; ww++) {
            const unsigned c = sm.whist[ww][d];
            sm.whist[ww][d] = acc;
            acc += c;
        }
        sum[q] = acc;
    }
    // look back, digit by digit, and publish the inclusive counts
#pragma unroll
    for (int q = 0; q < DPT; q++) {
        const int d = DPT * tid + q;
        unsigned excl = 0;
        if (tile != 0) {
            // windowed look-back: GG_SORT_LB_WINDOW predecessors' words per
            // round trip, taken in order until the first inclusive one; a word
            // not yet published is polled again (bounded)
            int t = tile - 1;
            int spins = 0;
            while (t >= 0) {
                unsigned w[GG_SORT_LB_WINDOW];
#pragma unroll
                for (int i = 0; i < GG_SORT_LB_WINDOW; i++)
                    w[i] = t - i >= 0 ? ld_status(status + (size_t)(t - i) * RADIX + d) : ST_INC;
                int used = 0;
                bool done = false, waiting = false;
#pragma unroll
                for (int i = 0; i < GG_SORT_LB_WINDOW; i++) {
                    if (done || waiting) continue;
                    const unsigned f = w[i] & ST_FLAGS;
                    if (f == 0u) { waiting = true; continue; }
                    excl += w[i] & ST_VALUE;
                    used++;
                    if (f == ST_INC) done = true;
                }
                if (done) break;
                t -= used;
                if (waiting) {
                    if (++spins > GG_SORT_SPIN_LIMIT) {
                        atomicOr(err, GG_EBIT_SORT_TIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            st_status(&st[d], ST_INC | ((excl + sum[q]) & ST_VALUE));
        }
        sm.gbase[d] = g_off[d] + excl;
        if (status_next) status_next[(size_t)tile * RADIX + d] = 0u;
    }

    // exclusive scan of the tile's digit counts
    {
        unsigned e[DPT];
        block_excl_scan(sum, e, sm.wsum);
#pragma unroll
        for (int q = 0; q < DPT; q++) sm.texcl[DPT * tid + q] = e[q];
    }
    __syncthreads();

    // scatter into shared memory in digit order
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        const long long idx = wbase + j * 32 + lane;
        if (idx < n) {
            const unsigned dd = dg[j];
            const unsigned pos = sm.texcl[dd] + sm.whist[w][dd] + rank[j];
            sm.keys[pos] = k[j];
            sm.vals[pos] = v[j];
            sm.dig[pos] = (unsigned short)dd;
        }
    }
    __syncthreads();
    const long long rem = (long long)n - tile_base;
    const int nvalid = rem < SORT_TILE ? (int)rem : SORT_TILE;
    for (int i = tid; i < nvalid; i += SORT_THREADS) {
        const unsigned dd = sm.dig[i];
        const unsigned gpos = sm.gbase[dd] + (unsigned)i - sm.texcl[dd];
        if (gpos < (unsigned)n) {   // always true unless a look-back gave up
            const unsigned v = sm.vals[i];
            kout[gpos] = sm.keys[i];
            vout[gpos] = v;
            if (GATHER) {
                const unsigned src = v < (unsigned)n ? v : 0u;   // only after a failed sort, which is reported
                const int4 *from = reinterpret_cast<const int4 *>(gather.in + src);
                int4 *to = reinterpret_cast<int4 *>(gather.out + gpos);
                to[0] = __ldg(from);
                to[1] = __ldg(from + 1);
                gather.rank[src] = gpos;
            }
        }
    }
}

static int sort_passes(int bits) { return bits <= 0 ? 0 : (bits + SORT_BITS - 1) / SORT_BITS; }

// Scratch of a sort of n pairs, whatever the number of passes (at most
// GG_SORT_MAX_PASSES), so that one buffer serves every sort of up to n pairs.
size_t gg_sort_scratch_bytes(long long n)
{
    const long long ntiles = (n + SORT_TILE - 1) / SORT_TILE;
    size_t b = 0;
    b += (size_t)n * 8 + 256;                                // alternate keys
    b += (size_t)n * 4 + 256;                                // alternate values
    b += (size_t)GG_SORT_MAX_PASSES * RADIX * 4 * 2 + 512;   // histograms + offsets
    b += 256;                                                // tile counters
    b += 2 * ((size_t)ntiles * RADIX * 4 + 256);             // two arrays of status words
    return b;
}

static int sort_smem_bytes() { return (int)sizeof(SortSmem); }

// Sorts (keys, vals) of length n by the low key_bits bits of the key, then
// stably by the low sys_bits bits of each value's system id (the system whose
// range [poff[s], poff[s+1]) holds the value).  Scratch must be
// gg_sort_scratch_bytes(n) bytes, 256-byte aligned.  The
// result is left in keys/vals.
gg_status gg_sort_pairs_run(unsigned long long *keys, unsigned *vals, long long n, int key_bits, int sys_bits,
                            const int *poff, int S, void *scratch, int *err, cudaStream_t st,
                            const SortGather *gather, bool *gathered)
{
    if (gathered) *gathered = false;
    const int nkey = sort_passes(key_bits), nsys = sort_passes(sys_bits), np = nkey + nsys;
    if (np <= 0 || n <= 1) return GG_OK;
    if (np > GG_SORT_MAX_PASSES || n >= (1ll << 30)) return GG_ERR_TOO_LARGE;
    const long long ntiles = (n + SORT_TILE - 1) / SORT_TILE;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    unsigned long long *kalt = (unsigned long long *)take((size_t)n * 8);
    unsigned *valt = (unsigned *)take((size_t)n * 4);
    unsigned *hist = (unsigned *)take((size_t)np * RADIX * 4);
    unsigned *off = (unsigned *)take((size_t)np * RADIX * 4);
    unsigned *counters = (unsigned *)take(256);
    unsigned *status[2] = {(unsigned *)take((size_t)ntiles * RADIX * 4), (unsigned *)take((size_t)ntiles * RADIX * 4)};

    GG_CUDA_TRY(cudaMemsetAsync(hist, 0, (size_t)np * RADIX * 4, st));
    GG_CUDA_TRY(cudaMemsetAsync(counters, 0, 256, st));
    GG_CUDA_TRY(cudaMemsetAsync(status[0], 0, (size_t)ntiles * RADIX * 4, st));
    {
        int threads = 256, blocks = gg_num_sms() * 4;
        const long long need = (n + threads - 1) / threads;
        if (need < blocks) blocks = (int)need;
        const int hsmem = np * RADIX * 4;
        GG_CUDA_TRY(cudaFuncSetAttribute(k_sort_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, hsmem));
        k_sort_hist<<<blocks, threads, hsmem, st>>>(keys, vals, (int)n, nkey, nsys, poff, S, hist);
        k_sort_hist_scan<<<np, SORT_THREADS, 0, st>>>(hist, off);
        gg_note_launches(2);
    }
    // the attribute is per device: set it on every call (cheap)
    GG_CUDA_TRY(cudaFuncSetAttribute(k_sort_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sort_smem_bytes()));
    if (gather) {
        GG_CUDA_TRY(cudaFuncSetAttribute(k_sort_pass<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         sort_smem_bytes()));
    }
    const SortGather none = {nullptr, nullptr, nullptr};
    unsigned long long *ka = keys, *kb = kalt;
    unsigned *va = vals, *vb = valt;
    for (int pass = 0; pass < np; pass++) {
        const int sys_mode = pass >= nkey;
        const int shift = sys_mode ? SORT_BITS * (pass - nkey) : SORT_BITS * pass;
        if (gather && pass == np - 1)
            k_sort_pass<true><<<(unsigned)ntiles, SORT_THREADS, sort_smem_bytes(), st>>>(
                ka, va, kb, vb, (int)n, shift, sys_mode, poff, S, off + pass * RADIX, status[pass & 1], nullptr,
                counters + pass, err, *gather);
        else
            k_sort_pass<false><<<(unsigned)ntiles, SORT_THREADS, sort_smem_bytes(), st>>>(
                ka, va, kb, vb, (int)n, shift, sys_mode, poff, S, off + pass * RADIX, status[pass & 1],
                pass + 1 < np ? status[(pass + 1) & 1] : nullptr, counters + pass, err, none);
        gg_note_launches(1);
        unsigned long long *tk = ka; ka = kb; kb = tk;
        unsigned *tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        GG_CUDA_TRY(cudaMemcpyAsync(keys, ka, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
        GG_CUDA_TRY(cudaMemcpyAsync(vals, va, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    }
    if (gathered) *gathered = gather != nullptr;
    return GG_OK;
}

// Self-test of the bounded look-back: one CTA runs tile 1 of a two-tile pass
// whose tile 0 never runs, so its look-back gives up after GG_SORT_SPIN_LIMIT
// polls and records GG_EBIT_SORT_TIMEOUT.  Every access stays in bounds: the
// status words and buffers are sized for two tiles and the scatter checks
// gpos < n.  Returns GG_ERR_TIMEOUT when the limit works, GG_OK if the wait
// completed (it cannot), or a CUDA error.
gg_status gg_sort_timeout_selftest(cudaStream_t st)
{
    const int n = 2 * SORT_TILE;
    char *base = nullptr;
    const size_t bytes = (size_t)n * 24 + 2 * RADIX * 4 + RADIX * 4 + 4096;
    GG_CUDA_TRY(cudaMallocAsync((void **)&base, bytes, st));
    char *p = base;
    auto take = [&](size_t b) { char *r = p; p += (b + 255) & ~(size_t)255; return (void *)r; };
    unsigned long long *kin = (unsigned long long *)take((size_t)n * 8);
    unsigned *vin = (unsigned *)take((size_t)n * 4);
    unsigned long long *kout = (unsigned long long *)take((size_t)n * 8);
    unsigned *vout = (unsigned *)take((size_t)n * 4);
    unsigned *off = (unsigned *)take(RADIX * 4);
    unsigned *status = (unsigned *)take(2 * RADIX * 4);
    unsigned *counter = (unsigned *)take(256);
    int *err = (int *)take(256);
    cudaMemsetAsync(base, 0, (size_t)(p - base), st);
    const unsigned one = 1;   // the CTA takes tile 1; tile 0 is never started
    cudaMemcpyAsync(counter, &one, sizeof one, cudaMemcpyHostToDevice, st);
    cudaFuncSetAttribute(k_sort_pass<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sort_smem_bytes());
    const SortGather none = {nullptr, nullptr, nullptr};
    k_sort_pass<false><<<1, SORT_THREADS, sort_smem_bytes(), st>>>(kin, vin, kout, vout, n, 0, 0, nullptr, 1, off, status,
                                                             nullptr, counter, err, none);
    gg_note_launches(1);
    int herr = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(base, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gg_cuda_fail(e);
    return (herr & GG_EBIT_SORT_TIMEOUT) ? GG_ERR_TIMEOUT : GG_OK;
}
