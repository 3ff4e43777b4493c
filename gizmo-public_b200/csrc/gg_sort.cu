// gg_sort.cu -- stable LSD radix sort of (64-bit key, 32-bit value) pairs.
//
// Replaces the reference's stable mergesort of {peanokey, index} records
// (mysort_peano, system/peano.c:414-462; mysort_domain, domain.c:2674-2723).
// Design (one-sweep): one up-front pass builds the digit histograms of every
// pass; each pass is then a single kernel in which a CTA ranks a 2048-key tile
// in shared memory, publishes its per-digit counts, sums its predecessors'
// counts with a decoupled look-back, and writes the tile out digit-sorted so
// that global stores are contiguous runs.  8-bit digits.  For several systems
// a second set of passes sorts stably by system id (taken from the value, an
// index into the concatenated particle array), so the final order is
// (system, key).
//
// Every wait in the look-back is bounded: after GG_SORT_SPIN_LIMIT polls the
// CTA records GG_EBIT_SORT_TIMEOUT in the error word and carries on, so a
// failure returns an error instead of hanging the device.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define SORT_THREADS 256
#define SORT_ITEMS 8      // 2048-key tiles: 4 blocks of 8 warps fit an SM (registers and shared memory)
#define SORT_TILE (SORT_THREADS * SORT_ITEMS)
#define SORT_WARPS (SORT_THREADS / 32)
#define RADIX 256
#define ST_AGG (1u << 30)
#define ST_INC (2u << 30)
#define ST_FLAGS (3u << 30)
#define ST_VALUE 0x3FFFFFFFu
#define GG_SORT_SPIN_LIMIT (1 << 22)

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
    __shared__ unsigned sh[GG_SORT_MAX_PASSES * RADIX];
    int np = nkey + nsys;
    for (int i = threadIdx.x; i < np * RADIX; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        unsigned long long k = keys[i];
        for (int p = 0; p < nkey; p++) atomicAdd(&sh[p * RADIX + ((k >> (8 * p)) & 255)], 1u);
        if (nsys) {
            unsigned s = (unsigned)sort_sys_of(poff, S, vals[i]);
            for (int p = 0; p < nsys; p++) atomicAdd(&sh[(nkey + p) * RADIX + ((s >> (8 * p)) & 255)], 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np * RADIX; i += blockDim.x)
        if (sh[i]) atomicAdd(&g_hist[i], sh[i]);
}

// exclusive scan of each pass's 256 counts (one block per pass, 256 threads)
__global__ void k_sort_hist_scan(const unsigned *g_hist, unsigned *g_off)
{
    __shared__ unsigned ws[8];
    int p = blockIdx.x, d = threadIdx.x, lane = d & 31, w = d >> 5;
    unsigned v = g_hist[p * RADIX + d], x = v;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned t = lane < 8 ? ws[lane] : 0, u = t;
        for (int o = 1; o < 8; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, u, o);
            if (lane >= o) u += y;
        }
        if (lane < 8) ws[lane] = u - t;
    }
    __syncthreads();
    g_off[p * RADIX + d] = x - v + ws[w];
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

// one pass: digit = (key >> shift) & 255, or (system id >> shift) & 255 when sys_mode
__global__ void __launch_bounds__(SORT_THREADS, 4) k_sort_pass(
    const unsigned long long *__restrict__ kin, const unsigned *__restrict__ vin, unsigned long long *__restrict__ kout,
    unsigned *__restrict__ vout, int n, int shift, int sys_mode, const int *__restrict__ poff, int S,
    const unsigned *__restrict__ g_off, unsigned *status, unsigned *tile_counter, int *err)
{
    extern __shared__ unsigned long long s_keys[];             // SORT_TILE keys
    unsigned *s_vals = (unsigned *)(s_keys + SORT_TILE);       // SORT_TILE values
    unsigned char *s_dig = (unsigned char *)(s_vals + SORT_TILE);  // SORT_TILE digits
    __shared__ unsigned s_whist[SORT_WARPS][RADIX];
    __shared__ unsigned s_texcl[RADIX];
    __shared__ unsigned s_gbase[RADIX];
    __shared__ unsigned s_wsum[SORT_WARPS];
    __shared__ int s_tile;

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) s_tile = (int)atomicAdd(tile_counter, 1u);
    for (int i = tid; i < SORT_WARPS * RADIX; i += SORT_THREADS) (&s_whist[0][0])[i] = 0;
    __syncthreads();
    const int tile = s_tile;
    const long long tile_base = (long long)tile * SORT_TILE;
    const long long wbase = tile_base + (long long)w * 32 * SORT_ITEMS;
    const unsigned lt_mask = (1u << lane) - 1u;

    unsigned long long k[SORT_ITEMS];
    unsigned v[SORT_ITEMS], rank[SORT_ITEMS], dg[SORT_ITEMS];
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        long long idx = wbase + j * 32 + lane;
        bool valid = idx < n;
        k[j] = valid ? kin[idx] : ~0ull;
        v[j] = valid ? vin[idx] : 0u;
    }
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        long long idx = wbase + j * 32 + lane;
        unsigned d;
        if (idx >= n) d = 255u;
        else if (sys_mode) d = ((unsigned)sort_sys_of(poff, S, v[j]) >> shift) & 255u;
        else d = (unsigned)(k[j] >> shift) & 255u;
        dg[j] = d;
    }
    // stable warp-level ranking in (item, lane) order == index order
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        unsigned d = dg[j];
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int leader = __ffs(peers) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(&s_whist[w][d], (unsigned)__popc(peers));
        base = __shfl_sync(peers, base, leader);
        rank[j] = base + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();

    // per digit: warp-exclusive offsets and the tile's count
    const int d = tid;   // SORT_THREADS == RADIX
    unsigned sum = 0;
#pragma unroll
    for (int ww = 0; ww < SORT_WARPS; ww++) {
        unsigned c = s_whist[ww][d];
        s_whist[ww][d] = sum;
        sum += c;
    }
    // publish and look back
    unsigned *st = status + (size_t)tile * RADIX;
    unsigned excl = 0;
    if (tile == 0) {
        st_status(&st[d], ST_INC | (sum & ST_VALUE));
    } else {
        st_status(&st[d], ST_AGG | (sum & ST_VALUE));
        int t = tile - 1;
        int spins = 0;
        while (t >= 0) {
            unsigned sv = ld_status(status + (size_t)t * RADIX + d);
            if ((sv & ST_FLAGS) == 0u) {
                if (++spins > GG_SORT_SPIN_LIMIT) {
                    atomicOr(err, GG_EBIT_SORT_TIMEOUT);
                    break;
                }
                __nanosleep(32);
                continue;
            }
            excl += sv & ST_VALUE;
            if ((sv & ST_FLAGS) == ST_INC) break;
            t--;
        }
        st_status(&st[d], ST_INC | ((excl + sum) & ST_VALUE));
    }
    s_gbase[d] = g_off[d] + excl;

    // exclusive scan of the tile's digit counts
    unsigned x = sum;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[w] = x;
    __syncthreads();
    unsigned wo = 0;
    for (int ww = 0; ww < w; ww++) wo += s_wsum[ww];
    s_texcl[d] = x - sum + wo;
    __syncthreads();

    // scatter into shared memory in digit order
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        long long idx = wbase + j * 32 + lane;
        if (idx < n) {
            unsigned dd = dg[j];
            unsigned pos = s_texcl[dd] + s_whist[w][dd] + rank[j];
            s_keys[pos] = k[j];
            s_vals[pos] = v[j];
            s_dig[pos] = (unsigned char)dd;
        }
    }
    __syncthreads();
    long long rem = (long long)n - tile_base;
    int nvalid = rem < SORT_TILE ? (int)rem : SORT_TILE;
    for (int i = tid; i < nvalid; i += SORT_THREADS) {
        unsigned dd = s_dig[i];
        unsigned gpos = s_gbase[dd] + (unsigned)i - s_texcl[dd];
        if (gpos < (unsigned)n) {   // always true unless a look-back gave up
            kout[gpos] = s_keys[i];
            vout[gpos] = s_vals[i];
        }
    }
}

size_t gg_sort_scratch_bytes(long long n, int npasses)
{
    long long ntiles = (n + SORT_TILE - 1) / SORT_TILE;
    size_t b = 0;
    b += (size_t)n * 8 + 256;                                // alternate keys
    b += (size_t)n * 4 + 256;                                // alternate values
    b += (size_t)npasses * RADIX * 4 * 2;                    // histograms + offsets
    b += 256;                                                // tile counters
    b += (size_t)npasses * ntiles * RADIX * 4 + 256;         // status words
    return b;
}

static int sort_smem_bytes() { return SORT_TILE * (8 + 4 + 1); }

// Sorts (keys, vals) of length n.  nkey key passes (8 bits each, from bit 0),
// then nsys system-id passes.  Scratch must be gg_sort_scratch_bytes(n, nkey+nsys)
// bytes, 256-byte aligned.  The result is left in keys/vals.
gg_status gg_sort_pairs_run(unsigned long long *keys, unsigned *vals, long long n, int nkey, int nsys,
                            const int *poff, int S, void *scratch, int *err, cudaStream_t st)
{
    int np = nkey + nsys;
    if (np <= 0 || n <= 1) return GG_OK;
    if (np > GG_SORT_MAX_PASSES || n >= (1ll << 30)) return GG_ERR_TOO_LARGE;
    long long ntiles = (n + SORT_TILE - 1) / SORT_TILE;
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
    unsigned *status = (unsigned *)take((size_t)np * ntiles * RADIX * 4);

    GG_CUDA_TRY(cudaMemsetAsync(hist, 0, (size_t)np * RADIX * 4, st));
    GG_CUDA_TRY(cudaMemsetAsync(counters, 0, 256, st));
    GG_CUDA_TRY(cudaMemsetAsync(status, 0, (size_t)np * ntiles * RADIX * 4, st));
    {
        int threads = 256, blocks = gg_num_sms() * 4;
        long long need = (n + threads - 1) / threads;
        if (need < blocks) blocks = (int)need;
        k_sort_hist<<<blocks, threads, 0, st>>>(keys, vals, (int)n, nkey, nsys, poff, S, hist);
        k_sort_hist_scan<<<np, RADIX, 0, st>>>(hist, off);
        gg_note_launches(2);
    }
    static bool attr_set = false;
    if (!attr_set) {
        GG_CUDA_TRY(cudaFuncSetAttribute(k_sort_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, sort_smem_bytes()));
        attr_set = true;
    }
    unsigned long long *ka = keys, *kb = kalt;
    unsigned *va = vals, *vb = valt;
    for (int pass = 0; pass < np; pass++) {
        int sys_mode = pass >= nkey;
        int shift = sys_mode ? 8 * (pass - nkey) : 8 * pass;
        k_sort_pass<<<(unsigned)ntiles, SORT_THREADS, sort_smem_bytes(), st>>>(
            ka, va, kb, vb, (int)n, shift, sys_mode, poff, S, off + pass * RADIX, status + (size_t)pass * ntiles * RADIX,
            counters + pass, err);
        gg_note_launches(1);
        unsigned long long *tk = ka; ka = kb; kb = tk;
        unsigned *tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        GG_CUDA_TRY(cudaMemcpyAsync(keys, ka, (size_t)n * 8, cudaMemcpyDeviceToDevice, st));
        GG_CUDA_TRY(cudaMemcpyAsync(vals, va, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
    }
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
    const size_t bytes = gg_sort_scratch_bytes(n, 1);
    char *base = nullptr;
    GG_CUDA_TRY(cudaMallocAsync((void **)&base, bytes + 4 * (size_t)n * 12 + 1024, st));
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
    static bool attr_set = false;
    if (!attr_set) {
        cudaFuncSetAttribute(k_sort_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, sort_smem_bytes());
        attr_set = true;
    }
    k_sort_pass<<<1, SORT_THREADS, sort_smem_bytes(), st>>>(kin, vin, kout, vout, n, 0, 0, nullptr, 1, off, status,
                                                             counter, err);
    gg_note_launches(1);
    int herr = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(base, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return gg_cuda_fail(e);
    return (herr & GG_EBIT_SORT_TIMEOUT) ? GG_ERR_TIMEOUT : GG_OK;
}
