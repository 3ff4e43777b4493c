// gg_keys.cu -- root cube per system and 63-bit Peano-Hilbert keys.
//
// domain_findExtent (domain.c:2518-2570): FP64 min/max per axis, cube side
// len = 1.001 * max extent, centre = bbox middle, corner = centre - len/2.
// Keys: domain_double_to_int (domain.c:2504-2513) at 21 bits per dimension,
// then the Peano-Hilbert key (system/peano.c:303-319).  At 21 bits the key is
// exactly the reference's 42-bit key shifted right by 63 bits, because the
// reference's key is built most-significant level first.
#include "gg_internal.cuh"
#include "gg_ph_table.h"
#include "gg_kernels.cuh"

__device__ __forceinline__ int gg_sys_of(const int *__restrict__ poff, int S, int i)
{
    // largest s with poff[s] <= i
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(poff + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_extent_init(unsigned long long *mm, unsigned *hmm, int S)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < S * 6) mm[t] = (t % 6) < 3 ? ~0ull : 0ull;   // [min x,y,z | max x,y,z] in ordered encoding
    if (hmm && t < S * 2) hmm[t] = (t & 1) ? 0u : 0x7f800000u;
}

// Each warp reduces a contiguous chunk of particles, reading it coalesced
// (lane l takes every 32nd record), one system segment at a time, and flushes
// the segment's min/max with 64-bit atomics on an order-preserving encoding:
// order-independent, so the result is exact and deterministic.  The per-system
// range of kernel radii (positive floats, ordered as their bit patterns) goes
// to hmm[2s], hmm[2s+1].
#define EXTENT_CHUNK 4096
__global__ void k_extent(const GGPart *__restrict__ rec, int n, const int *__restrict__ poff, int S,
                         unsigned long long *mm, unsigned *hmm, int *err)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    bool bad = false;
    for (long long c0 = (long long)warp * EXTENT_CHUNK; c0 < n; c0 += (long long)nwarps * EXTENT_CHUNK) {
        const int cb = (int)c0, ce = (int)min((long long)n, c0 + EXTENT_CHUNK);
        int s = gg_sys_of(poff, S, cb);
        for (int seg = cb; seg < ce; s++) {
            const int se = min(ce, __ldg(poff + s + 1));
            double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
            float hmin = INFINITY, hmax = 0.f;
            for (int i = seg + lane; i < se; i += 32) {
                GGPart p = rec[i];
                double v[3] = {p.x, p.y, p.z};
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    if (!isfinite(v[k])) bad = true;
                    mn[k] = fmin(mn[k], v[k]);
                    mx[k] = fmax(mx[k], v[k]);
                }
                hmin = fminf(hmin, p.h);
                hmax = fmaxf(hmax, p.h);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    mn[k] = fmin(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
                    mx[k] = fmax(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
                }
                hmin = fminf(hmin, __shfl_xor_sync(0xffffffffu, hmin, o));
                hmax = fmaxf(hmax, __shfl_xor_sync(0xffffffffu, hmax, o));
            }
            if (lane == 0 && se > seg) {
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    atomicMin(&mm[s * 6 + k], gg_dbl_to_ordered(mn[k]));
                    atomicMax(&mm[s * 6 + 3 + k], gg_dbl_to_ordered(mx[k]));
                }
                if (hmm) {
                    atomicMin(&hmm[2 * s], __float_as_uint(fmaxf(hmin, 0.f)));
                    atomicMax(&hmm[2 * s + 1], __float_as_uint(fmaxf(hmax, 0.f)));
                }
            }
            seg = se;
        }
    }
    if (bad) atomicOr(err, GG_EBIT_BAD_INPUT);
}

__global__ void k_extent_finalize(const unsigned long long *mm, int S, GGDomainDev *dom)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    double mn[3], mx[3], len = 0;
    for (int k = 0; k < 3; k++) {
        mn[k] = gg_ordered_to_dbl(mm[s * 6 + k]);
        mx[k] = gg_ordered_to_dbl(mm[s * 6 + 3 + k]);
        if (!(mn[k] <= mx[k])) { mn[k] = 0; mx[k] = 0; }   // empty system
    }
    for (int k = 0; k < 3; k++) {
        double e = __dsub_rn(mx[k], mn[k]);
        if (e > len) len = e;
    }
    len = __dmul_rn(len, 1.001);
    if (len <= 0) len = 1.0;   // a single particle or empty system: any cube works
    GGDomainDev d;
    for (int k = 0; k < 3; k++) {
        double mid = __dmul_rn(0.5, __dadd_rn(mn[k], mx[k]));
        d.center[k] = mid;
        d.corner[k] = __dsub_rn(mid, __dmul_rn(0.5, len));
    }
    d.len = len;
    d.pad = 0;
    dom[s] = d;
}

// 21 levels: the top one from the one-level table, then ten steps of two
// levels each from the two-level table (half the dependent table reads)
__device__ __forceinline__ unsigned long long gg_ph_key21(unsigned x, unsigned y, unsigned z,
                                                          const unsigned short *tab, const unsigned short *tab2)
{
    const int top = GG_MAX_LEVEL - 1;
    unsigned pix = (((x >> top) & 1u) << 2) | (((y >> top) & 1u) << 1) | ((z >> top) & 1u);
    unsigned e = tab[pix];   // state 0
    unsigned long long key = e & 7u;
    unsigned state = e >> 3;
#pragma unroll
    for (int lev = top - 1; lev > 0; lev -= 2) {
        const unsigned hi = (((x >> lev) & 1u) << 2) | (((y >> lev) & 1u) << 1) | ((z >> lev) & 1u);
        const unsigned lo = (((x >> (lev - 1)) & 1u) << 2) | (((y >> (lev - 1)) & 1u) << 1) | ((z >> (lev - 1)) & 1u);
        e = tab2[state * 64 + ((hi << 3) | lo)];
        key = (key << 6) | (e & 63u);
        state = e >> 6;
    }
    return key;
}

// keys + identity values for the sort; positions must lie in [corner, corner+len)
__global__ void k_keys(const GGPart *__restrict__ rec, int n, const int *__restrict__ poff, int S,
                       const GGDomainDev *__restrict__ dom, unsigned long long *keys, unsigned *vals, int *err)
{
    __shared__ unsigned short tab[GG_PH_NSTATES * 8], tab2[GG_PH_NSTATES * 64];
    for (int i = threadIdx.x; i < GG_PH_NSTATES * 8; i += blockDim.x) tab[i] = GG_PH_TABLE_INIT[i];
    for (int i = threadIdx.x; i < GG_PH_NSTATES * 64; i += blockDim.x) tab2[i] = GG_PH_TABLE2_INIT[i];
    __syncthreads();
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int s = (S == 1) ? 0 : gg_sys_of(poff, S, i);
        GGDomainDev d = dom[s];
        GGPart p = rec[i];
        double v[3] = {p.x, p.y, p.z};
        unsigned q[3];
        for (int k = 0; k < 3; k++) {
            double f = __dadd_rn(__ddiv_rn(__dsub_rn(v[k], d.corner[k]), d.len), 1.0);
            if (!(f >= 1.0 && f < 2.0)) { bad = true; f = fmin(fmax(f, 1.0), 1.9999999999999998); }
            unsigned long long u = (unsigned long long)__double_as_longlong(f);
            q[k] = (unsigned)((u & 0xFFFFFFFFFFFFFull) >> (52 - GG_MAX_LEVEL));
        }
        keys[i] = gg_ph_key21(q[0], q[1], q[2], tab, tab2);
        vals[i] = (unsigned)i;
    }
    if (bad) atomicOr(err, GG_EBIT_BAD_INPUT);
}

// keys of plain (n x 3) FP64 positions in one cube: the kernel-level entry point
__global__ void k_keys_plain(const double *__restrict__ pos, long long n, GGDomainDev d, unsigned long long *keys,
                             int *err)
{
    __shared__ unsigned short tab[GG_PH_NSTATES * 8], tab2[GG_PH_NSTATES * 64];
    for (int i = threadIdx.x; i < GG_PH_NSTATES * 8; i += blockDim.x) tab[i] = GG_PH_TABLE_INIT[i];
    for (int i = threadIdx.x; i < GG_PH_NSTATES * 64; i += blockDim.x) tab2[i] = GG_PH_TABLE2_INIT[i];
    __syncthreads();
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        unsigned q[3];
        for (int k = 0; k < 3; k++) {
            double f = __dadd_rn(__ddiv_rn(__dsub_rn(pos[3 * i + k], d.corner[k]), d.len), 1.0);
            if (!(f >= 1.0 && f < 2.0)) { bad = true; f = fmin(fmax(f, 1.0), 1.9999999999999998); }
            unsigned long long u = (unsigned long long)__double_as_longlong(f);
            q[k] = (unsigned)((u & 0xFFFFFFFFFFFFFull) >> (52 - GG_MAX_LEVEL));
        }
        keys[i] = gg_ph_key21(q[0], q[1], q[2], tab, tab2);
    }
    if (bad && err) atomicOr(err, GG_EBIT_BAD_INPUT);
}

void gg_launch_extent(const GGPart *rec, int n, const int *poff, int S, unsigned long long *mm, unsigned *hmm,
                      GGDomainDev *dom, int *err, cudaStream_t st)
{
    k_extent_init<<<(S * 6 + 255) / 256, 256, 0, st>>>(mm, hmm, S);
    int threads = 256, blocks = gg_num_sms() * 4;
    long long chunks = ((long long)n + EXTENT_CHUNK - 1) / EXTENT_CHUNK;
    if ((long long)blocks * (threads / 32) > chunks) blocks = (int)((chunks + (threads / 32) - 1) / (threads / 32));
    if (blocks < 1) blocks = 1;
    k_extent<<<blocks, threads, 0, st>>>(rec, n, poff, S, mm, hmm, err);
    k_extent_finalize<<<(S + 127) / 128, 128, 0, st>>>(mm, S, dom);
    gg_note_launches(3);
}

void gg_launch_keys(const GGPart *rec, int n, const int *poff, int S, const GGDomainDev *dom,
                    unsigned long long *keys, unsigned *vals, int *err, cudaStream_t st)
{
    int threads = 256, blocks = gg_num_sms() * 8;
    if ((long long)blocks * threads > n) blocks = (n + threads - 1) / threads;
    if (blocks < 1) blocks = 1;
    k_keys<<<blocks, threads, 0, st>>>(rec, n, poff, S, dom, keys, vals, err);
    gg_note_launches(1);
}

void gg_launch_keys_plain(const double *pos, long long n, const GGDomainDev &d, unsigned long long *keys, int *err,
                          cudaStream_t st)
{
    int threads = 256;
    long long b = (n + threads - 1) / threads;
    int blocks = (int)(b < gg_num_sms() * 8 ? (b < 1 ? 1 : b) : gg_num_sms() * 8);
    k_keys_plain<<<blocks, threads, 0, st>>>(pos, n, d, keys, err);
    gg_note_launches(1);
}
