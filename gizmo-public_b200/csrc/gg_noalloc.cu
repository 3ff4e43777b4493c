// gg_noalloc.cu -- the radix sort of (key, value) pairs without any device allocation.
//
// gg_radix_sort_pairs allocates its scratch (alternate key/value buffers,
// digit histograms, look-back status words) with cudaMallocAsync on every call.
// Some callers cannot do that: a process whose device memory is already
// reserved in full by another allocator (a framework's caching allocator, or
// a serving loop that admits work against a fixed device-memory budget) gets
// an out-of-memory error or breaks its own accounting, and a latency-critical
// loop cannot afford the implicit device synchronisation of cudaFree.  This
// variant takes its scratch from one file-scope __device__ array instead.
//
// The array holds at most GG_NOALLOC_SORT_MAX_N pairs' scratch; every GPU that
// loads this library keeps it (about 20 MB) until the process exits.  All
// calls share it and it keeps the previous call's contents: the call clears
// what must start at zero (histograms, tile counters, status words, error
// word).  Two calls whose work overlaps on the GPU (on different streams, or
// from different host threads) race on the array and must not be issued.
#include <mutex>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

// scratch of gg_sort_pairs_run for GG_NOALLOC_SORT_MAX_N pairs (12.6 MB for
// the alternate keys and values, about 1 MB of look-back status words), plus
// the error word in the last 256 bytes; the entry point checks the fit
#define GG_NOALLOC_SCRATCH_BYTES (20u << 20)

static __device__ __align__(256) unsigned char gg_noalloc_scratch[GG_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64];

// Device address of the array on the current device.  In host code the
// symbol name is only a host-side stand-in; the address is looked up once per
// device, with that device current, on the first call there, and kept for the
// life of the process.  A cudaDeviceReset by the application ends the
// context the address belongs to: after one, this entry point must not be
// called again in the same process.
static gg_status noalloc_scratch(void **out)
{
    int dev = 0;
    GG_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return GG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, gg_noalloc_scratch);
        if (e != cudaSuccess || !p) return gg_cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e);
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return GG_OK;
}

extern "C" gg_status gg_radix_sort_pairs_noalloc(int64_t n, uint64_t *d_keys, uint32_t *d_vals, int32_t key_bits,
                                                 void *stream)
{
    if (n < 0 || key_bits < 1 || key_bits > 64 || (n && (!d_keys || !d_vals))) return GG_ERR_INVALID;
    if (n > GG_NOALLOC_SORT_MAX_N) return GG_ERR_TOO_LARGE;
    if (n <= 1) return GG_OK;
    if (gg_sort_scratch_bytes(n) + 256 > GG_NOALLOC_SCRATCH_BYTES) return GG_ERR_TOO_LARGE;
    // the pairs must be device memory of the current device, where the array is
    int dev = 0;
    GG_CUDA_TRY(cudaGetDevice(&dev));
    for (const void *ptr : {(const void *)d_keys, (const void *)d_vals}) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
            cudaGetLastError();
            return GG_ERR_INVALID;
        }
        if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != dev)
            return GG_ERR_INVALID;
    }
    void *scratch = nullptr;
    gg_status st = noalloc_scratch(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    int *err = (int *)((char *)scratch + GG_NOALLOC_SCRATCH_BYTES - 256);
    GG_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
    st = gg_sort_pairs_run((unsigned long long *)d_keys, d_vals, n, key_bits, 0, nullptr, 1, scratch, err, s);
    if (st) return st;
    int herr = 0;
    GG_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    GG_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr & GG_EBIT_SORT_TIMEOUT) return GG_ERR_TIMEOUT;
    return GG_OK;
}
