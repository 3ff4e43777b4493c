// gg_api.cu -- the C ABI: context, device memory, and the build/walk pipeline.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <omp.h>
#include <atomic>
#include <iterator>
#include <map>
#include <mutex>
#include <cmath>
#include <vector>

#include "gg_internal.cuh"
#include "gg_kernels.cuh"

#define GG_STACK_CAP 8192                 // default walk-stack entries per warp in device memory
static const int kStackMax = 1 << 17;     // largest a retry grows them to

static thread_local char g_last_cuda_error[256];

gg_status gg_cuda_fail(cudaError_t e)
{
    snprintf(g_last_cuda_error, sizeof g_last_cuda_error, "%s", cudaGetErrorString(e));
    cudaGetLastError();   // clear a sticky launch error where possible
    return e == cudaErrorMemoryAllocation ? GG_ERR_NOMEM : GG_ERR_CUDA;
}

static std::atomic<long long> g_launches{0};
void gg_note_launches(int k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
extern "C" int64_t gg_kernel_launches(void) { return (int64_t)g_launches.load(); }

int gg_num_sms()
{
    static int cached[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!cached[dev]) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = v > 0 ? v : 148;
    }
    return cached[dev];
}

// Device buffers are allocated in stream order on the context's stream
// (cudaMallocAsync / cudaFreeAsync from the device's default pool, which keeps
// freed memory cached), so creating, growing or destroying a context never
// waits for the whole device.  Contents are not kept across a growth.
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    const cudaStream_t *sref = nullptr;   // the owning context's current stream
    long long *gen = nullptr;              // the owning context's count of buffer moves
    gg_status ensure(size_t n)
    {
        if (n <= cap && p) return GG_OK;
        if (gen) ++*gen;   // a captured graph holding the old address is stale from here on
        const cudaStream_t s = sref ? *sref : (cudaStream_t)0;
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
        cap = 0;
        size_t want = n < 1 ? 1 : n;
        cudaError_t e = cudaMallocAsync((void **)&p, want * sizeof(T), s);
        if (e != cudaSuccess) { p = nullptr; return gg_cuda_fail(e); }
        cap = want;
        return GG_OK;
    }
    void release()
    {
        if (p) cudaFreeAsync(p, sref ? *sref : (cudaStream_t)0);
        p = nullptr;
        cap = 0;
    }
};

// Pinned host blocks shared by every context of the process: host staging of
// particle loads, active lists and results is borrowed for the duration of a
// transfer and given back, so a new context does not page-lock memory again.
// Blocks come in power-of-two sizes from 1 MB, so that a block given back
// serves any later request of its size class; they are kept for reuse up to
// kPinnedCacheBytes in total.
static const size_t kPinnedCacheBytes = (size_t)16 << 30;
static std::mutex g_pinned_mu;
static std::multimap<size_t, void *> g_pinned_free;
static size_t g_pinned_cached = 0;

static size_t pinned_class(size_t bytes)
{
    size_t c = (size_t)1 << 20;
    while (c < bytes) c <<= 1;
    return c;
}

static void *pinned_get(size_t bytes, size_t *got)
{
    const size_t want = pinned_class(bytes);
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        auto it = g_pinned_free.find(want);
        if (it != g_pinned_free.end()) {
            void *p = it->second;
            *got = it->first;
            g_pinned_cached -= it->first;
            g_pinned_free.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, want, cudaHostAllocPortable) != cudaSuccess) return nullptr;
    *got = want;
    return p;
}

static void pinned_put(void *p, size_t bytes)
{
    if (!p) return;
    std::vector<void *> drop;
    {
        std::lock_guard<std::mutex> lk(g_pinned_mu);
        g_pinned_free.emplace(bytes, p);
        g_pinned_cached += bytes;
        while (g_pinned_cached > kPinnedCacheBytes && !g_pinned_free.empty()) {
            auto it = std::prev(g_pinned_free.end());
            g_pinned_cached -= it->first;
            drop.push_back(it->second);
            g_pinned_free.erase(it);
        }
    }
    for (void *q : drop) cudaFreeHost(q);
}

// A pinned host buffer borrowed from the pool; `guard` is the event recorded
// after the last transfer that reads or writes it.
template <typename T>
struct HostBuf {
    T *p = nullptr;
    size_t cap = 0, bytes = 0;
    gg_status ensure(size_t n, cudaEvent_t guard)
    {
        if (n <= cap && p) {
            GG_CUDA_TRY(cudaEventSynchronize(guard));   // may still feed the previous transfer
            return GG_OK;
        }
        give_back(guard);
        size_t want = n < 1 ? 1 : n;
        p = (T *)pinned_get(want * sizeof(T), &bytes);
        if (!p) { bytes = 0; return GG_ERR_NOMEM; }
        cap = bytes / sizeof(T);
        return GG_OK;
    }
    void give_back(cudaEvent_t guard)
    {
        if (!p) return;
        if (guard) cudaEventSynchronize(guard);
        pinned_put(p, bytes);
        p = nullptr;
        cap = bytes = 0;
    }
};

// host copy spread over the OpenMP threads (results of large batches run to
// hundreds of MB): pieces of at least 256 KB, about four per thread, so that
// a pipelined chunk of a few MB keeps every thread busy and the copy keeps
// pace with the link
static void parallel_copy(void *dst, const void *src, size_t bytes)
{
    const size_t per = bytes / (4 * (size_t)std::max(1, omp_get_max_threads()));
    const size_t chunk = std::max((size_t)256 << 10, (per + 4095) & ~(size_t)4095);
    const long long nchunks = (long long)((bytes + chunk - 1) / chunk);
    if (nchunks <= 1) { memcpy(dst, src, bytes); return; }
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < nchunks; k++) {
        const size_t off = (size_t)k * chunk, len = std::min(chunk, bytes - off);
        memcpy((char *)dst + off, (const char *)src + off, len);
    }
}

// Host transfers of large arrays are cut into chunks of this many particles:
// the host gathers or copies one chunk while the previous one crosses the link
// (small chunks keep the pipeline's fill and drain short).
static const long long kPipeChunk = 1ll << 18;
static const int kPipeEvents = 64;

struct gg_ctx {
    gg_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr, own_stream = nullptr;
    // systems
    int S = 0;
    long long N = 0;
    std::vector<int> h_poff;
    bool built = false;
    // particles
    DevBuf<int> poff;
    DevBuf<GGPart> in_rec, part;
    DevBuf<GGDomainDev> dom;
    DevBuf<unsigned long long> extent_mm;
    DevBuf<unsigned> hmm;          // per system [min h, max h] as float bits
    bool h_mixed = false;          // some system holds several kernel radii: group targets by softening
    // gg_load_particles_device: the per-system kernel-radius range crosses to
    // pinned memory behind the extent pass; the first walk reads it (hmm_ev)
    bool h_mixed_pending = false;
    HostBuf<unsigned> h_hmm;
    cudaEvent_t hmm_ev = nullptr;
    int order_by_softening = 1;    // from gg_config.target_order
    DevBuf<unsigned long long> tkey;
    DevBuf<unsigned> tval;
    DevBuf<int> tlist2, tout2;
    DevBuf<unsigned long long> keys;
    DevBuf<unsigned> perm, rank;
    DevBuf<char> sort_scratch;
    // tree
    int ncap = 0;
    DevBuf<int> t_start, t_end, t_level, t_parent, t_sys, t_nch, t_child, t_bnd, t_depth, t_nnodes;
    DevBuf<unsigned> t_bstat, t_ticket;
    DevBuf<double> t_mass64;
    DevBuf<GGNode> nodes;
    // walk
    DevBuf<double> oldacc;
    // drift of the resident tree (force_drift_node): velocities in load order,
    // node kinematics {vs, vmax} of the current build, per-system steps
    DevBuf<double> vel;
    DevBuf<double> newpos;                // gg_set_positions: the caller's positions, load order
    bool have_vel = false;
    DevBuf<double4> kin;
    DevBuf<int> kin_counter;
    bool kin_valid = false;
    bool kin_any = false;                  // kinematics computed at least once for this build
    DevBuf<double> dts;
    HostBuf<double> h_vstage;
    DevBuf<double> oldacc_save;           // autotuner: every trial starts from the same OldAcc
    DevBuf<int4> e_chunks;                // energy checks: chunk descriptors, partials, results
    DevBuf<int> e_first;
    DevBuf<double> e_part, e_out;
    bool oldacc_valid = false;
    // group order by measured cost: per target (load order) the previous walk's
    // group cycles per target, and the sorted group order
    DevBuf<float> tcost;
    bool tcost_valid = false;
    DevBuf<unsigned long long> gkey;
    DevBuf<unsigned> gorder;
    DevBuf<GGGroup> groups;
    DevBuf<int> ngroups, gscan, toff, flag, flagscan, tlist, tout, scan_scratch, active_d;
    DevBuf<int> g_node, g_flag, g_seg, g_segstart;   // group building scratch
    DevBuf<int> counters;                  // [0] group counter
    DevBuf<unsigned long long> inter;      // interaction total
    DevBuf<int> stack;
    DevBuf<int> err;
    DevBuf<double> acc_d, pot_d;
    // autotuner accuracy gate: sampled targets, their FP64 direct sums and a
    // configuration's outputs gathered at them
    DevBuf<int2> tune_tg, tune_rows;
    DevBuf<double> tune_acc, tune_pot, tune_mass, tune_gacc, tune_gpot;
    DevBuf<int> nint_d;
    int walk_blocks = 0;
    int stack_cap = 0;                    // walk-stack entries per warp in device memory
    int tune_tried = 0, tune_refused = 0;   // the last gg_autotune: trials, and trials the accuracy gate refused
    // host staging
    HostBuf<GGPart> h_stage;
    // timing
    cudaEvent_t ev[8];
    // a captured step (build + walk) replayed as one CUDA graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_launches = 0;               // kernels inside the captured step
    // the same step captured as two graphs (0: build, 1: walk)
    cudaGraph_t part_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t part_exec[2] = {nullptr, nullptr};
    int part_launches[2] = {0, 0};
    // device buffers move when they grow: graphs captured before a move are refused
    long long buf_gen = 0, graph_gen = -1, part_gen = -1;
    bool have_events = false;
    // host staging copies in flight: the next reuse of a staging buffer waits
    // for its own copy only
    cudaEvent_t stage_ev = nullptr, vstage_ev = nullptr;
    // asynchronous evaluation: staged active list, pinned results, completion
    HostBuf<int> h_active, h_nint;
    HostBuf<double> h_acc, h_pot, h_old;
    long long async_n = 0;
    int async_flags = 0;
    bool async_pinned = false;             // the last async walk copied into the caller's pinned arrays
    cudaEvent_t act_ev = nullptr, done_ev = nullptr;
    // host OldAcc of gg_evaluate crosses the link on its own stream into its
    // own array, while the build runs; the walk waits for it (old_ready_ev) and
    // the next upload waits for that walk (old_used_ev)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t old_ready_ev = nullptr, old_used_ev = nullptr;
    DevBuf<double> oldacc_in;
    cudaEvent_t pipe_ev[kPipeEvents] = {};   // completion of each chunk of a pipelined copy to the host
    gg_stats last;

    // every device buffer of the context, for release and accounting
    template <class F> void for_each_buf(F f)
    {
        f(poff); f(in_rec); f(part); f(dom); f(extent_mm); f(hmm); f(tkey); f(tval); f(tlist2); f(tout2);
        f(keys); f(perm); f(rank); f(sort_scratch);
        f(t_start); f(t_end); f(t_level); f(t_parent); f(t_sys); f(t_nch); f(t_child); f(t_bnd);
        f(t_depth); f(t_nnodes); f(t_bstat); f(t_ticket); f(t_mass64); f(nodes);
        f(oldacc); f(vel); f(newpos); f(kin); f(kin_counter); f(dts); f(oldacc_save); f(tcost); f(gkey); f(gorder);
        f(e_chunks); f(e_first); f(e_part); f(e_out);
        f(groups); f(ngroups); f(gscan); f(toff); f(flag); f(flagscan); f(tlist); f(tout); f(scan_scratch);
        f(g_node); f(g_flag); f(g_seg); f(g_segstart);
        f(active_d); f(counters); f(inter); f(stack); f(err); f(acc_d); f(pot_d); f(nint_d); f(oldacc_in);
        f(tune_tg); f(tune_rows); f(tune_acc); f(tune_pot); f(tune_mass); f(tune_gacc); f(tune_gpot);
    }
};

struct ReleaseBuf {
    template <class B> void operator()(B &b) const { b.release(); }
};
struct CountBuf {
    long long *total;
    template <class B> void operator()(B &b) const { *total += (long long)(b.cap * sizeof(*b.p)); }
};

static gg_status set_device(gg_ctx *c)
{
    GG_CUDA_TRY(cudaSetDevice(c->device));
    return GG_OK;
}

extern "C" void gg_config_default(gg_config *cfg)
{
    memset(cfg, 0, sizeof *cfg);
    cfg->device = 0;
    cfg->leaf_size = 8;
    cfg->group_size = 32;
    cfg->flush_threshold = 128;
    cfg->walk_blocks_per_sm = 0;
    cfg->timing = 0;
    cfg->target_order = 1;
    cfg->group_order = 1;
    cfg->node_staging = 0;
    cfg->walk_stack_entries = 0;
}

extern "C" const char *gg_strerror(gg_status s)
{
    switch (s) {
    case GG_PENDING: return "pending";
    case GG_OK: return "ok";
    case GG_ERR_INVALID: return "invalid argument";
    case GG_ERR_CUDA: return g_last_cuda_error[0] ? g_last_cuda_error : "CUDA error";
    case GG_ERR_NOMEM: return "device allocation failed";
    case GG_ERR_OVERFLOW: return "node pool or walk stack overflow";
    case GG_ERR_TIMEOUT: return "bounded device wait gave up";
    case GG_ERR_NOT_BUILT: return "evaluate called before build";
    case GG_ERR_BAD_INPUT: return "non-finite position, position outside the root cube, or bad index";
    case GG_ERR_TOO_LARGE: return "size beyond the call's limit";
    default: return "unknown status";
    }
}

// Keep memory freed by contexts cached in the device's default pool for the
// next context (the default threshold hands it back to the driver at every
// synchronisation).  A property of this process's pool only.
static void keep_pool_memory(int device)
{
    static std::mutex mu;
    static bool done[64] = {false};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    done[device] = true;
}

extern "C" gg_status gg_create(const gg_config *cfg, gg_ctx **out)
{
    if (!out) return GG_ERR_INVALID;
    *out = nullptr;
    gg_config c;
    if (cfg) c = *cfg; else gg_config_default(&c);
    if (c.leaf_size < 1 || c.leaf_size > 32) return GG_ERR_INVALID;
    if (c.group_size < 1 || c.group_size > 64) return GG_ERR_INVALID;
    if (c.flush_threshold < 32 || c.flush_threshold > 128) return GG_ERR_INVALID;
    if (c.group_order != 0 && c.group_order != 1) return GG_ERR_INVALID;
    if (c.node_staging != 0 && c.node_staging != 1) return GG_ERR_INVALID;
    if (c.walk_stack_entries < 0 || c.walk_stack_entries > kStackMax) return GG_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c.device || c.device < 0) {
        cudaGetLastError();
        snprintf(g_last_cuda_error, sizeof g_last_cuda_error, "no CUDA device %d (found %d)", c.device, ndev);
        return GG_ERR_CUDA;
    }
    gg_ctx *ctx = new gg_ctx();
    ctx->cfg = c;
    ctx->device = c.device;
    ctx->order_by_softening = c.target_order == 1;
    gg_status st = set_device(ctx);
    if (st) { delete ctx; return st; }
    cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { delete ctx; return gg_cuda_fail(e); }
    ctx->stream = ctx->own_stream;
    ctx->for_each_buf([ctx](auto &b) { b.sref = &ctx->stream; b.gen = &ctx->buf_gen; });
    keep_pool_memory(ctx->device);
    if ((e = cudaEventCreateWithFlags(&ctx->stage_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->vstage_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->act_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->done_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->old_ready_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->old_used_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->hmm_ev, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) != cudaSuccess) {
        gg_destroy(ctx);
        return gg_cuda_fail(e);
    }
    for (int i = 0; i < kPipeEvents; i++) {
        if ((e = cudaEventCreateWithFlags(&ctx->pipe_ev[i], cudaEventDisableTiming)) != cudaSuccess) {
            gg_destroy(ctx);
            return gg_cuda_fail(e);
        }
    }
    for (int i = 0; i < 8; i++) cudaEventCreate(&ctx->ev[i]);
    ctx->have_events = true;
    memset(&ctx->last, 0, sizeof ctx->last);
    if ((st = ctx->err.ensure(8)) || (st = ctx->counters.ensure(8)) || (st = ctx->inter.ensure(4))) {
        gg_destroy(ctx);
        return st;
    }
    cudaMemset(ctx->err.p, 0, 8 * sizeof(int));
    *out = ctx;
    return GG_OK;
}

extern "C" gg_status gg_destroy(gg_ctx *c)
{
    if (!c) return GG_ERR_INVALID;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    c->for_each_buf(ReleaseBuf());
    c->h_active.give_back(c->act_ev);
    c->h_acc.give_back(c->done_ev);
    c->h_pot.give_back(c->done_ev);
    c->h_old.give_back(c->done_ev);
    c->h_nint.give_back(c->done_ev);
    c->h_vstage.give_back(c->vstage_ev);
    c->h_stage.give_back(c->stage_ev);
    c->h_hmm.give_back(c->hmm_ev);
    if (c->act_ev) cudaEventDestroy(c->act_ev);
    if (c->hmm_ev) cudaEventDestroy(c->hmm_ev);
    for (int i = 0; i < kPipeEvents; i++)
        if (c->pipe_ev[i]) cudaEventDestroy(c->pipe_ev[i]);
    if (c->done_ev) cudaEventDestroy(c->done_ev);
    if (c->stage_ev) cudaEventDestroy(c->stage_ev);
    if (c->vstage_ev) cudaEventDestroy(c->vstage_ev);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    for (int i = 0; i < 2; i++) {
        if (c->part_exec[i]) cudaGraphExecDestroy(c->part_exec[i]);
        if (c->part_graph[i]) cudaGraphDestroy(c->part_graph[i]);
    }
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->have_events)
        for (int i = 0; i < 8; i++) cudaEventDestroy(c->ev[i]);
    if (c->old_ready_ev) cudaEventDestroy(c->old_ready_ev);
    if (c->old_used_ev) cudaEventDestroy(c->old_used_ev);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return GG_OK;
}

extern "C" gg_status gg_set_stream(gg_ctx *c, void *s)
{
    if (!c) return GG_ERR_INVALID;
    if (c->stream != (cudaStream_t)s) {
        // buffers are freed in stream order: finish what the old stream may still do with them
        cudaSetDevice(c->device);
        GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    }
    c->stream = (cudaStream_t)s;   // NULL is the legacy default stream, as for any CUDA call
    return GG_OK;
}

extern "C" gg_status gg_synchronize(gg_ctx *c)
{
    if (!c) return GG_ERR_INVALID;
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return GG_OK;
}

// ---------------------------------------------------------------- particles
static gg_status set_systems(gg_ctx *c, int S, const int64_t *counts)
{
    if (S < 1 || !counts) return GG_ERR_INVALID;
    long long N = 0;
    std::vector<int> poff(S + 1);
    for (int s = 0; s < S; s++) {
        if (counts[s] < 0) return GG_ERR_INVALID;
        poff[s] = (int)N;
        N += counts[s];
        if (N >= (1ll << 30)) return GG_ERR_TOO_LARGE;
    }
    poff[S] = (int)N;
    if (N != c->N || S != c->S) c->tcost_valid = false;   // same particles reloaded keep their costs
    c->S = S;
    c->N = N;
    c->h_poff = poff;
    c->built = false;
    c->oldacc_valid = false;
    c->have_vel = false;
    c->kin_valid = false;
    gg_status st;
    if ((st = c->poff.ensure(S + 1))) return st;
    GG_CUDA_TRY(cudaMemcpyAsync(c->poff.p, poff.data(), (S + 1) * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if ((st = c->in_rec.ensure(N)) || (st = c->part.ensure(N)) || (st = c->dom.ensure(S)) ||
        (st = c->extent_mm.ensure((size_t)S * 6)) || (st = c->hmm.ensure((size_t)S * 2)) || (st = c->keys.ensure(N)) || (st = c->perm.ensure(N)) ||
        (st = c->rank.ensure(N)) || (st = c->oldacc.ensure(N)))
        return st;
    return GG_OK;
}

extern "C" gg_status gg_load_particles(gg_ctx *c, int32_t S, const int64_t *counts, const double *pos,
                                       int64_t pos_stride, const double *mass, int64_t mass_stride,
                                       const double *soft_h, int64_t soft_stride)
{
    if (!c || !pos || !mass || !soft_h) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if ((st = set_systems(c, S, counts))) return st;
    if (pos_stride <= 0) pos_stride = 3 * sizeof(double);
    if (mass_stride <= 0) mass_stride = sizeof(double);
    if (soft_stride <= 0) soft_stride = sizeof(double);
    long long N = c->N;
    if ((st = c->h_stage.ensure((size_t)N, c->stage_ev))) return st;
    const char *pb = (const char *)pos, *mb = (const char *)mass, *hb = (const char *)soft_h;
    GGPart *dst = c->h_stage.p;
    int mixed = 0;
    for (long long b = 0; b < N; b += kPipeChunk) {   // gather one chunk while the previous one is copied
        const long long e = std::min(N, b + kPipeChunk);
#pragma omp parallel for schedule(static) reduction(| : mixed)
        for (long long i = b; i < e; i++) {
            const double *x = (const double *)(pb + i * pos_stride);
            GGPart r;
            r.x = x[0]; r.y = x[1]; r.z = x[2];
            r.m = (float)*(const double *)(mb + i * mass_stride);
            r.h = (float)*(const double *)(hb + i * soft_stride);
            dst[i] = r;
            if (i > 0 && r.h != (float)*(const double *)(hb + (i - 1) * soft_stride)) mixed = 1;
        }
        GG_CUDA_TRY(cudaMemcpyAsync(c->in_rec.p + b, dst + b, (e - b) * sizeof(GGPart), cudaMemcpyHostToDevice,
                                    c->stream));
    }
    // a change of kernel radius between neighbouring particles of different
    // systems also counts: harmless (ordering then just keeps each system's order)
    c->h_mixed = mixed != 0;
    c->h_mixed_pending = false;
    GG_CUDA_TRY(cudaEventRecord(c->stage_ev, c->stream));
    return GG_OK;
}

extern "C" gg_status gg_load_particles_device(gg_ctx *c, int32_t S, const int64_t *counts, const void *d_records)
{
    if (!c || !d_records) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if ((st = set_systems(c, S, counts))) return st;
    if (c->N) {
        GG_CUDA_TRY(cudaMemcpyAsync(c->in_rec.p, d_records, c->N * sizeof(GGPart), cudaMemcpyDeviceToDevice, c->stream));
        // the range of kernel radii decides whether walks order targets by
        // softening; it crosses to pinned memory behind the extent pass and the
        // first walk reads it, so the load does not wait for the device
        gg_launch_extent(c->in_rec.p, (int)c->N, c->poff.p, S, c->extent_mm.p, c->hmm.p, c->dom.p, c->err.p, c->stream);
        if ((st = c->h_hmm.ensure(2 * (size_t)S, c->hmm_ev))) return st;
        GG_CUDA_TRY(cudaMemcpyAsync(c->h_hmm.p, c->hmm.p, 2 * (size_t)S * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                    c->stream));
        GG_CUDA_TRY(cudaEventRecord(c->hmm_ev, c->stream));
        c->h_mixed_pending = true;
    }
    return GG_OK;
}

// the kernel-radius ranges of a device load, once they have reached the host
static gg_status resolve_h_mixed(gg_ctx *c)
{
    if (!c->h_mixed_pending) return GG_OK;
    GG_CUDA_TRY(cudaEventSynchronize(c->hmm_ev));
    c->h_mixed = false;
    for (int s = 0; s < c->S; s++)
        if (c->h_hmm.p[2 * s] != c->h_hmm.p[2 * s + 1] && c->h_hmm.p[2 * s] != 0x7f800000u) c->h_mixed = true;
    c->h_mixed_pending = false;
    return GG_OK;
}

// ---------------------------------------------------------------- build
// bits of a system id (0 for one system): the sort's last passes order by it
static int sys_bits(int S)
{
    if (S <= 1) return 0;
    int bits = 0;
    while ((1 << bits) < S) bits++;
    return bits;
}

static gg_status ensure_tree(gg_ctx *c)
{
    long long cap = 2 * c->N + c->S + 64;
    if (cap >= (1ll << 31)) return GG_ERR_TOO_LARGE;
    gg_status st;
    int G = gg_tree_grid();
    if ((st = c->t_start.ensure(cap)) || (st = c->t_end.ensure(cap)) || (st = c->t_level.ensure(cap)) ||
        (st = c->t_parent.ensure(cap)) || (st = c->t_sys.ensure(cap)) || (st = c->t_nch.ensure(cap)) ||
        (st = c->t_child.ensure(cap)) || (st = c->t_bnd.ensure(cap * 8)) ||
        (st = c->t_mass64.ensure(cap)) || (st = c->nodes.ensure(cap)) || (st = c->t_depth.ensure(GG_MAX_DEPTH + 4)) ||
        (st = c->t_nnodes.ensure(4)) || (st = c->t_bstat.ensure((size_t)GG_MAX_DEPTH * G)) ||
        (st = c->t_ticket.ensure(GG_MAX_DEPTH)))
        return st;
    c->ncap = (int)cap;
    return GG_OK;
}

static TreeBuf tree_buf(gg_ctx *c)
{
    TreeBuf tb;
    tb.start = c->t_start.p; tb.end = c->t_end.p; tb.level = c->t_level.p; tb.parent = c->t_parent.p;
    tb.sys = c->t_sys.p; tb.nch = c->t_nch.p; tb.child = c->t_child.p;
    tb.bnd = c->t_bnd.p; tb.mass64 = c->t_mass64.p; tb.depth_beg = c->t_depth.p; tb.nnodes = c->t_nnodes.p;
    tb.bstat = c->t_bstat.p; tb.ticket = c->t_ticket.p; tb.err = c->err.p;
    tb.cap = c->ncap;
    return tb;
}

extern "C" gg_status gg_build(gg_ctx *c, const gg_domain *domains)
{
    if (!c || c->S < 1) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    cudaStream_t s = c->stream;
    const int S = c->S, N = (int)c->N;
    const int sbits = sys_bits(S);
    if ((st = c->sort_scratch.ensure(gg_sort_scratch_bytes(N)))) return st;
    if ((st = ensure_tree(c))) return st;
    GG_CUDA_TRY(cudaMemsetAsync(c->err.p, 0, 8 * sizeof(int), s));
    bool timing = c->cfg.timing != 0;
    if (timing) cudaEventRecord(c->ev[0], s);
    // the extent pass also gives each system's range of kernel radii (used to
    // order walk targets); explicit domains then replace its root cubes
    if (N > 0) gg_launch_extent(c->in_rec.p, N, c->poff.p, S, c->extent_mm.p, c->hmm.p, c->dom.p, c->err.p, s);
    if (domains) {
        std::vector<GGDomainDev> d(S);
        for (int i = 0; i < S; i++) {
            for (int k = 0; k < 3; k++) { d[i].center[k] = domains[i].center[k]; d[i].corner[k] = domains[i].corner[k]; }
            d[i].len = domains[i].len;
            d[i].pad = 0;
            if (!(domains[i].len > 0)) return GG_ERR_INVALID;
        }
        GG_CUDA_TRY(cudaMemcpyAsync(c->dom.p, d.data(), S * sizeof(GGDomainDev), cudaMemcpyHostToDevice, s));
        GG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (N > 0) gg_launch_keys(c->in_rec.p, N, c->poff.p, S, c->dom.p, c->keys.p, c->perm.p, c->err.p, s);
    if (timing) cudaEventRecord(c->ev[1], s);
    // the sort's last pass also moves the records into key order
    bool gathered = false;
    if (N > 1) {
        const SortGather g = {c->in_rec.p, c->part.p, c->rank.p};
        st = gg_sort_pairs_run(c->keys.p, c->perm.p, N, 3 * GG_MAX_LEVEL, sbits, c->poff.p, S, c->sort_scratch.p,
                               c->err.p, s, &g, &gathered);
        if (st) return st;
    }
    if (N > 0 && !gathered) gg_launch_permute(c->perm.p, c->in_rec.p, c->part.p, c->rank.p, N, s);
    if (timing) cudaEventRecord(c->ev[2], s);
    gg_launch_tree(c->keys.p, c->poff.p, S, c->cfg.leaf_size, c->ncap, tree_buf(c), c->part.p, c->dom.p, c->nodes.p, s);
    if (timing) cudaEventRecord(c->ev[3], s);
    GG_CUDA_TRY(cudaGetLastError());
    c->built = true;
    c->kin_valid = false;
    c->kin_any = false;
    return GG_OK;
}

extern "C" gg_status gg_get_domains(gg_ctx *c, gg_domain *out)
{
    if (!c || !out || c->S < 1) return GG_ERR_INVALID;
    std::vector<GGDomainDev> d(c->S);
    GG_CUDA_TRY(cudaMemcpyAsync(d.data(), c->dom.p, c->S * sizeof(GGDomainDev), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->S; i++) {
        for (int k = 0; k < 3; k++) { out[i].center[k] = d[i].center[k]; out[i].corner[k] = d[i].corner[k]; }
        out[i].len = d[i].len;
    }
    return GG_OK;
}

// ---------------------------------------------------------------- walk
static gg_status walk_setup(gg_ctx *c)
{
    gg_status st;
    if (!c->stack_cap) c->stack_cap = c->cfg.walk_stack_entries > 0 ? c->cfg.walk_stack_entries : GG_STACK_CAP;
    if (!c->walk_blocks) {
        int per_sm = c->cfg.walk_blocks_per_sm;
        if (per_sm <= 0) per_sm = 2;   // measured best or tied on the galaxy, clustered and Plummer workloads
        if (per_sm > 3) per_sm = 3;
        c->walk_blocks = per_sm;   // blocks per SM; the grid is that many per SM
    }
    const long long maxg = gg_max_groups(c->N, c->S, c->cfg.group_size);
    if ((st = c->groups.ensure(maxg)) || (st = c->ngroups.ensure(2)) || (st = c->gscan.ensure(c->S + 1)) ||
        (st = c->toff.ensure(c->S + 1)) ||
        (c->cfg.group_size > 1 &&
         ((st = c->g_node.ensure(c->N + 1)) || (st = c->g_flag.ensure(c->N + 1)) || (st = c->g_seg.ensure(c->N + 1)) ||
          (st = c->g_segstart.ensure(c->N + 1)))) ||
        (st = c->stack.ensure((size_t)c->walk_blocks * gg_num_sms() * (gg_walk_threads() / 32) * c->stack_cap)) ||
        (st = c->scan_scratch.ensure(gg_scan_scratch_ints())))
        return st;
    if (c->cfg.group_order &&
        ((st = c->tcost.ensure(c->N + 1)) || (st = c->gkey.ensure(maxg)) || (st = c->gorder.ensure(maxg)) ||
         (st = c->sort_scratch.ensure(gg_sort_scratch_bytes(maxg)))))
        return st;
    return GG_OK;
}

// run the walk; outputs to device pointers.  pot_only: the potential-only
// walk (no acceleration output, OldAcc left as it is)
static gg_status run_walk(gg_ctx *c, const int *d_active, int n_active, const double *d_old_acc, double tol,
                          double theta, double *d_acc, double *d_pot, int *d_nint, bool pot_only = false)
{
    gg_status st;
    cudaStream_t s = c->stream;
    if ((st = walk_setup(c))) return st;
    if ((st = resolve_h_mixed(c))) return st;
    const int S = c->S, N = (int)c->N;
    const int *tlist = nullptr, *tout = nullptr;
    const int *toff = c->poff.p;
    if (d_active) {
        if ((st = c->flag.ensure(N)) || (st = c->flagscan.ensure(N + 1)) || (st = c->tlist.ensure(N)) ||
            (st = c->tout.ensure(N)))
            return st;
        gg_launch_active(d_active, n_active, c->rank.p, N, c->flag.p, c->flagscan.p, c->tlist.p, c->tout.p, c->poff.p,
                         S, c->toff.p, c->scan_scratch.p, c->err.p, s);
        tlist = c->tlist.p;
        tout = c->tout.p;
        toff = c->toff.p;
    }
    if (c->h_mixed && c->order_by_softening) {
        const int nt = d_active ? n_active : N;
        if ((st = c->tkey.ensure(nt)) || (st = c->tval.ensure(nt)) || (st = c->tlist2.ensure(nt)) ||
            (st = c->tout2.ensure(nt)))
            return st;
        st = gg_order_targets_by_softening(nt, tlist, tout, c->part.p, c->keys.p, c->poff.p, S, c->dom.p, c->hmm.p,
                                           c->tkey.p, c->tval.p,
                                           c->tlist2.p, tout ? c->tout2.p : nullptr, c->sort_scratch.p, c->err.p, s);
        if (st) return st;
        tlist = c->tlist2.p;
        if (tout) tout = c->tout2.p;
    }
    if (d_old_acc) {
        GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc.p, d_old_acc, (size_t)N * sizeof(double), cudaMemcpyDeviceToDevice, s));
        c->oldacc_valid = true;
    }
    const long long maxg = gg_max_groups(c->N, c->S, c->cfg.group_size);
    if (c->cfg.group_size > 1) {
        const bool by_soft = c->h_mixed && c->order_by_softening;
        gg_launch_groups_tree(d_active ? n_active : N, tlist, d_active ? c->flagscan.p : nullptr, toff, S,
                              c->cfg.group_size, tree_buf(c), by_soft ? c->dom.p : nullptr, c->hmm.p,
                              gg_target_order_lmax(S), c->g_node.p, c->g_flag.p, c->g_seg.p, c->g_segstart.p,
                              (int)maxg, c->groups.p, c->ngroups.p, c->scan_scratch.p, c->err.p, s);
    } else {
        gg_launch_groups(toff, S, c->cfg.group_size, c->groups.p, c->ngroups.p, c->gscan.p, s);
    }
    const unsigned *gorder = nullptr;
    if (c->cfg.group_order && !c->tcost_valid)   // a fresh history: targets not walked yet cost 0
        GG_CUDA_TRY(cudaMemsetAsync(c->tcost.p, 0, (size_t)c->N * sizeof(float), s));
    if (c->cfg.group_order && c->tcost_valid) {
        if ((st = gg_order_groups_by_cost(c->groups.p, c->ngroups.p, (int)maxg, tlist, c->perm.p, c->tcost.p,
                                          c->gkey.p, c->gorder.p, c->sort_scratch.p, c->err.p, s)))
            return st;
        gorder = c->gorder.p;
    }
    GG_CUDA_TRY(cudaMemsetAsync(c->counters.p, 0, 8 * sizeof(int), s));
    GG_CUDA_TRY(cudaMemsetAsync(c->inter.p, 0, 4 * sizeof(unsigned long long), s));
    WalkParams p;
    p.nodes = c->nodes.p;
    p.parts = c->part.p;
    p.groups = c->groups.p;
    p.ngroups = c->ngroups.p;
    p.tlist = tlist;
    p.tout = tout;
    p.perm = c->perm.p;
    p.oldacc_in = c->oldacc_valid ? c->oldacc.p : nullptr;
    p.oldacc_out = pot_only ? nullptr : c->oldacc.p;
    p.tol = tol;
    p.theta = theta;
    p.acc = d_acc;
    p.pot = d_pot;
    p.ninter = d_nint;
    p.interactions = c->inter.p;
    p.group_counter = c->counters.p;
    p.stack = c->stack.p;
    p.stack_cap = c->stack_cap;
    p.err = c->err.p;
    p.group_size = c->cfg.group_size;
    p.flush = c->cfg.flush_threshold;
    p.pot_only = pot_only ? 1 : 0;
    if (pot_only) p.acc = nullptr;
    p.gorder = gorder;
    p.node_staging = c->cfg.node_staging;
    p.cost_out = c->cfg.group_order ? c->tcost.p : nullptr;
    int tpl = c->cfg.group_size > 32 ? 2 : 1;
    if (c->cfg.timing) cudaEventRecord(c->ev[4], s);
    gg_launch_walk(p, tpl, c->walk_blocks, s);
    if (c->cfg.timing) cudaEventRecord(c->ev[5], s);
    if (!pot_only) c->oldacc_valid = true;
    if (c->cfg.group_order) c->tcost_valid = true;
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

static gg_status collect_stats(gg_ctx *c, gg_stats *out);

// A blocking walk: when a warp's node stack overflowed (its group's results
// were skipped and the error bit set), the walk runs again with four times
// the stack, from the OldAcc the first attempt started from, like the
// reference growing its node pool and rebuilding (forcetree.c:112-125).
static gg_status walk_with_stack_retry(gg_ctx *c, const int *d_active, int n_active, const double *d_old, double tol,
                                       double theta, double *d_acc, double *d_pot, int *d_nint, bool pot_only)
{
    gg_status st;
    cudaStream_t s = c->stream;
    // the walk rewrites the device OldAcc of the groups that finished: keep
    // the starting values for a second attempt
    const bool keep = !d_old && c->oldacc_valid && !pot_only && c->N > 0;
    if (keep) {
        if ((st = c->oldacc_save.ensure(c->N + 1))) return st;
        GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc_save.p, c->oldacc.p, c->N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    for (;;) {
        if ((st = run_walk(c, d_active, n_active, d_old, tol, theta, d_acc, d_pot, d_nint, pot_only))) return st;
        int err = 0;
        GG_CUDA_TRY(cudaMemcpyAsync(&err, c->err.p, sizeof err, cudaMemcpyDeviceToHost, s));
        GG_CUDA_TRY(cudaStreamSynchronize(s));
        if (!(err & GG_EBIT_STACK_OVERFLOW) || c->stack_cap >= kStackMax) return GG_OK;
        c->stack_cap = std::min(kStackMax, 4 * c->stack_cap);
        // a captured step holds the old stack's address: it must be captured again
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
        const int rest = err & ~GG_EBIT_STACK_OVERFLOW;
        GG_CUDA_TRY(cudaMemcpyAsync(c->err.p, &rest, sizeof rest, cudaMemcpyHostToDevice, s));
        if (keep)
            GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc.p, c->oldacc_save.p, c->N * sizeof(double), cudaMemcpyDeviceToDevice,
                                        s));
        GG_CUDA_TRY(cudaStreamSynchronize(s));   // `rest` is on the stack of this frame
    }
}

static gg_status collect_stats(gg_ctx *c, gg_stats *out)
{
    int err[8];
    unsigned long long inter4[4] = {0, 0, 0, 0};
    int nn = 0, ng = 0;
    GG_CUDA_TRY(cudaMemcpyAsync(err, c->err.p, sizeof err, cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaMemcpyAsync(inter4, c->inter.p, sizeof inter4, cudaMemcpyDeviceToHost, c->stream));
    if (c->t_nnodes.p) GG_CUDA_TRY(cudaMemcpyAsync(&nn, c->t_nnodes.p, sizeof nn, cudaMemcpyDeviceToHost, c->stream));
    if (c->ngroups.p) GG_CUDA_TRY(cudaMemcpyAsync(&ng, c->ngroups.p, sizeof ng, cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    gg_stats &L = c->last;
    L.interactions = (int64_t)inter4[0];
    L.far_entries = (int64_t)inter4[1];
    L.near_entries = (int64_t)inter4[2];
    L.nodes_tested = (int64_t)inter4[3];
    L.n_nodes = nn;
    L.n_groups = ng;
    L.error_word = err[0];
    if (c->cfg.timing) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]) == cudaSuccess) L.ms_keys = ms;
        if (cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]) == cudaSuccess) L.ms_sort = ms;
        if (cudaEventElapsedTime(&ms, c->ev[2], c->ev[3]) == cudaSuccess) L.ms_build = ms;
        if (cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]) == cudaSuccess) L.ms_walk = ms;
        cudaGetLastError();
    }
    if (out) *out = L;
    if (err[0] & (GG_EBIT_SORT_TIMEOUT | GG_EBIT_WALK_TIMEOUT)) return GG_ERR_TIMEOUT;
    if (err[0] & (GG_EBIT_NODE_OVERFLOW | GG_EBIT_STACK_OVERFLOW)) return GG_ERR_OVERFLOW;
    if (err[0] & GG_EBIT_BAD_INPUT) return GG_ERR_BAD_INPUT;
    return GG_OK;
}

extern "C" gg_status gg_last_stats(gg_ctx *c, gg_stats *out)
{
    if (!c) return GG_ERR_INVALID;
    return collect_stats(c, out);
}

extern "C" gg_status gg_evaluate_device(gg_ctx *c, const int32_t *d_active, int64_t n_active, const double *d_old_acc,
                                        double tol, double theta, double *d_acc, double *d_pot, int32_t *d_nint)
{
    if (!c || !d_acc) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (d_active && (n_active < 0 || n_active > c->N)) return GG_ERR_INVALID;
    if (tol < 0 || theta < 0) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    return run_walk(c, d_active, (int)n_active, d_old_acc, tol, theta, d_acc, d_pot, d_nint);
}

extern "C" gg_status gg_evaluate(gg_ctx *c, const int32_t *active, int64_t n_active, const double *old_acc,
                                 double tol, double theta, double *acc_out, double *pot_out, int64_t *ninter_out,
                                 gg_stats *stats)
{
    if (!c || !acc_out) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (tol < 0 || theta < 0) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    cudaStream_t s = c->stream;
    long long nt = active ? n_active : c->N;
    if (active && (n_active < 0 || n_active > c->N)) return GG_ERR_INVALID;
    size_t outn = (size_t)(c->N > 0 ? c->N : 1);
    if ((st = c->acc_d.ensure(outn * 3)) || (st = c->pot_d.ensure(outn)) || (st = c->nint_d.ensure(outn))) return st;
    // host arrays go through pinned staging (copied in and out by all host
    // threads): transfers from and to pageable memory run at a fraction of the
    // link's speed
    const int *d_active = nullptr;
    if (active) {
        if ((st = c->active_d.ensure(n_active > 0 ? n_active : 1))) return st;
        if (n_active) {
            if ((st = c->h_active.ensure((size_t)n_active, c->act_ev))) return st;
            parallel_copy(c->h_active.p, active, (size_t)n_active * sizeof(int));
            GG_CUDA_TRY(cudaMemcpyAsync(c->active_d.p, c->h_active.p, n_active * sizeof(int), cudaMemcpyHostToDevice, s));
            GG_CUDA_TRY(cudaEventRecord(c->act_ev, s));
        }
        d_active = c->active_d.p;
    }
    const double *d_old = nullptr;
    if (old_acc && c->N) {
        // the upload overlaps the build already queued on the compute stream
        const bool fresh = c->oldacc_in.cap < (size_t)c->N;
        if ((st = c->h_old.ensure((size_t)c->N, c->done_ev)) || (st = c->oldacc_in.ensure(c->N))) return st;
        if (fresh) GG_CUDA_TRY(cudaEventRecord(c->old_used_ev, s));   // the new array exists from here on
        GG_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->old_used_ev, 0));
        for (long long b = 0; b < c->N; b += kPipeChunk) {
            const long long e = std::min((long long)c->N, b + kPipeChunk);
            parallel_copy(c->h_old.p + b, old_acc + b, (size_t)(e - b) * sizeof(double));
            GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc_in.p + b, c->h_old.p + b, (e - b) * sizeof(double),
                                        cudaMemcpyHostToDevice, c->copy_stream));
        }
        GG_CUDA_TRY(cudaEventRecord(c->old_ready_ev, c->copy_stream));
        GG_CUDA_TRY(cudaStreamWaitEvent(s, c->old_ready_ev, 0));
        d_old = c->oldacc_in.p;
    }
    if ((st = walk_with_stack_retry(c, d_active, (int)n_active, d_old, tol, theta, c->acc_d.p, c->pot_d.p,
                                    c->nint_d.p, false)))
        return st;
    if (d_old) GG_CUDA_TRY(cudaEventRecord(c->old_used_ev, s));
    // results come back in chunks; each chunk is copied out while the next crosses the link
    long long chunk = kPipeChunk, nchunks = 0;
    if (nt) {
        if ((st = c->h_acc.ensure((size_t)nt * 3, c->done_ev))) return st;
        if (pot_out && (st = c->h_pot.ensure((size_t)nt, c->done_ev))) return st;
        if (ninter_out && (st = c->h_nint.ensure((size_t)nt, c->done_ev))) return st;
        nchunks = (nt + chunk - 1) / chunk;
        if (nchunks > kPipeEvents) {
            chunk = (nt + kPipeEvents - 1) / kPipeEvents;
            nchunks = (nt + chunk - 1) / chunk;
        }
        for (long long k = 0; k < nchunks; k++) {
            const long long b = k * chunk, e = std::min(nt, b + chunk);
            GG_CUDA_TRY(cudaMemcpyAsync(c->h_acc.p + 3 * b, c->acc_d.p + 3 * b, (e - b) * 3 * sizeof(double),
                                        cudaMemcpyDeviceToHost, s));
            if (pot_out)
                GG_CUDA_TRY(cudaMemcpyAsync(c->h_pot.p + b, c->pot_d.p + b, (e - b) * sizeof(double),
                                            cudaMemcpyDeviceToHost, s));
            if (ninter_out)
                GG_CUDA_TRY(cudaMemcpyAsync(c->h_nint.p + b, c->nint_d.p + b, (e - b) * sizeof(int),
                                            cudaMemcpyDeviceToHost, s));
            GG_CUDA_TRY(cudaEventRecord(c->pipe_ev[k], s));
        }
    }
    GG_CUDA_TRY(cudaEventRecord(c->done_ev, s));
    for (long long k = 0; k < nchunks; k++) {
        const long long b = k * chunk, e = std::min(nt, b + chunk);
        GG_CUDA_TRY(cudaEventSynchronize(c->pipe_ev[k]));
        parallel_copy(acc_out + 3 * b, c->h_acc.p + 3 * b, (size_t)(e - b) * 3 * sizeof(double));
        if (pot_out) parallel_copy(pot_out + b, c->h_pot.p + b, (size_t)(e - b) * sizeof(double));
    }
    st = collect_stats(c, stats);   // synchronises the stream
    if (nt) {
        if (ninter_out) {
            const int *ni = c->h_nint.p;
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < nt; i++) ninter_out[i] = ni[i];
        }
    }
    // every transfer of this call and of the loads before it is complete
    c->h_stage.give_back(c->stage_ev);
    c->h_vstage.give_back(c->vstage_ev);
    c->h_active.give_back(c->act_ev);
    c->h_old.give_back(c->done_ev);
    c->h_acc.give_back(c->done_ev);
    c->h_pot.give_back(c->done_ev);
    c->h_nint.give_back(c->done_ev);
    c->last.n_targets = nt;
    if (stats) stats->n_targets = nt;
    return st;
}

// ---------------------------------------------------------------- kernel-level entry points
extern "C" gg_status gg_peano_hilbert_keys(int64_t n, const double *d_pos, const gg_domain *dom, uint64_t *d_keys,
                                           void *stream)
{
    if (n < 0 || !dom || (n && (!d_pos || !d_keys)) || !(dom->len > 0)) return GG_ERR_INVALID;
    if (n == 0) return GG_OK;
    GGDomainDev d;
    for (int k = 0; k < 3; k++) { d.center[k] = dom->center[k]; d.corner[k] = dom->corner[k]; }
    d.len = dom->len;
    d.pad = 0;
    gg_launch_keys_plain(d_pos, n, d, (unsigned long long *)d_keys, nullptr, (cudaStream_t)stream);
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

extern "C" gg_status gg_radix_sort_pairs(int64_t n, uint64_t *d_keys, uint32_t *d_vals, int32_t key_bits, void *stream)
{
    if (n < 0 || key_bits < 1 || key_bits > 64 || (n && (!d_keys || !d_vals))) return GG_ERR_INVALID;
    if (n <= 1) return GG_OK;
    if (n >= (1ll << 30)) return GG_ERR_TOO_LARGE;
    cudaStream_t s = (cudaStream_t)stream;
    size_t bytes = gg_sort_scratch_bytes(n);
    void *scratch = nullptr;
    int *err = nullptr;
    GG_CUDA_TRY(cudaMallocAsync(&scratch, bytes, s));
    cudaError_t e = cudaMallocAsync((void **)&err, 64, s);
    if (e != cudaSuccess) { cudaFreeAsync(scratch, s); return gg_cuda_fail(e); }
    cudaMemsetAsync(err, 0, 64, s);
    gg_status st = gg_sort_pairs_run((unsigned long long *)d_keys, d_vals, n, key_bits, 0, nullptr, 1, scratch, err, s);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(scratch, s);
    cudaFreeAsync(err, s);
    GG_CUDA_TRY(cudaStreamSynchronize(s));
    if (st) return st;
    if (herr & GG_EBIT_SORT_TIMEOUT) return GG_ERR_TIMEOUT;
    return GG_OK;
}

extern "C" gg_status gg_direct_sum_fp64(int64_t n_src, const double *d_pos, const double *d_mass, const double *d_h,
                                        int64_t n_tgt, const int32_t *d_targets, double *d_acc, double *d_pot,
                                        void *stream)
{
    if (n_src < 0 || n_tgt < 0 || (n_src && (!d_pos || !d_mass || !d_h)) || (n_tgt && !d_acc)) return GG_ERR_INVALID;
    if (!d_targets && n_tgt > n_src) return GG_ERR_INVALID;
    gg_launch_direct(n_src, d_pos, d_mass, d_h, n_tgt, d_targets, d_acc, d_pot, (cudaStream_t)stream);
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

// ---------------------------------------------------------------- graphs and autotuning
// One step of a resident batch (keys, sort, tree, moments, walk of every
// target of every system) captured once and replayed as a single CUDA graph.
// The capture reuses the context's buffers, so the step must have run once
// uncaptured with the same systems (every buffer is then already allocated
// and nothing inside the capture allocates or synchronises).
extern "C" gg_status gg_graph_capture_step(gg_ctx *c, double tol, double theta, double *d_acc, double *d_pot)
{
    if (!c || !d_acc || tol < 0 || theta < 0) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (!c->stream) return GG_ERR_INVALID;   // the legacy default stream cannot be captured
    gg_status st;
    if ((st = set_device(c))) return st;
    if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    // grow every buffer the walk may need, and read the kernel-radius ranges, before capturing
    if ((st = walk_setup(c))) return st;
    if ((st = resolve_h_mixed(c))) return st;
    const int timing = c->cfg.timing;
    c->cfg.timing = 0;
    long long before = gg_kernel_launches();
    const long long gen0 = c->buf_gen;
    GG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    st = gg_build(c, nullptr);
    if (!st) st = run_walk(c, nullptr, 0, nullptr, tol, theta, d_acc, d_pot, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->cfg.timing = timing;
    if (!st && e == cudaSuccess && c->buf_gen != gen0) st = GG_ERR_NOT_BUILT;   // a buffer grew: step once uncaptured
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return gg_cuda_fail(e);
    c->graph_launches = (int)(gg_kernel_launches() - before);
    c->graph = g;
    e = cudaGraphInstantiate(&c->graph_exec, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); c->graph = nullptr; c->graph_exec = nullptr; return gg_cuda_fail(e); }
    c->graph_gen = c->buf_gen;
    return GG_OK;
}

static void drop_part_graphs(gg_ctx *c)
{
    for (int i = 0; i < 2; i++) {
        if (c->part_exec[i]) { cudaGraphExecDestroy(c->part_exec[i]); c->part_exec[i] = nullptr; }
        if (c->part_graph[i]) { cudaGraphDestroy(c->part_graph[i]); c->part_graph[i] = nullptr; }
    }
    c->part_gen = -1;
}

extern "C" gg_status gg_graph_capture_parts(gg_ctx *c, double tol, double theta, double *d_acc, double *d_pot)
{
    if (!c || !d_acc || tol < 0 || theta < 0) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (!c->stream) return GG_ERR_INVALID;   // the legacy default stream cannot be captured
    gg_status st;
    if ((st = set_device(c))) return st;
    drop_part_graphs(c);
    if ((st = walk_setup(c))) return st;
    if ((st = resolve_h_mixed(c))) return st;
    const int timing = c->cfg.timing;
    c->cfg.timing = 0;
    const long long gen0 = c->buf_gen;
    for (int part = 0; part < 2; part++) {
        const long long before = gg_kernel_launches();
        GG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        st = part == 0 ? gg_build(c, nullptr) : run_walk(c, nullptr, 0, nullptr, tol, theta, d_acc, d_pot, nullptr);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (!st && e != cudaSuccess) st = gg_cuda_fail(e);
        if (!st && c->buf_gen != gen0) st = GG_ERR_NOT_BUILT;   // a buffer grew: step once uncaptured
        if (!st) {
            c->part_graph[part] = g;
            c->part_launches[part] = (int)(gg_kernel_launches() - before);
            e = cudaGraphInstantiate(&c->part_exec[part], g, 0);
            if (e != cudaSuccess) st = gg_cuda_fail(e);
        } else if (g) {
            cudaGraphDestroy(g);
        }
        if (st) {
            c->cfg.timing = timing;
            drop_part_graphs(c);
            return st;
        }
    }
    c->cfg.timing = timing;
    c->part_gen = c->buf_gen;
    return GG_OK;
}

extern "C" gg_status gg_graph_launch_part(gg_ctx *c, int32_t part)
{
    if (!c || part < 0 || part > 1) return GG_ERR_INVALID;
    if (!c->part_exec[part] || c->part_gen != c->buf_gen) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    GG_CUDA_TRY(cudaGraphLaunch(c->part_exec[part], c->stream));
    gg_note_launches(c->part_launches[part]);
    return GG_OK;
}

extern "C" gg_status gg_graph_launch(gg_ctx *c)
{
    if (!c) return GG_ERR_INVALID;
    if (!c->graph_exec || c->graph_gen != c->buf_gen) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    GG_CUDA_TRY(cudaGraphLaunch(c->graph_exec, c->stream));
    gg_note_launches(c->graph_launches);
    return GG_OK;
}

// Timed search over the walk's tunables on the resident systems: leaf size
// (rebuilds the tree), group size (targets per warp), blocks per SM (stack
// depth per warp follows from it) and the list-flush threshold; then the
// other node staging on the winner.  Every trial
// walks from the same OldAcc, so trials see the same opening decisions for a
// given tree; the fastest configuration is kept and the tree rebuilt with it.
// ---------------------------------------------------------------- autotuner accuracy gate
// A faster configuration is only taken if it is no less accurate than the
// configuration the context had (the default one, whose errors the parity
// tests hold to the reference tree's).  Accuracy is measured on a fixed sample
// of targets against their FP64 direct sums: every target of a system of up to
// 2,048 particles, else 16,384 / S targets (at least 64, at most 4,096) evenly
// spaced in load order, S being the number of systems.  A candidate passes when
//   - its 99th-percentile relative force error over all sampled targets, and
//     the largest of the systems' own 99th percentiles, are each at most 1.1x
//     the base configuration's (plus 1e-7 for errors at rounding level), and
//   - the root mean square over systems of the relative error of the sample
//     potential energy W = 1/2 sum m phi is at most 1.1x the base's, or below
//     1e-5.
// With one system these are that system's p99 and |W - W_direct| / |W_direct|.
// (A system-by-system test of W would refuse almost any change on a large
// ensemble: W's error is a signed sum, and its sign and size move from system
// to system with any change of the interaction lists.)
static const int kTuneAllBelow = 2048, kTuneBudget = 16384, kTuneMin = 64, kTuneMax = 4096;

struct TuneRef {
    std::vector<int2> tg;                 // (load index, system) of each sampled target
    std::vector<int2> rows;               // (output row, 0) of each sampled target
    std::vector<int> first;               // first sample row of each system (S + 1 entries)
    std::vector<double> acc_dir, pot_dir, mass;
};
struct TuneErr {
    double p99_all = 0, p99_worst = 0, w_rms = 0;
};

// The sample: in each system, its targets (all of them, or the walk's active
// ones), every one of them up to kTuneAllBelow, else `per` evenly spaced in
// walk order.  h_active: the active load indices (n_active), or null for all.
static gg_status tune_reference(gg_ctx *c, TuneRef &R, const int *h_active, long long n_active)
{
    gg_status st;
    R.tg.clear();
    R.rows.clear();
    R.first.assign(c->S + 1, 0);
    const long long per = std::min<long long>(kTuneMax, std::max<long long>(kTuneMin, kTuneBudget / c->S));
    std::vector<std::vector<int>> act_rows;   // per system, the rows of its active targets
    if (h_active) {
        act_rows.resize(c->S);
        for (long long r = 0; r < n_active; r++) {
            const int i = h_active[r];
            if (i < 0 || i >= c->N) return GG_ERR_INVALID;
            const int s = (int)(std::upper_bound(c->h_poff.begin(), c->h_poff.begin() + c->S + 1, i) -
                                c->h_poff.begin()) - 1;
            act_rows[s].push_back((int)r);
        }
    }
    for (int s = 0; s < c->S; s++) {
        const long long o = c->h_poff[s];
        const long long n = h_active ? (long long)act_rows[s].size() : c->h_poff[s + 1] - o;
        R.first[s] = (int)R.tg.size();
        const long long k = n <= kTuneAllBelow ? n : per;
        for (long long j = 0; j < k; j++) {
            const long long q = n <= kTuneAllBelow ? j : (2 * j + 1) * n / (2 * k);   // q-th target of the system
            const int row = h_active ? act_rows[s][q] : (int)(o + q);
            R.tg.push_back(make_int2(h_active ? h_active[row] : row, s));
            R.rows.push_back(make_int2(row, 0));
        }
    }
    R.first[c->S] = (int)R.tg.size();
    const int nt = (int)R.tg.size();
    if ((st = c->tune_tg.ensure(nt)) || (st = c->tune_rows.ensure(nt)) || (st = c->tune_acc.ensure(3 * (size_t)nt)) ||
        (st = c->tune_pot.ensure(nt)) || (st = c->tune_mass.ensure(nt)) || (st = c->tune_gacc.ensure(3 * (size_t)nt)) ||
        (st = c->tune_gpot.ensure(nt)))
        return st;
    GG_CUDA_TRY(cudaMemcpyAsync(c->tune_tg.p, R.tg.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA_TRY(cudaMemcpyAsync(c->tune_rows.p, R.rows.data(), nt * sizeof(int2), cudaMemcpyHostToDevice, c->stream));
    gg_launch_direct_records(c->in_rec.p, c->poff.p, c->tune_tg.p, nt, c->tune_acc.p, c->tune_pot.p, c->tune_mass.p,
                             c->stream);
    R.acc_dir.resize(3 * (size_t)nt);
    R.pot_dir.resize(nt);
    R.mass.resize(nt);
    GG_CUDA_TRY(cudaMemcpyAsync(R.acc_dir.data(), c->tune_acc.p, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost,
                                c->stream));
    GG_CUDA_TRY(cudaMemcpyAsync(R.pot_dir.data(), c->tune_pot.p, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaMemcpyAsync(R.mass.data(), c->tune_mass.p, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

// p-th percentile with linear interpolation between order statistics
static double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double x = q / 100.0 * (double)(v.size() - 1);
    const size_t i = (size_t)x;
    return i + 1 < v.size() ? v[i] + (x - (double)i) * (v[i + 1] - v[i]) : v[i];
}

// errors of the outputs the last walk left in acc_d / pot_d (load order)
static gg_status tune_errors(gg_ctx *c, const TuneRef &R, TuneErr &E)
{
    const int nt = (int)R.tg.size();
    gg_launch_gather_rows(c->acc_d.p, c->pot_d.p, c->tune_rows.p, nt, c->tune_gacc.p, c->tune_gpot.p, c->stream);
    std::vector<double> a(3 * (size_t)nt), p(nt);
    GG_CUDA_TRY(cudaMemcpyAsync(a.data(), c->tune_gacc.p, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaMemcpyAsync(p.data(), c->tune_gpot.p, nt * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    std::vector<double> all;
    double w2 = 0;
    int nsys = 0;
    E = TuneErr();
    for (int s = 0; s < c->S; s++) {
        std::vector<double> e;
        double w = 0, wd = 0;
        for (int t = R.first[s]; t < R.first[s + 1]; t++) {
            double d2 = 0, r2 = 0;
            for (int k = 0; k < 3; k++) {
                const double d = a[3 * (size_t)t + k] - R.acc_dir[3 * (size_t)t + k];
                d2 += d * d;
                r2 += R.acc_dir[3 * (size_t)t + k] * R.acc_dir[3 * (size_t)t + k];
            }
            if (r2 > 0) e.push_back(sqrt(d2 / r2));
            w += 0.5 * R.mass[t] * p[t];
            wd += 0.5 * R.mass[t] * R.pot_dir[t];
        }
        if (e.empty()) continue;
        E.p99_worst = std::max(E.p99_worst, percentile(e, 99.0));
        all.insert(all.end(), e.begin(), e.end());
        if (wd != 0) {
            w2 += (w - wd) * (w - wd) / (wd * wd);
            nsys++;
        }
    }
    E.p99_all = percentile(all, 99.0);
    E.w_rms = nsys ? sqrt(w2 / nsys) : 0.0;
    return GG_OK;
}

static bool tune_accepts(const TuneErr &base, const TuneErr &cand)
{
    return cand.p99_all <= 1.1 * base.p99_all + 1e-7 && cand.p99_worst <= 1.1 * base.p99_worst + 1e-7 &&
           (cand.w_rms <= 1.1 * base.w_rms || cand.w_rms < 1e-5);
}

extern "C" gg_status gg_autotune(gg_ctx *c, double tol, double theta, gg_config *chosen, double *best_ms)
{
    return gg_autotune_active(c, nullptr, 0, tol, theta, chosen, best_ms);
}

extern "C" gg_status gg_autotune_active(gg_ctx *c, const int32_t *d_active, int64_t n_active, double tol, double theta,
                                        gg_config *chosen, double *best_ms)
{
    if (!c || tol < 0 || theta < 0 || n_active < 0 || (n_active && !d_active)) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (n_active > c->N) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    cudaStream_t s = c->stream;
    const long long N = c->N;
    if ((st = c->acc_d.ensure(N * 3 + 3)) || (st = c->pot_d.ensure(N + 1))) return st;
    if (!n_active) d_active = nullptr;
    std::vector<int> h_active(d_active ? n_active : 0);
    if (d_active) {
        GG_CUDA_TRY(cudaMemcpyAsync(h_active.data(), d_active, n_active * sizeof(int), cudaMemcpyDeviceToHost, s));
        GG_CUDA_TRY(cudaStreamSynchronize(s));
    }
    TuneRef R;
    if ((st = tune_reference(c, R, d_active ? h_active.data() : nullptr, n_active))) return st;
    const bool had_old = c->oldacc_valid;
    if (had_old && ((st = c->oldacc_save.ensure(N + 1)))) return st;
    if (had_old)
        GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc_save.p, c->oldacc.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    cudaEvent_t e0, e1;
    GG_CUDA_TRY(cudaEventCreate(&e0));
    GG_CUDA_TRY(cudaEventCreate(&e1));
    const gg_config base = c->cfg;
    const int base_blocks = c->walk_blocks;
    static const int leafs[] = {8, 16}, groups[] = {32, 64}, bpss[] = {2, 3}, flushes[] = {64, 128};
    float best = 1e30f;
    gg_config best_cfg = base;
    int best_blocks = base_blocks;
    st = GG_OK;
    TuneErr base_err, err;
    bool have_base = false;
    int tried = 0, refused = 0;
    // one configuration: the faster of two timed walks from the same OldAcc,
    // and whether its outputs pass the accuracy gate against the base
    // configuration's (the first call measures the base itself)
    auto trial = [&](float *ms_out, bool *ok) -> gg_status {
        float ms_min = 1e30f;
        for (int rep = 0; rep < 2; rep++) {
            if (had_old) {
                cudaError_t ce =
                    cudaMemcpyAsync(c->oldacc.p, c->oldacc_save.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s);
                if (ce != cudaSuccess) return gg_cuda_fail(ce);
            }
            c->oldacc_valid = had_old;
            cudaEventRecord(e0, s);
            gg_status r = run_walk(c, d_active, (int)n_active, nullptr, tol, theta, c->acc_d.p, c->pot_d.p, nullptr);
            cudaEventRecord(e1, s);
            if (r) return r;
            if ((r = collect_stats(c, nullptr))) return r;
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < ms_min) ms_min = ms;
        }
        *ms_out = ms_min;
        gg_status r = tune_errors(c, R, err);
        if (r) return r;
        if (!have_base) { base_err = err; have_base = true; }
        *ok = tune_accepts(base_err, err);
        tried++;
        if (!*ok) refused++;
        return GG_OK;
    };
    // the base configuration first: its errors are the gate's bar
    {
        float ms = 0;
        bool ok = false;
        st = trial(&ms, &ok);
        if (!st) best = ms;
    }
    for (int li = 0; li < 2 && !st; li++) {
        c->cfg.leaf_size = leafs[li];
        if ((st = gg_build(c, nullptr))) break;
        for (int gi = 0; gi < 2 && !st; gi++)
            for (int bi = 0; bi < 2 && !st; bi++)
                for (int fi = 0; fi < 2 && !st; fi++) {
                    c->cfg.group_size = groups[gi];
                    c->cfg.flush_threshold = flushes[fi];
                    c->walk_blocks = bpss[bi];
                    float ms = 0;
                    bool ok = false;
                    if ((st = trial(&ms, &ok))) break;
                    if (ok && ms < best) {
                        best = ms;
                        best_cfg = c->cfg;
                        best_blocks = c->walk_blocks;
                    }
                }
    }
    // the other node staging, on the winner
    if (!st) {
        c->cfg = best_cfg;
        c->walk_blocks = best_blocks;
        c->cfg.node_staging = 1 - best_cfg.node_staging;
        float ms = 0;
        bool ok = false;
        if (!(st = gg_build(c, nullptr)) && !(st = trial(&ms, &ok)) && ok && ms < best) {
            best = ms;
            best_cfg = c->cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // keep the winner (or restore the original configuration after a failure)
    c->cfg = st ? base : best_cfg;
    c->walk_blocks = st ? base_blocks : best_blocks;
    c->cfg.walk_blocks_per_sm = c->walk_blocks;
    gg_status st2 = gg_build(c, nullptr);
    if (had_old) {
        cudaError_t ce = cudaMemcpyAsync(c->oldacc.p, c->oldacc_save.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (ce != cudaSuccess && !st2) st2 = gg_cuda_fail(ce);
    }
    c->oldacc_valid = had_old;
    if (!st) st = st2;
    if (!st && chosen) *chosen = c->cfg;
    if (!st && best_ms) *best_ms = best;
    c->tune_tried = tried;
    c->tune_refused = refused;
    return st;
}

// The accuracy gate of gg_autotune for one candidate configuration against
// the context's own, from the same OldAcc; the context is left as it was.
extern "C" gg_status gg_tune_accuracy(gg_ctx *c, double tol, double theta, const gg_config *cand, int32_t *accepted)
{
    if (!c || !cand || !accepted || tol < 0 || theta < 0) return GG_ERR_INVALID;
    if (cand->leaf_size < 1 || cand->leaf_size > 32 || cand->group_size < 1 || cand->group_size > 64 ||
        cand->flush_threshold < 32 || cand->flush_threshold > 128 || cand->walk_blocks_per_sm < 0 ||
        cand->walk_blocks_per_sm > 3 || cand->node_staging < 0 || cand->node_staging > 1)
        return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    cudaStream_t s = c->stream;
    const long long N = c->N;
    if ((st = c->acc_d.ensure(N * 3 + 3)) || (st = c->pot_d.ensure(N + 1))) return st;
    TuneRef R;
    if ((st = tune_reference(c, R, nullptr, 0))) return st;
    const bool had_old = c->oldacc_valid;
    if (had_old && ((st = c->oldacc_save.ensure(N + 1)))) return st;
    if (had_old)
        GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc_save.p, c->oldacc.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
    auto walk_errors = [&](TuneErr &E) -> gg_status {
        if (had_old)
            GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc.p, c->oldacc_save.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s));
        c->oldacc_valid = had_old;
        gg_status r = run_walk(c, nullptr, 0, nullptr, tol, theta, c->acc_d.p, c->pot_d.p, nullptr);
        if (r || (r = collect_stats(c, nullptr))) return r;
        return tune_errors(c, R, E);
    };
    TuneErr base, cerr;
    if ((st = walk_errors(base))) return st;
    const gg_config keep = c->cfg;
    const int keep_blocks = c->walk_blocks;
    c->cfg.leaf_size = cand->leaf_size;
    c->cfg.group_size = cand->group_size;
    c->cfg.flush_threshold = cand->flush_threshold;
    c->cfg.node_staging = cand->node_staging;
    c->cfg.target_order = cand->target_order;
    c->cfg.group_order = cand->group_order;
    if (cand->walk_blocks_per_sm > 0) c->walk_blocks = cand->walk_blocks_per_sm;
    const bool rebuild = cand->leaf_size != keep.leaf_size;
    if (rebuild) st = gg_build(c, nullptr);
    if (!st) st = walk_errors(cerr);
    if (!st) *accepted = tune_accepts(base, cerr) ? 1 : 0;
    c->cfg = keep;
    c->walk_blocks = keep_blocks;
    gg_status st2 = rebuild ? gg_build(c, nullptr) : GG_OK;
    if (had_old) {
        cudaError_t ce = cudaMemcpyAsync(c->oldacc.p, c->oldacc_save.p, N * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (ce != cudaSuccess && !st2) st2 = gg_cuda_fail(ce);
    }
    c->oldacc_valid = had_old;
    return st ? st : st2;
}

// ---------------------------------------------------------------- drift
extern "C" gg_status gg_load_velocities(gg_ctx *c, const double *vel, int64_t vel_stride)
{
    if (!c || !vel || c->S < 1) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if (vel_stride <= 0) vel_stride = 3 * sizeof(double);
    const long long N = c->N;
    if ((st = c->vel.ensure((size_t)3 * N + 3))) return st;
    if ((st = c->h_vstage.ensure((size_t)N * 3, c->vstage_ev))) return st;
    const char *vb = (const char *)vel;
    double *dst = c->h_vstage.p;
    for (long long b = 0; b < N; b += kPipeChunk) {
        const long long e = std::min(N, b + kPipeChunk);
#pragma omp parallel for schedule(static)
        for (long long i = b; i < e; i++) {
            const double *v = (const double *)(vb + i * vel_stride);
            dst[3 * i] = v[0]; dst[3 * i + 1] = v[1]; dst[3 * i + 2] = v[2];
        }
        GG_CUDA_TRY(cudaMemcpyAsync(c->vel.p + 3 * b, dst + 3 * b, (size_t)(e - b) * 3 * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
    }
    GG_CUDA_TRY(cudaEventRecord(c->vstage_ev, c->stream));
    c->have_vel = true;
    c->kin_valid = false;
    return GG_OK;
}

extern "C" gg_status gg_load_velocities_device(gg_ctx *c, const double *d_vel)
{
    if (!c || !d_vel || c->S < 1) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if ((st = c->vel.ensure((size_t)3 * c->N + 3))) return st;
    if (c->N)
        GG_CUDA_TRY(cudaMemcpyAsync(c->vel.p, d_vel, (size_t)c->N * 3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                    c->stream));
    c->have_vel = true;
    c->kin_valid = false;
    return GG_OK;
}

extern "C" gg_status gg_set_positions(gg_ctx *c, const double *pos, int64_t pos_stride)
{
    if (!c || !pos || c->S < 1) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    if (pos_stride <= 0) pos_stride = 3 * sizeof(double);
    const long long N = c->N;
    if ((st = c->newpos.ensure((size_t)3 * N + 3))) return st;
    if ((st = c->h_vstage.ensure((size_t)N * 3, c->vstage_ev))) return st;
    const char *pb = (const char *)pos;
    double *dst = c->h_vstage.p;
    for (long long b = 0; b < N; b += kPipeChunk) {   // gather one chunk while the previous one is copied
        const long long e = std::min(N, b + kPipeChunk);
#pragma omp parallel for schedule(static)
        for (long long i = b; i < e; i++) {
            const double *x = (const double *)(pb + i * pos_stride);
            dst[3 * i] = x[0]; dst[3 * i + 1] = x[1]; dst[3 * i + 2] = x[2];
        }
        GG_CUDA_TRY(cudaMemcpyAsync(c->newpos.p + 3 * b, dst + 3 * b, (size_t)(e - b) * 3 * sizeof(double),
                                    cudaMemcpyHostToDevice, c->stream));
    }
    GG_CUDA_TRY(cudaEventRecord(c->vstage_ev, c->stream));
    gg_launch_set_positions(c->in_rec.p, c->part.p, c->perm.p, c->newpos.p, (int)N, c->err.p, c->stream);
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

// dt_host: one step per system, or NULL for `dt_all` everywhere (no host copy,
// so the call stays asynchronous)
static gg_status drift_common(gg_ctx *c, const double *dt_host, double dt_all)
{
    if (!c) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (!c->have_vel) return GG_ERR_INVALID;
    if (!std::isfinite(dt_all)) return GG_ERR_INVALID;
    for (int s = 0; dt_host && s < c->S; s++)
        if (!std::isfinite(dt_host[s])) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if ((st = c->kin.ensure(c->ncap)) || (st = c->kin_counter.ensure(c->ncap)) || (st = c->dts.ensure(c->S)))
        return st;
    cudaStream_t s = c->stream;
    if (!c->kin_valid) {
        GG_CUDA_TRY(cudaMemsetAsync(c->kin_counter.p, 0, (size_t)c->ncap * sizeof(int), s));
        gg_launch_node_kinematics(c->part.p, c->perm.p, c->vel.p, tree_buf(c), c->kin_counter.p, c->kin.p, (int)c->N,
                                  c->ncap, c->kin_any ? 1 : 0, s);
        c->kin_valid = true;
        c->kin_any = true;
    }
    // pageable source: the copy has taken the values when it returns
    if (dt_host)
        GG_CUDA_TRY(cudaMemcpyAsync(c->dts.p, dt_host, (size_t)c->S * sizeof(double), cudaMemcpyHostToDevice, s));
    gg_launch_drift(c->in_rec.p, c->part.p, c->perm.p, c->vel.p, c->poff.p, c->S, dt_host ? c->dts.p : nullptr,
                    dt_all, c->nodes.p, c->kin.p, c->t_sys.p, c->t_nnodes.p, (int)c->N, c->ncap, s);
    GG_CUDA_TRY(cudaGetLastError());
    return GG_OK;
}

extern "C" gg_status gg_drift(gg_ctx *c, double dt)
{
    return drift_common(c, nullptr, dt);
}

extern "C" gg_status gg_drift_systems(gg_ctx *c, const double *dt)
{
    if (!c || !dt) return GG_ERR_INVALID;
    return drift_common(c, dt, 0.0);
}

// ---------------------------------------------------------------- accounting
extern "C" gg_status gg_device_bytes(gg_ctx *c, int64_t *bytes)
{
    if (!c || !bytes) return GG_ERR_INVALID;
    long long total = 0;
    c->for_each_buf(CountBuf{&total});
    *bytes = (int64_t)total;
    return GG_OK;
}

// ---------------------------------------------------------------- batches of separate host systems
// Host gather of per-system arrays into the pinned staging buffer, in chunks
// of at most 64K particles so that one large system spreads over the threads.
struct HostChunk { int sys; long long first, count, dst; };

static std::vector<HostChunk> host_chunks(const gg_ctx *c)
{
    std::vector<HostChunk> ch;
    for (int s = 0; s < c->S; s++) {
        const long long n = c->h_poff[s + 1] - c->h_poff[s];
        for (long long f = 0; f < n; f += 65536)
            ch.push_back({s, f, std::min(65536ll, n - f), (long long)c->h_poff[s] + f});
    }
    return ch;
}

static gg_status ensure_stage(gg_ctx *c)
{
    return c->h_stage.ensure((size_t)c->N, c->stage_ev);
}

extern "C" gg_status gg_load_systems(gg_ctx *c, int32_t S, const int64_t *counts, const double *const *pos,
                                     const double *const *mass, const double *const *soft_h)
{
    if (!c || !pos || !mass || !soft_h || !counts || S < 1) return GG_ERR_INVALID;
    for (int s = 0; s < S; s++)
        if (counts[s] > 0 && (!pos[s] || !mass[s] || !soft_h[s])) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if ((st = set_systems(c, S, counts))) return st;
    if ((st = ensure_stage(c))) return st;
    const std::vector<HostChunk> ch = host_chunks(c);
    GGPart *dst = c->h_stage.p;
    int mixed = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : mixed)
    for (long long k = 0; k < (long long)ch.size(); k++) {
        const HostChunk q = ch[k];
        const double *x = pos[q.sys], *m = mass[q.sys], *h = soft_h[q.sys];
        const double h0 = h[0];
        for (long long i = q.first; i < q.first + q.count; i++) {
            GGPart r;
            r.x = x[3 * i]; r.y = x[3 * i + 1]; r.z = x[3 * i + 2];
            r.m = (float)m[i];
            r.h = (float)h[i];
            dst[q.dst + (i - q.first)] = r;
            if ((float)h[i] != (float)h0) mixed = 1;
        }
    }
    c->h_mixed = mixed != 0;
    c->h_mixed_pending = false;
    if (c->N) GG_CUDA_TRY(cudaMemcpyAsync(c->in_rec.p, c->h_stage.p, c->N * sizeof(GGPart), cudaMemcpyHostToDevice,
                                          c->stream));
    GG_CUDA_TRY(cudaEventRecord(c->stage_ev, c->stream));
    return GG_OK;
}

extern "C" gg_status gg_load_system_velocities(gg_ctx *c, const double *const *vel)
{
    if (!c || !vel || c->S < 1) return GG_ERR_INVALID;
    for (int s = 0; s < c->S; s++)
        if (c->h_poff[s + 1] > c->h_poff[s] && !vel[s]) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    const long long N = c->N;
    if ((st = c->vel.ensure((size_t)3 * N + 3))) return st;
    if ((st = c->h_vstage.ensure((size_t)N * 3, c->vstage_ev))) return st;
    const std::vector<HostChunk> ch = host_chunks(c);
    double *dst = c->h_vstage.p;
#pragma omp parallel for schedule(dynamic, 1)
    for (long long k = 0; k < (long long)ch.size(); k++) {
        const HostChunk q = ch[k];
        memcpy(dst + 3 * q.dst, vel[q.sys] + 3 * q.first, (size_t)q.count * 3 * sizeof(double));
    }
    if (N) GG_CUDA_TRY(cudaMemcpyAsync(c->vel.p, dst, (size_t)N * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    GG_CUDA_TRY(cudaEventRecord(c->vstage_ev, c->stream));
    c->have_vel = true;
    c->kin_valid = false;
    return GG_OK;
}

// ---------------------------------------------------------------- asynchronous evaluation
// the asynchronous walk; with acc_pinned / pot_pinned (pinned mode) the
// results go straight to the caller's page-locked arrays, otherwise per flags
// into the context's own pinned buffers
static gg_status evaluate_async(gg_ctx *c, const int32_t *active, int64_t n_active, double tol, double theta,
                                int32_t flags, bool pinned, double *acc_pinned, double *pot_pinned)
{
    if (!c) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (tol < 0 || theta < 0 || (active && (n_active < 0 || n_active > c->N))) return GG_ERR_INVALID;
    if (flags & ~(GG_ASYNC_COPY_ACC | GG_ASYNC_COPY_POT)) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    if (pinned) {
        for (const void *ptr : {(const void *)acc_pinned, (const void *)pot_pinned}) {
            if (!ptr) continue;
            cudaPointerAttributes a;
            if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
                cudaGetLastError();
                return GG_ERR_INVALID;
            }
            if (a.type != cudaMemoryTypeHost) return GG_ERR_INVALID;
        }
    }
    cudaStream_t s = c->stream;
    const long long nt = active ? n_active : c->N;
    size_t outn = (size_t)(c->N > 0 ? c->N : 1);
    if ((st = c->acc_d.ensure(outn * 3)) || (st = c->pot_d.ensure(outn))) return st;
    const int *d_active = nullptr;
    if (active) {
        if ((st = c->h_active.ensure((size_t)n_active, c->act_ev))) return st;
        if ((st = c->active_d.ensure(n_active > 0 ? n_active : 1))) return st;
        memcpy(c->h_active.p, active, (size_t)n_active * sizeof(int));
        if (n_active)
            GG_CUDA_TRY(cudaMemcpyAsync(c->active_d.p, c->h_active.p, n_active * sizeof(int), cudaMemcpyHostToDevice, s));
        GG_CUDA_TRY(cudaEventRecord(c->act_ev, s));
        d_active = c->active_d.p;
    }
    if ((st = run_walk(c, d_active, (int)n_active, nullptr, tol, theta, c->acc_d.p, c->pot_d.p, nullptr))) return st;
    c->async_pinned = pinned;
    if (pinned) {
        if (nt && acc_pinned)
            GG_CUDA_TRY(cudaMemcpyAsync(acc_pinned, c->acc_d.p, nt * 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (nt && pot_pinned)
            GG_CUDA_TRY(cudaMemcpyAsync(pot_pinned, c->pot_d.p, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
        c->async_n = nt;
        c->async_flags = 0;
    } else if (flags) {
        // unfetched results of an earlier call are overwritten in stream order
        if ((flags & GG_ASYNC_COPY_ACC) && (st = c->h_acc.ensure((size_t)nt * 3, c->done_ev))) return st;
        if ((flags & GG_ASYNC_COPY_POT) && (st = c->h_pot.ensure((size_t)nt, c->done_ev))) return st;
        if (nt && (flags & GG_ASYNC_COPY_ACC))
            GG_CUDA_TRY(cudaMemcpyAsync(c->h_acc.p, c->acc_d.p, nt * 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (nt && (flags & GG_ASYNC_COPY_POT))
            GG_CUDA_TRY(cudaMemcpyAsync(c->h_pot.p, c->pot_d.p, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
        c->async_n = nt;
        c->async_flags = flags;
    }
    c->last.n_targets = nt;
    GG_CUDA_TRY(cudaEventRecord(c->done_ev, s));
    return GG_OK;
}

extern "C" gg_status gg_evaluate_async(gg_ctx *c, const int32_t *active, int64_t n_active, double tol, double theta,
                                       int32_t flags)
{
    return evaluate_async(c, active, n_active, tol, theta, flags, false, nullptr, nullptr);
}

extern "C" gg_status gg_evaluate_async_pinned(gg_ctx *c, const int32_t *active, int64_t n_active, double tol,
                                              double theta, double *acc_pinned, double *pot_pinned)
{
    return evaluate_async(c, active, n_active, tol, theta, 0, true, acc_pinned, pot_pinned);
}

// page-locked blocks handed to callers: pointer -> block size
static std::mutex g_user_pinned_mu;
static std::map<void *, size_t> g_user_pinned;

extern "C" gg_status gg_host_alloc(int64_t bytes, void **out)
{
    if (!out || bytes < 0) return GG_ERR_INVALID;
    size_t got = 0;
    void *p = pinned_get(bytes > 0 ? (size_t)bytes : 1, &got);
    if (!p) return GG_ERR_NOMEM;
    {
        std::lock_guard<std::mutex> lk(g_user_pinned_mu);
        g_user_pinned[p] = got;
    }
    *out = p;
    return GG_OK;
}

extern "C" gg_status gg_host_free(void *ptr)
{
    if (!ptr) return GG_OK;
    size_t bytes = 0;
    {
        std::lock_guard<std::mutex> lk(g_user_pinned_mu);
        auto it = g_user_pinned.find(ptr);
        if (it == g_user_pinned.end()) return GG_ERR_INVALID;
        bytes = it->second;
        g_user_pinned.erase(it);
    }
    pinned_put(ptr, bytes);
    return GG_OK;
}

extern "C" gg_status gg_query(gg_ctx *c)
{
    if (!c) return GG_ERR_INVALID;
    cudaError_t e = cudaEventQuery(c->done_ev);
    if (e == cudaSuccess) return GG_OK;
    if (e == cudaErrorNotReady) { cudaGetLastError(); return GG_PENDING; }
    return gg_cuda_fail(e);
}

extern "C" gg_status gg_fetch_results(gg_ctx *c, double *acc_out, double *pot_out, gg_stats *stats)
{
    if (!c) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    GG_CUDA_TRY(cudaEventSynchronize(c->done_ev));
    const long long nt = c->async_n;
    if (c->async_pinned && (acc_out || pot_out)) return GG_ERR_INVALID;   // already in the caller's arrays
    if (acc_out) {
        if (!(c->async_flags & GG_ASYNC_COPY_ACC)) return GG_ERR_INVALID;
        parallel_copy(acc_out, c->h_acc.p, (size_t)nt * 3 * sizeof(double));
    }
    if (pot_out) {
        if (!(c->async_flags & GG_ASYNC_COPY_POT)) return GG_ERR_INVALID;
        parallel_copy(pot_out, c->h_pot.p, (size_t)nt * sizeof(double));
    }
    // the evaluation and every transfer before it are done: hand the pinned
    // buffers back for other contexts
    c->h_stage.give_back(c->stage_ev);
    c->h_vstage.give_back(c->vstage_ev);
    c->h_active.give_back(c->act_ev);
    c->h_acc.give_back(c->done_ev);
    c->h_pot.give_back(c->done_ev);
    c->async_flags = 0;
    st = collect_stats(c, stats);
    if (stats) stats->n_targets = nt;
    return st;
}

// ---------------------------------------------------------------- device memory reservation
extern "C" gg_status gg_reserve_device_pool(int32_t device, int64_t bytes)
{
    if (bytes < 0) return GG_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return GG_ERR_INVALID;
    }
    GG_CUDA_TRY(cudaSetDevice(device));
    keep_pool_memory(device);
    cudaStream_t s;
    GG_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    // grow the pool in 2 GB pieces, then give them all back to it
    const size_t piece = (size_t)2 << 30;
    std::vector<void *> got;
    gg_status st = GG_OK;
    for (int64_t left = bytes; left > 0; left -= (int64_t)piece) {
        void *p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, std::min((size_t)left, piece), s);
        if (e != cudaSuccess) { cudaGetLastError(); st = GG_ERR_NOMEM; break; }
        got.push_back(p);
    }
    for (void *p : got) cudaFreeAsync(p, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess && !st) st = gg_cuda_fail(e);
    return st;
}

// ---------------------------------------------------------------- potential-only walk
extern "C" gg_status gg_evaluate_potential_device(gg_ctx *c, const int32_t *d_active, int64_t n_active,
                                                  const double *d_old_acc, double tol, double theta, double *d_pot)
{
    if (!c || !d_pot) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (d_active && (n_active < 0 || n_active > c->N)) return GG_ERR_INVALID;
    if (tol < 0 || theta < 0) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    return run_walk(c, d_active, (int)n_active, d_old_acc, tol, theta, nullptr, d_pot, nullptr, true);
}

extern "C" gg_status gg_evaluate_potential(gg_ctx *c, const int32_t *active, int64_t n_active, const double *old_acc,
                                           double tol, double theta, double *pot_out, gg_stats *stats)
{
    if (!c || !pot_out) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    if (tol < 0 || theta < 0) return GG_ERR_INVALID;
    if (active && (n_active < 0 || n_active > c->N)) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    cudaStream_t s = c->stream;
    const long long nt = active ? n_active : c->N;
    if ((st = c->pot_d.ensure((size_t)(c->N > 0 ? c->N : 1)))) return st;
    const int *d_active = nullptr;
    if (active) {
        if ((st = c->active_d.ensure(n_active > 0 ? n_active : 1))) return st;
        if (n_active) {
            if ((st = c->h_active.ensure((size_t)n_active, c->act_ev))) return st;
            parallel_copy(c->h_active.p, active, (size_t)n_active * sizeof(int));
            GG_CUDA_TRY(cudaMemcpyAsync(c->active_d.p, c->h_active.p, n_active * sizeof(int), cudaMemcpyHostToDevice, s));
            GG_CUDA_TRY(cudaEventRecord(c->act_ev, s));
        }
        d_active = c->active_d.p;
    }
    if (old_acc) {   // becomes the context's OldAcc, as in gg_evaluate
        if ((st = c->h_old.ensure((size_t)c->N, c->done_ev))) return st;
        parallel_copy(c->h_old.p, old_acc, (size_t)c->N * sizeof(double));
        GG_CUDA_TRY(cudaMemcpyAsync(c->oldacc.p, c->h_old.p, c->N * sizeof(double), cudaMemcpyHostToDevice, s));
        c->oldacc_valid = true;
    }
    st = walk_with_stack_retry(c, d_active, (int)n_active, nullptr, tol, theta, nullptr, c->pot_d.p, nullptr, true);
    if (st) return st;
    if (nt) {
        if ((st = c->h_pot.ensure((size_t)nt, c->done_ev))) return st;
        GG_CUDA_TRY(cudaMemcpyAsync(c->h_pot.p, c->pot_d.p, nt * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    GG_CUDA_TRY(cudaEventRecord(c->done_ev, s));
    st = collect_stats(c, stats);
    if (nt) parallel_copy(pot_out, c->h_pot.p, (size_t)nt * sizeof(double));
    c->h_active.give_back(c->act_ev);
    c->h_old.give_back(c->done_ev);
    c->h_pot.give_back(c->done_ev);
    c->last.n_targets = nt;
    if (stats) stats->n_targets = nt;
    return st;
}

// ---------------------------------------------------------------- energy and momentum checks
extern "C" gg_status gg_energy_device(gg_ctx *c, const double *d_acc, const double *d_pot, double *out)
{
    if (!c || !out || c->S < 1) return GG_ERR_INVALID;
    gg_status st;
    if ((st = set_device(c))) return st;
    const int S = c->S;
    const long long chunk = 65536;
    std::vector<int4> ch;
    std::vector<int> first(S + 1);
    for (int s = 0; s < S; s++) {
        first[s] = (int)ch.size();
        for (long long b = c->h_poff[s]; b < c->h_poff[s + 1]; b += chunk)
            ch.push_back(make_int4(s, (int)b, (int)std::min<long long>(b + chunk, c->h_poff[s + 1]), 0));
    }
    first[S] = (int)ch.size();
    const size_t nc = ch.size();
    if ((st = c->e_chunks.ensure(nc + 1)) || (st = c->e_first.ensure(S + 1)) || (st = c->e_part.ensure(4 * nc + 4)) ||
        (st = c->e_out.ensure(4 * (size_t)S)))
        return st;
    cudaStream_t s = c->stream;
    if (nc) GG_CUDA_TRY(cudaMemcpyAsync(c->e_chunks.p, ch.data(), nc * sizeof(int4), cudaMemcpyHostToDevice, s));
    GG_CUDA_TRY(cudaMemcpyAsync(c->e_first.p, first.data(), (S + 1) * sizeof(int), cudaMemcpyHostToDevice, s));
    gg_launch_energy(c->e_chunks.p, (int)nc, c->e_first.p, S, c->in_rec.p, d_acc, d_pot, c->e_part.p, c->e_out.p, s);
    GG_CUDA_TRY(cudaGetLastError());
    GG_CUDA_TRY(cudaMemcpyAsync(out, c->e_out.p, 4 * (size_t)S * sizeof(double), cudaMemcpyDeviceToHost, s));
    GG_CUDA_TRY(cudaStreamSynchronize(s));
    return GG_OK;
}

// ---------------------------------------------------------------- Peano-Hilbert order
extern "C" gg_status gg_get_order(gg_ctx *c, int32_t *order_out)
{
    if (!c || !order_out) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    if (c->N == 0) return GG_OK;
    // perm holds the load index of each sorted position (uint32 < 2^30)
    GG_CUDA_TRY(cudaMemcpyAsync(order_out, c->perm.p, (size_t)c->N * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    GG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return GG_OK;
}

extern "C" gg_status gg_get_order_device(gg_ctx *c, int32_t *d_order_out)
{
    if (!c || !d_order_out) return GG_ERR_INVALID;
    if (!c->built) return GG_ERR_NOT_BUILT;
    gg_status st;
    if ((st = set_device(c))) return st;
    if (c->N == 0) return GG_OK;
    GG_CUDA_TRY(cudaMemcpyAsync(d_order_out, c->perm.p, (size_t)c->N * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                c->stream));
    return GG_OK;
}

// ---------------------------------------------------------------- self-test of the bounded waits
extern "C" gg_status gg_selftest_bounded_wait(void *stream)
{
    return gg_sort_timeout_selftest((cudaStream_t)stream);
}
