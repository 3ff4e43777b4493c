/*
 * gizmo_gravity_b200.h -- C ABI of the B200 tree-gravity library.
 *
 * The library replaces GIZMO's tree-gravity force evaluation: the Peano-Hilbert
 * keys and sort (system/peano.c, domain.c), the oct-tree build with monopole
 * moments (gravity/forcetree.c force_treebuild / force_update_node_recursive)
 * and the tree walk (gravity/forcetree.c force_treeevaluate, driven by
 * gravity_tree in gravity/gravtree.c).  GIZMO selects it with the compile
 * flag GRAVITY_GPU_B200 inside gravity_tree(); kicks, timesteps and the
 * active-particle list are unchanged.
 *
 * Conventions (all paths below are within the GIZMO source tree):
 *   - accelerations and potentials come back in GIZMO's pre-G units: the walk
 *     accumulates sum m*dx/r^3 and the caller multiplies by All.G
 *     (gravity/gravtree.c:495, :501);
 *   - softening is passed as the kernel radius h = 2.8 * Plummer epsilon,
 *     i.e. ForceSoftening_KernelRadius() (proto.h:134-155, gravtree.c:774);
 *   - err_tol_theta > 0 selects the Barnes-Hut pass, err_tol_theta == 0 the
 *     relative criterion with err_tol_force_acc (forcetree.c:2104-2158);
 *   - old_acc is |a|/G of the previous pass, P[i].OldAcc (gravtree.c:514-522).
 *
 * Several independent systems can be loaded at once ("systems", each with its
 * own root cube and tree); a GIZMO rank uses one.  No function traps on the
 * device: kernels record failures in an error word and the call returns a
 * negative gg_status.  A context is not re-entrant; use one per host thread.
 */
#ifndef GIZMO_GRAVITY_B200_H
#define GIZMO_GRAVITY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gg_status;

enum {
    GG_PENDING = 1,           /* gg_query: the context's last asynchronous work is still running */
    GG_OK = 0,
    GG_ERR_INVALID = -1,      /* bad argument (null pointer, negative size, ...) */
    GG_ERR_CUDA = -2,         /* CUDA runtime error or no usable device */
    GG_ERR_NOMEM = -3,        /* device allocation failed */
    GG_ERR_OVERFLOW = -4,     /* node pool or walk stack overflow */
    GG_ERR_TIMEOUT = -5,      /* a bounded device-side wait gave up */
    GG_ERR_NOT_BUILT = -6,    /* gg_evaluate before gg_build */
    GG_ERR_BAD_INPUT = -7,    /* non-finite position, or positions outside the cube */
    GG_ERR_TOO_LARGE = -8     /* size beyond a fixed limit of the call */
};

typedef struct gg_config {
    int32_t device;           /* CUDA device ordinal */
    int32_t leaf_size;        /* max particles per leaf bucket, 1..32 (default 8) */
    int32_t group_size;       /* targets per walk group, 1..64 (default 32) */
    int32_t flush_threshold;  /* interaction-list entries per flush, 32..128 (default 128) */
    int32_t walk_blocks_per_sm; /* persistent walk blocks per SM, 0 = default */
    int32_t timing;           /* 1: record per-stage device times into gg_stats */
    int32_t target_order;     /* 1 (default): when a system holds several kernel radii, walk
                                 targets are ordered by Peano-Hilbert cell at the softening
                                 scale, then by radius, so groups are compact and of one radius
                                 where they can be; 0: plain key order */
    int32_t group_order;      /* 1 (default): walk groups are handed out most expensive first, by
                                 the cost each target had in the previous walk of this context
                                 (its group's device cycles per target); 0: in target order.
                                 The order changes no result, only when each group runs */
    int32_t node_staging;     /* how the walk stages node records in shared memory: 0 (default):
                                 each lane copies its own with cp.async (through L1); 1: the
                                 bulk-copy (TMA) engine, one copy per run of consecutive records,
                                 completing on an mbarrier (force walks of groups > 1; the
                                 exact and potential-only walks stage per lane).  Same results;
                                 gg_autotune tries both */
    int32_t walk_stack_entries; /* entries of each walk warp's node stack in device memory
                                 beyond its 512 in shared memory, 0 = default (8192).  A
                                 blocking evaluation whose stack overflows is run again with
                                 four times the entries (up to 131072), from the same OldAcc,
                                 as the reference grows its node pool and rebuilds
                                 (forcetree.c:112-125), and a step captured by
                                 gg_graph_capture_step must then be captured again; an
                                 asynchronous evaluation reports GG_ERR_OVERFLOW */
} gg_config;

/* root cube of one system: domain_findExtent (domain.c:2518-2570) */
typedef struct gg_domain {
    double center[3];
    double corner[3];
    double len;
} gg_domain;

typedef struct gg_stats {
    int64_t interactions;   /* sum over targets of used nodes/particles with r2>0 && m>0
                               (the reference's Costtotal, gravtree.c:700) */
    int64_t n_nodes;        /* tree nodes over all systems */
    int64_t n_targets;      /* targets walked */
    int32_t n_groups;       /* walk groups */
    int32_t error_word;     /* device error bits of the last call */
    double ms_keys;         /* extent + keys (device time, when timing is on) */
    double ms_sort;         /* key sort, whose last pass also moves the records into key order */
    double ms_build;        /* tree + moments */
    double ms_walk;
    int64_t far_entries;    /* interaction-list entries evaluated without softening (all groups) */
    int64_t near_entries;   /* entries that needed the softening branch */
    int64_t nodes_tested;   /* node opening tests */
} gg_stats;

typedef struct gg_ctx gg_ctx;

/* ---- context ------------------------------------------------------------ */
void gg_config_default(gg_config *cfg);
gg_status gg_create(const gg_config *cfg, gg_ctx **out);
gg_status gg_destroy(gg_ctx *ctx);
const char *gg_strerror(gg_status s);
/* run this context's work on the given cudaStream_t from now on; NULL selects
 * the CUDA legacy default stream.  A new context runs on a stream of its own. */
gg_status gg_set_stream(gg_ctx *ctx, void *cuda_stream);
gg_status gg_synchronize(gg_ctx *ctx);

/* ---- particles -----------------------------------------------------------
 * Replaces the particle gather of force_treebuild (forcetree.c:109) and the
 * P[] loads of force_treeevaluate (forcetree.c:1850-1968).  Host arrays may be
 * strided: GIZMO passes &P[0].Pos[0], sizeof(struct particle_data), and so on.
 * counts[n_systems] gives each system's particle count; particles of system s
 * follow those of system s-1.  Masses are stored in FP32 on the device. */
gg_status gg_load_particles(gg_ctx *ctx, int32_t n_systems, const int64_t *counts, const double *pos,
                            int64_t pos_stride_bytes, const double *mass, int64_t mass_stride_bytes,
                            const double *soft_h, int64_t soft_stride_bytes);
/* device-resident records {double x,y,z; float mass; float h} (32 bytes each).
 * Asynchronous on the context's stream: the per-system range of kernel radii
 * (which decides whether walks order targets by softening) is copied to the
 * host behind the load, and the first walk after it waits for that copy only. */
gg_status gg_load_particles_device(gg_ctx *ctx, int32_t n_systems, const int64_t *counts, const void *d_records);

/* ---- build -------------------------------------------------------------
 * domain_findExtent (domain.c:2518) + keys (domain.c:2236-2262, peano.c:303)
 * + sort (peano.c:28-92) + force_treebuild (forcetree.c:109-342) +
 * force_update_node_recursive (forcetree.c:434-942).  domains == NULL: the
 * root cube of each system is found on the device like domain_findExtent. */
gg_status gg_build(gg_ctx *ctx, const gg_domain *domains);
gg_status gg_get_domains(gg_ctx *ctx, gg_domain *out);
/* The Peano-Hilbert order of the last build: order_out[i] = load index of
 * the particle at sorted position i (N entries; systems in load order, each
 * sorted by key, ties by load index).  With GIZMO's domain cube passed to
 * gg_build this is peano_hilbert_order's sort (system/peano.c:28-92) down to
 * 21 bits per dimension; the reference orders particles that share a 21-bit
 * cell by its finer key bits.  Blocking. */
gg_status gg_get_order(gg_ctx *ctx, int32_t *order_out);
/* The same order into device memory, asynchronous on the context's stream
 * (a split of one system over several GPUs cuts it into Peano-Hilbert ranges
 * of targets, the way domain.c:2224-2300 cuts the curve into domains). */
gg_status gg_get_order_device(gg_ctx *ctx, int32_t *d_order_out);

/* ---- walk --------------------------------------------------------------
 * The force_treeevaluate loop of gravity_tree (gravtree.c:138-457).
 * active: indices of the particles to evaluate (NULL = all, in load order);
 * old_acc: per particle |a|/G in load order (NULL = the values the previous
 * evaluation of this context left on the device, or 0 before the first).
 * Outputs (per active particle, in the order of `active`): acc_out n*3 and
 * pot_out n (pre-G), ninter_out n (nullable each).  Blocking. */
gg_status gg_evaluate(gg_ctx *ctx, const int32_t *active, int64_t n_active, const double *old_acc,
                      double err_tol_force_acc, double err_tol_theta, double *acc_out, double *pot_out,
                      int64_t *ninter_out, gg_stats *stats);
/* Same on device pointers, asynchronous on the context's stream. */
gg_status gg_evaluate_device(gg_ctx *ctx, const int32_t *d_active, int64_t n_active, const double *d_old_acc,
                             double err_tol_force_acc, double err_tol_theta, double *d_acc_out,
                             double *d_pot_out, int32_t *d_ninter_out);
/* interaction count and error word of the last evaluation (synchronises) */
gg_status gg_last_stats(gg_ctx *ctx, gg_stats *stats);

/* device memory the context holds now (all its buffers), for callers that
 * admit work against a memory budget; no counterpart in the reference */
gg_status gg_device_bytes(gg_ctx *ctx, int64_t *bytes);
/* Contexts allocate their device buffers in stream order from the device's
 * default memory pool, which this library sets to keep freed memory for
 * reuse.  gg_reserve_device_pool grows that pool by `bytes` once (allocated
 * and handed back at once), so that later contexts are served from memory
 * already mapped: a server reserves its memory budget at start.  The memory
 * stays with the process.  Returns GG_ERR_NOMEM if the device cannot hold it
 * (what was reserved until then stays reserved).  Synchronous. */
gg_status gg_reserve_device_pool(int32_t device, int64_t bytes);

/* ---- potential-only walk and energy checks -------------------------------
 * compute_potential (gravity/potential.c:24-160) with its walk
 * force_treeevaluate_potential (gravity/forcetree.c:3169-3474): the force
 * walk's opening rules, the potential only, r = 0 pairs counted like any other
 * pair, then each particle's self term m_i kernel(0) / h_i removed
 * (potential.c:137-145).  Pre-G.  A given old_acc becomes the context's OldAcc
 * as in gg_evaluate; the potential walk itself does not update OldAcc.
 * gg_evaluate_potential blocks; the device form is asynchronous. */
gg_status gg_evaluate_potential(gg_ctx *ctx, const int32_t *active, int64_t n_active, const double *old_acc,
                                double err_tol_force_acc, double err_tol_theta, double *pot_out, gg_stats *stats);
gg_status gg_evaluate_potential_device(gg_ctx *ctx, const int32_t *d_active, int64_t n_active,
                                       const double *d_old_acc, double err_tol_force_acc, double err_tol_theta,
                                       double *d_pot_out);
/* FP64 checks per system over every particle, from load-order device arrays
 * of all particles (either may be NULL): out[4 s] = W = 1/2 sum m phi (the
 * potential energy of global.c:54, pre-G); out[4 s + 1..3] = sum m a, zero for
 * exact forces of an isolated system.  Masses as stored (FP32).  Blocking. */
gg_status gg_energy_device(gg_ctx *ctx, const double *d_acc, const double *d_pot, double *out);

/* ---- drift of the resident tree ----------------------------------------
 * Re-evaluation between rebuilds, as GIZMO does when TreeReconstructFlag is
 * not set: particles move by Vel*dt (drift_particle, predict.c:97-137) and
 * every node by force_drift_node (gravity/forcetree_update.c:265-338): centre
 * of mass s += vs*dt, side len += 2*vmax*dt, geometric centre unchanged, with
 * vs the node's mass-weighted mean velocity and vmax its largest |velocity
 * component| (gravity/forcetree.c:558-560, :629, :751).  Velocities are per
 * particle in load order (host arrays may be strided like the positions) and
 * stay until the next load of particles.  gg_drift moves every system by dt;
 * gg_drift_systems takes one dt per system (0 leaves a system where it is).
 * Drifts accumulate; the next gg_build rebuilds at the drifted positions.
 * Asynchronous on the context's stream (gg_drift_systems copies its host
 * array before returning). */
gg_status gg_load_velocities(gg_ctx *ctx, const double *vel, int64_t vel_stride_bytes);
gg_status gg_load_velocities_device(gg_ctx *ctx, const double *d_vel);
gg_status gg_drift(gg_ctx *ctx, double dt);
gg_status gg_drift_systems(gg_ctx *ctx, const double *dt);
/* The particles' current positions (load order, host, strided like
 * gg_load_particles) replace the resident ones without a rebuild; nodes are
 * left as they are.  For callers whose particles do not all move by Vel*dt
 * between rebuilds: the reference's walk reads P[].Pos, which drift_particle
 * (predict.c:97-137) advances by each build's own rule (advect_mesh_point for
 * MFV cells, super-timestepped binaries, frozen hydro), so GIZMO calls
 * gg_drift (nodes, by force_drift_node) and then gg_set_positions(P[].Pos).
 * A non-finite position makes the next evaluation return GG_ERR_BAD_INPUT.
 * Asynchronous on the context's stream (the host array has been read when it
 * returns). */
gg_status gg_set_positions(gg_ctx *ctx, const double *pos, int64_t pos_stride_bytes);

/* ---- batches of independent systems and asynchronous evaluation ----------
 * No counterpart in the reference, which holds one system per process.
 * gg_load_systems loads n_systems systems given as separate host arrays (one
 * pointer per system to its n*3 positions, n masses and n kernel radii),
 * gathered directly into the context's pinned staging buffer; the copy to the
 * device is asynchronous.  gg_load_system_velocities does the same for the
 * velocities the drift needs.
 * gg_evaluate_async queues the walk of `active` (host indices in load order,
 * NULL = all) and, per flags, the copy of the results into pinned buffers of
 * the context; it returns without waiting.  gg_query returns GG_PENDING while
 * that work runs and GG_OK when it is done; gg_fetch_results waits for it and
 * copies acc (n*3) and pot (n) out (nullable each) with the stats.  A later
 * gg_evaluate_async of the same context overwrites unfetched results. */
#define GG_ASYNC_COPY_ACC 1
#define GG_ASYNC_COPY_POT 2
gg_status gg_load_systems(gg_ctx *ctx, int32_t n_systems, const int64_t *counts, const double *const *pos,
                          const double *const *mass, const double *const *soft_h);
gg_status gg_load_system_velocities(gg_ctx *ctx, const double *const *vel);
gg_status gg_evaluate_async(gg_ctx *ctx, const int32_t *active, int64_t n_active, double err_tol_force_acc,
                            double err_tol_theta, int32_t flags);
gg_status gg_query(gg_ctx *ctx);
gg_status gg_fetch_results(gg_ctx *ctx, double *acc_out, double *pot_out, gg_stats *stats);
/* The same walk with the results copied straight into the caller's
 * page-locked host arrays (acc n*3, pot n; either may be NULL), so that
 * gg_fetch_results only waits and returns the stats (its acc_out and pot_out
 * must then be NULL).  The arrays must stay allocated until the fetch; a host
 * array that is not page-locked is refused with GG_ERR_INVALID.  A serving
 * loop that hands each request a view of its batch's result block saves the
 * copy out of the context's own pinned buffers, which otherwise takes a host
 * thread's time at memory bandwidth. */
gg_status gg_evaluate_async_pinned(gg_ctx *ctx, const int32_t *active, int64_t n_active, double err_tol_force_acc,
                                   double err_tol_theta, double *acc_pinned, double *pot_pinned);
/* Page-locked host blocks from the library's process-wide cache (the one its
 * contexts stage transfers through): gg_host_alloc returns a block of at least
 * `bytes`, gg_host_free gives it back to the cache (GG_ERR_INVALID for a
 * pointer gg_host_alloc did not return).  Thread-safe. */
gg_status gg_host_alloc(int64_t bytes, void **out);
gg_status gg_host_free(void *ptr);

/* ---- batched steps ------------------------------------------------------
 * No counterpart in the reference, which walks one system per process.  A
 * step of every resident system -- gg_build(ctx, NULL) then
 * gg_evaluate_device of all targets with d_acc_out / d_pot_out -- captured
 * once as a CUDA graph and replayed by gg_graph_launch on the context's
 * stream (set one with gg_set_stream first: the legacy default stream cannot
 * be captured).  Run one uncaptured build + evaluation with the same systems
 * before capturing, so that every buffer is allocated.  A replay re-reads the
 * particles last loaded into the same buffers and keeps the relative
 * criterion's OldAcc on the device between replays.  A graph holds the
 * device addresses of the context's buffers: once any of them has grown
 * (another system set, another configuration, a stack retry), gg_graph_launch
 * refuses the stale graph with GG_ERR_NOT_BUILT; capture again.  A capture
 * during which a buffer had to grow is refused the same way (step once
 * uncaptured first). */
gg_status gg_graph_capture_step(gg_ctx *ctx, double err_tol_force_acc, double err_tol_theta, double *d_acc_out,
                                double *d_pot_out);
gg_status gg_graph_launch(gg_ctx *ctx);
/* The same step captured as two graphs, part 0 the build and part 1 the walk,
 * replayed one after the other by gg_graph_launch_part, so that a caller can
 * time them apart with events between the launches.  Same rules as above. */
gg_status gg_graph_capture_parts(gg_ctx *ctx, double err_tol_force_acc, double err_tol_theta, double *d_acc_out,
                                 double *d_pot_out);
gg_status gg_graph_launch_part(gg_ctx *ctx, int32_t part);
/* Times the walk of the resident systems with the context's configuration
 * and over leaf size {8,16}, group size {32,64}, blocks per SM {2,3} and flush
 * threshold {64,128}, then the other node staging on the winner, each trial
 * from the same OldAcc, and keeps the fastest configuration that passes the
 * accuracy gate (rebuilding the tree with its leaf size); returns it in
 * *chosen and its walk time in *best_ms (nullable).  The gate: on a fixed
 * sample of targets (every target of a system of up to 2,048 particles, else
 * 16,384 / n_systems evenly spaced ones, at least 64 and at most 4,096)
 * against their FP64 direct sums, a candidate's 99th-percentile relative force
 * error over all sampled targets, and the largest of the systems' own 99th
 * percentiles, must each be at most 1.1x the context's own configuration's
 * (plus 1e-7), and the root mean square over systems of the sample potential
 * energy's (1/2 sum m phi) relative error at most 1.1x the context's own or
 * below 1e-5; so a faster configuration is never taken at the price of
 * accuracy.  No counterpart in the reference.  Synchronises. */
gg_status gg_autotune(gg_ctx *ctx, double err_tol_force_acc, double err_tol_theta, gg_config *chosen,
                      double *best_ms);
/* The same search for the walk of an active subset (device indices in load
 * order, as gg_evaluate_device takes them): individual timesteps walk sparser
 * groups of targets, whose best configuration differs from the all-target
 * walk's.  The gate's sample is drawn from the active targets. */
gg_status gg_autotune_active(gg_ctx *ctx, const int32_t *d_active, int64_t n_active, double err_tol_force_acc,
                             double err_tol_theta, gg_config *chosen, double *best_ms);
/* The accuracy gate of gg_autotune for one candidate configuration (leaf and
 * group size, flush threshold, blocks per SM, node staging, target and group
 * order) against the context's own, from the same OldAcc: *accepted = 1 if it
 * passes, else 0.  The context is left as it was.  Synchronises. */
gg_status gg_tune_accuracy(gg_ctx *ctx, double err_tol_force_acc, double err_tol_theta, const gg_config *candidate,
                           int32_t *accepted);

/* ---- kernel-level entry points (device pointers, cudaStream_t or NULL) ---- */
/* domain_double_to_int (domain.c:2504-2513) + peano_hilbert_key (peano.c:303-319)
 * at 21 bits per dimension: equals the reference's 42-bit key shifted right by 63 */
gg_status gg_peano_hilbert_keys(int64_t n, const double *d_pos, const gg_domain *dom, uint64_t *d_keys,
                                void *stream);
/* stable LSD radix sort of (key, value) pairs, replacing mysort_peano
 * (peano.c:414-462); key_bits <= 64; scratch is allocated by the call */
gg_status gg_radix_sort_pairs(int64_t n, uint64_t *d_keys, uint32_t *d_vals, int32_t key_bits, void *stream);
/* The same stable radix sort without any device allocation.  It has no
 * counterpart in the reference (whose sort runs on the host).  It is for
 * callers that cannot allocate device memory: a process whose device memory
 * is already reserved in full by another allocator (a framework's caching
 * allocator, a serving loop admitting work against a fixed memory budget)
 * would see cudaMalloc fail or bypass its accounting, and a latency-critical
 * loop cannot take cudaFree's implicit device synchronisation.  The scratch is
 * one static device array of the library (about 20 MB, held by every GPU that
 * loads the library until the process exits), so n is limited to
 * GG_NOALLOC_SORT_MAX_N; larger n returns GG_ERR_TOO_LARGE.  The first call on
 * a device looks up the array's device address; make that first call before
 * any stream capture.  The address is kept for the life of the process, so
 * after a cudaDeviceReset by the application the function must not be called
 * again.  d_keys and d_vals must be device memory of the current device
 * (GG_ERR_INVALID otherwise).  All calls share the array: calls whose work
 * overlaps on the GPU race and must not be issued.  Blocking (synchronises
 * `stream`). */
#define GG_NOALLOC_SORT_MAX_N (1 << 20)
gg_status gg_radix_sort_pairs_noalloc(int64_t n, uint64_t *d_keys, uint32_t *d_vals, int32_t key_bits, void *stream);
/* Self-test of the library's only device-side wait, the radix sort's
 * look-back: one sort pass is run as the second tile of a two-tile pass whose
 * first tile never runs, so the wait cannot complete.  It gives up after its
 * poll limit (about a second) and the call returns GG_ERR_TIMEOUT, which is
 * the expected result; the device stays usable.  No counterpart in the
 * reference (its sort runs on the host).  Blocking. */
gg_status gg_selftest_bounded_wait(void *stream);
/* FP64 direct summation over all sources with the walk's pair rule (the
 * reference declares force_treeevaluate_direct, gravity/forcetree.h:76, but
 * ships no definition); used to measure force errors at full size */
gg_status gg_direct_sum_fp64(int64_t n_src, const double *d_pos, const double *d_mass, const double *d_h,
                             int64_t n_tgt, const int32_t *d_targets, double *d_acc, double *d_pot, void *stream);

/* measured FP32 FMA throughput of the device in TFLOP/s (2 flops per FMA):
 * the CUDA-core roofline the walk is reported against */
gg_status gg_fp32_peak_probe(double *tflops, void *stream);
/* kernels this library has launched in this process (all contexts) */
int64_t gg_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
