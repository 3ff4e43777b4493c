// gg_kernels.cuh -- launch functions shared between the kernel files and the API.
#pragma once
#include "gg_internal.cuh"

#define GG_SORT_MAX_PASSES 12

// per-node build arrays (device pointers), capacity `cap` nodes
struct TreeBuf {
    int *start, *end, *level, *parent, *sys, *nch, *child;
    int *bnd;          // 8 digit boundaries per node
    double *mass64;    // FP64 node mass (parent sums)
    int *depth_beg;    // GG_MAX_DEPTH + 2 entries
    int *nnodes;       // total nodes (device)
    unsigned *bstat;   // per depth and block: published children totals (GG_MAX_DEPTH x grid)
    unsigned *ticket;  // per depth: block tickets
    int cap;           // node capacity (set by gg_launch_tree)
    int *err;
};

void gg_launch_extent(const GGPart *rec, int n, const int *poff, int S, unsigned long long *mm, unsigned *hmm,
                      GGDomainDev *dom, int *err, cudaStream_t st);
void gg_launch_keys(const GGPart *rec, int n, const int *poff, int S, const GGDomainDev *dom,
                    unsigned long long *keys, unsigned *vals, int *err, cudaStream_t st);
void gg_launch_keys_plain(const double *pos, long long n, const GGDomainDev &d, unsigned long long *keys, int *err,
                          cudaStream_t st);

size_t gg_sort_scratch_bytes(long long n);
int gg_sort_bits();
// Records moved by the last pass of a sort whose values are record indices:
// out[position] = in[value], rank[value] = position.
struct SortGather {
    const GGPart *in;
    GGPart *out;
    unsigned *rank;
};
// gather (nullable): done by the last pass; *gathered says whether it was (no
// pass runs for n <= 1 or no bits).
gg_status gg_sort_pairs_run(unsigned long long *keys, unsigned *vals, long long n, int key_bits, int sys_bits,
                            const int *poff, int S, void *scratch, int *err, cudaStream_t st,
                            const SortGather *gather = nullptr, bool *gathered = nullptr);

void gg_launch_permute(const unsigned *perm, const GGPart *in, GGPart *out, unsigned *rank, int n, cudaStream_t st);
int gg_tree_grid();
void gg_launch_tree(const unsigned long long *keys, const int *poff, int S, int leaf, int cap, TreeBuf tb,
                    const GGPart *parts, const GGDomainDev *dom, GGNode *nodes, cudaStream_t st);

struct WalkParams {
    const GGNode *nodes;
    const GGPart *parts;        // sorted
    const GGGroup *groups;
    const int *ngroups;         // device count
    const int *tlist;           // sorted particle index per target, NULL = identity
    const int *tout;            // output slot per target, NULL = load-order index of the particle
    const unsigned *perm;       // sorted position -> load-order index
    const double *oldacc_in;    // per particle (load order), NULL = 0
    double *oldacc_out;         // per particle (load order), may be NULL
    double tol, theta;
    double *acc;                // 3 per output slot
    double *pot;                // per output slot, may be NULL
    int *ninter;                // per output slot, may be NULL
    unsigned long long *interactions;   // [0] interactions, [1] far / [2] near list entries, [3] nodes tested
    int *group_counter;
    int *stack;
    int stack_cap;
    int *err;
    int group_size;
    int flush;
    int pot_only;               // potential-only walk: acc and oldacc_out unused, pot required
    const unsigned *gorder;     // order in which groups are handed out, NULL = index order
    float *cost_out;            // per particle (load order): its group's cycles per target, may be NULL
    int node_staging;           // 0: per-lane cp.async, 1: bulk copies (TMA) per run of consecutive nodes
};
int gg_walk_smem_bytes(int flush, int tpl);
void gg_launch_walk(const WalkParams &p, int tpl, int blocks_per_sm, cudaStream_t st);
int gg_walk_threads();

// groups of `gs` consecutive targets per system; toff[S+1] target offsets per system
void gg_launch_groups(const int *toff, int S, int gs, GGGroup *groups, int *ngroups, int *gscan, cudaStream_t st);
long long gg_max_groups(long long n, int S, int gs);
int gg_target_order_lmax(int S);
void gg_launch_groups_tree(int nt, const int *tlist, const int *tscan, const int *toff, int S, int gs,
                           const TreeBuf &tb, const GGDomainDev *order_dom, const unsigned *hmm, int lmax, int *gnode,
                           int *flag, int *seg, int *segstart, int maxg, GGGroup *groups, int *ngroups,
                           int *scan_scratch, int *err, cudaStream_t st);
// exclusive scan of n ints (scratch: 2 * (gg_num_sms()*4) ints)
void gg_launch_scan(const int *in, int *out, int n, int *scratch, cudaStream_t st);
// active targets: flags in sorted order -> tlist/tout, and per-system offsets
void gg_launch_active(const int *active, int n_active, const unsigned *rank, int n, int *flag, int *flagscan,
                      int *tlist, int *tout, const int *poff, int S, int *toff, int *scratch, int *err,
                      cudaStream_t st);
int gg_scan_scratch_ints();
// walk groups sorted by the summed previous cost of their targets, most
// expensive first: gorder[0..maxg) (groups past the device count sort last)
gg_status gg_order_groups_by_cost(const GGGroup *groups, const int *ngroups, int maxg, const int *tlist,
                                  const unsigned *perm, const float *cost, unsigned long long *key,
                                  unsigned *gorder, void *sort_scratch, int *err, cudaStream_t st);
// targets reordered by (system, kernel radius), key order kept within a class
gg_status gg_order_targets_by_softening(int nt, const int *tlist_in, const int *tout_in, const GGPart *parts,
                                        const unsigned long long *pkeys, const int *poff, int S,
                                        const GGDomainDev *dom, const unsigned *hmm, unsigned long long *key,
                                        unsigned *val, int *tlist_out, int *tout_out, void *sort_scratch, int *err,
                                        cudaStream_t st);

void gg_launch_direct_records(const GGPart *rec, const int *poff, const int2 *tg, int ntg, double *acc, double *pot,
                              double *mass, cudaStream_t st);
void gg_launch_gather_rows(const double *acc, const double *pot, const int2 *tg, int ntg, double *acc_out,
                           double *pot_out, cudaStream_t st);
void gg_launch_direct(long long n_src, const double *pos, const double *mass, const double *h, long long n_tgt,
                      const int *targets, double *acc, double *pot, cudaStream_t st);

// drift of a resident tree (gg_drift.cu)
void gg_launch_node_kinematics(const GGPart *parts, const unsigned *perm, const double *vel, TreeBuf tb, int *counter,
                               double4 *kin, int n, int ncap, int keep_max, cudaStream_t st);
void gg_launch_set_positions(GGPart *in_rec, GGPart *parts, const unsigned *perm, const double *pos, int n, int *err,
                             cudaStream_t st);
void gg_launch_drift(GGPart *in_rec, GGPart *parts, const unsigned *perm, const double *vel, const int *poff, int S,
                     const double *dts, double dt_all, GGNode *nodes, const double4 *kin, const int *node_sys, const int *nnodes,
                     int n, int ncap, cudaStream_t st);

// FP64 per-system sums {1/2 sum m phi, sum m a} (gg_util.cu)
void gg_launch_energy(const int4 *chunks, int nchunks, const int *sys_first_chunk, int S, const GGPart *rec,
                      const double *acc, const double *pot, double *part, double *out, cudaStream_t st);

// bounded look-back self-test (gg_sort.cu)
gg_status gg_sort_timeout_selftest(cudaStream_t st);
