// gg_drift.cu -- re-evaluation of a resident tree after a drift, without a rebuild.
//
// GIZMO keeps its tree between rebuilds and moves it with the particles:
// drift_particle (predict.c:97-137) moves a particle by Vel*dt, and
// force_drift_node (gravity/forcetree_update.c:265-338) moves a node's centre
// of mass by vs*dt and grows its side by 2*vmax*dt, leaving the geometric
// centre where it was.  vs is the node's mass-weighted mean velocity and vmax
// the largest |velocity component| of its particles
// (force_update_node_recursive, gravity/forcetree.c:558-560, :629, :751,
// :764-781).  The reference drifts lazily when the walk first reaches a node;
// drifting every node once before the walk gives the same tree.
//
// Three kernels: node kinematics (bottom-up like the moments, once per build
// or velocity load), the particle drift (load-order records and the sorted
// copy the walk reads, both updated) and the node drift.  Products are rounded
// separately from sums (no fused multiply-add), like the reference's FP64
// expressions.
#include "gg_internal.cuh"
#include "gg_kernels.cuh"

// Bottom-up velocity moments: each leaf sums its particles; the last child to
// finish computes its parent (children summed in index order, so the result
// does not depend on scheduling).  kin[k] = {vs.x, vs.y, vs.z, vmax}.
// keep_max: velocities were reloaded since the tree's last kinematics; vmax
// keeps the largest value seen since the build, as kicks only ever raise it in
// the reference (force_kick_node, gravity/forcetree_update.c).
__global__ void k_node_kinematics(const GGPart *__restrict__ parts, const unsigned *__restrict__ perm,
                                  const double *__restrict__ vel, TreeBuf tb, int *__restrict__ counter,
                                  double4 *__restrict__ kin, int n, int keep_max)
{
    const int total = tb.nnodes[0];
    for (int k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < total; k0 += gridDim.x * blockDim.x) {
        if (tb.child[k0] >= 0) continue;   // only leaves start a climb
        int k = k0;
        bool is_leaf = true;
        for (;;) {
            double M = 0, vx = 0, vy = 0, vz = 0, vmax = 0;
            if (is_leaf) {
                for (int i = tb.start[k]; i < tb.end[k]; i++) {
                    unsigned j = perm[i];
                    if (j >= (unsigned)n) j = 0;
                    const double m = (double)parts[i].m;
                    const double ux = vel[3 * (size_t)j], uy = vel[3 * (size_t)j + 1], uz = vel[3 * (size_t)j + 2];
                    M = __dadd_rn(M, m);
                    vx = __dadd_rn(vx, __dmul_rn(m, ux));
                    vy = __dadd_rn(vy, __dmul_rn(m, uy));
                    vz = __dadd_rn(vz, __dmul_rn(m, uz));
                    vmax = fmax(vmax, fmax(fabs(ux), fmax(fabs(uy), fabs(uz))));
                }
            } else {
                const int c0 = tb.child[k], nc = tb.nch[k];
                for (int c = c0; c < c0 + nc; c++) {
                    const double m = __ldcg(tb.mass64 + c);
                    // written by another thread of this launch: read through L2
                    const double2 q01 = __ldcg(reinterpret_cast<const double2 *>(kin + c));
                    const double2 q23 = __ldcg(reinterpret_cast<const double2 *>(kin + c) + 1);
                    const double4 q = make_double4(q01.x, q01.y, q23.x, q23.y);
                    M = __dadd_rn(M, m);
                    vx = __dadd_rn(vx, __dmul_rn(m, q.x));
                    vy = __dadd_rn(vy, __dmul_rn(m, q.y));
                    vz = __dadd_rn(vz, __dmul_rn(m, q.z));
                    vmax = fmax(vmax, q.w);
                }
            }
            if (keep_max) vmax = fmax(vmax, kin[k].w);   // this thread alone writes node k
            double4 out;
            if (M > 0) { out.x = __ddiv_rn(vx, M); out.y = __ddiv_rn(vy, M); out.z = __ddiv_rn(vz, M); }
            else { out.x = out.y = out.z = 0.0; }
            out.w = vmax;
            kin[k] = out;
            const int par = tb.parent[k];
            if (par < 0) break;
            __threadfence();
            const int old = atomicAdd(counter + par, 1);
            if (old != tb.nch[par] - 1) break;
            __threadfence();
            k = par;
            is_leaf = false;
        }
    }
}

// system of sorted particle i: poff is ascending with poff[0] = 0, poff[S] = n
__device__ __forceinline__ int system_of(const int *__restrict__ poff, int S, int i)
{
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(poff + mid) <= i) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// x += v*dt for every particle (drift_particle, predict.c:135)
__global__ void k_drift_particles(GGPart *__restrict__ in_rec, GGPart *__restrict__ parts,
                                  const unsigned *__restrict__ perm, const double *__restrict__ vel,
                                  const int *__restrict__ poff, int S, const double *__restrict__ dts, double dt_all,
                                  int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double dt = dts ? dts[system_of(poff, S, i)] : dt_all;
        if (dt == 0.0) continue;
        unsigned j = perm[i];
        if (j >= (unsigned)n) continue;   // only after a failed sort, which is reported
        GGPart p = in_rec[j];
        p.x = __dadd_rn(p.x, __dmul_rn(vel[3 * (size_t)j], dt));
        p.y = __dadd_rn(p.y, __dmul_rn(vel[3 * (size_t)j + 1], dt));
        p.z = __dadd_rn(p.z, __dmul_rn(vel[3 * (size_t)j + 2], dt));
        in_rec[j] = p;
        parts[i] = p;
    }
}

// The caller's current positions (load order, FP64 xyz) into the load-order
// records and the sorted copy the walk reads; the tree is kept.  A non-finite
// position is refused (error bit) and leaves that particle where it was.
__global__ void k_set_positions(GGPart *__restrict__ in_rec, GGPart *__restrict__ parts,
                                const unsigned *__restrict__ perm, const double *__restrict__ pos, int n,
                                int *__restrict__ err)
{
    bool bad = false;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned j = perm[i];
        if (j >= (unsigned)n) continue;   // only after a failed sort, which is reported
        const double x = pos[3 * (size_t)j], y = pos[3 * (size_t)j + 1], z = pos[3 * (size_t)j + 2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) { bad = true; continue; }
        GGPart p = in_rec[j];
        p.x = x; p.y = y; p.z = z;
        in_rec[j] = p;
        parts[i] = p;
    }
    if (bad) atomicOr(err, GG_EBIT_BAD_INPUT);
}

// s += vs*dt, len += 2*vmax*dt, geometric centre fixed (force_drift_node)
__global__ void k_drift_nodes(GGNode *__restrict__ nodes, const double4 *__restrict__ kin, const int *__restrict__ sys,
                              const int *__restrict__ nnodes, const double *__restrict__ dts, double dt_all)
{
    const int total = nnodes[0];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const double dt = dts ? dts[sys[k]] : dt_all;
        if (dt == 0.0) continue;
        const double4 q = kin[k];
        GGNode nd = nodes[k];
        const double mx = __dmul_rn(q.x, dt), my = __dmul_rn(q.y, dt), mz = __dmul_rn(q.z, dt);
        nd.cx = __dadd_rn(nd.cx, mx);
        nd.cy = __dadd_rn(nd.cy, my);
        nd.cz = __dadd_rn(nd.cz, mz);
        nd.gx = (float)__dsub_rn((double)nd.gx, mx);
        nd.gy = (float)__dsub_rn((double)nd.gy, my);
        nd.gz = (float)__dsub_rn((double)nd.gz, mz);
        nd.len = (float)__dadd_rn((double)nd.len, __dmul_rn(2.0 * q.w, dt));
        nodes[k] = nd;
    }
}

static int grid_for(long long n, int threads)
{
    long long blocks = (n + threads - 1) / threads, cap = (long long)gg_num_sms() * 8;
    if (blocks > cap) blocks = cap;
    return blocks < 1 ? 1 : (int)blocks;
}

void gg_launch_node_kinematics(const GGPart *parts, const unsigned *perm, const double *vel, TreeBuf tb, int *counter,
                               double4 *kin, int n, int ncap, int keep_max, cudaStream_t st)
{
    k_node_kinematics<<<grid_for(ncap, 256), 256, 0, st>>>(parts, perm, vel, tb, counter, kin, n, keep_max);
    gg_note_launches(1);
}

void gg_launch_drift(GGPart *in_rec, GGPart *parts, const unsigned *perm, const double *vel, const int *poff, int S,
                     const double *dts, double dt_all, GGNode *nodes, const double4 *kin, const int *node_sys, const int *nnodes,
                     int n, int ncap, cudaStream_t st)
{
    if (n > 0) {
        k_drift_particles<<<grid_for(n, 256), 256, 0, st>>>(in_rec, parts, perm, vel, poff, S, dts, dt_all, n);
        gg_note_launches(1);
    }
    k_drift_nodes<<<grid_for(ncap, 256), 256, 0, st>>>(nodes, kin, node_sys, nnodes, dts, dt_all);
    gg_note_launches(1);
}

void gg_launch_set_positions(GGPart *in_rec, GGPart *parts, const unsigned *perm, const double *pos, int n, int *err,
                             cudaStream_t st)
{
    if (n < 1) return;
    k_set_positions<<<grid_for(n, 256), 256, 0, st>>>(in_rec, parts, perm, pos, n, err);
    gg_note_launches(1);
}
