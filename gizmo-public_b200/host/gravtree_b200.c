/*
 * gravtree_b200.c -- GIZMO-side host code of the B200 tree-gravity path.
 *
 * This file is compiled inside a GIZMO build (it includes GIZMO's allvars.h
 * and proto.h) with the compile flag GRAVITY_GPU_B200 and linked with
 * libgizmo_gravity_b200.so.  It replaces, inside gravity_tree()
 * (gravity/gravtree.c:51-654), the tree construction block (gravtree.c:67-78,
 * force_treebuild) and the local walk / export loop (gravtree.c:138-457,
 * force_treeevaluate per active particle), and leaves everything else to the
 * reference: the post-processing (x G, OldAcc, switch to the relative
 * criterion, gravtree.c:475-602), kicks, timesteps and the active list.
 *
 * Particle data is passed straight out of P[] with its record stride, so
 * nothing is copied on the host except the per-particle kernel radii
 * (ForceSoftening_KernelRadius, proto.h:134-155) and the active index list
 * (the FirstActiveParticle / NextActiveParticle chain, run.c:473-496).
 * Between rebuilds the reference's walk drifts particles and nodes to the
 * current time itself (drift_particle and force_drift_node, called lazily at
 * forcetree.c:1841 and :2051-2057); here the resident device tree's nodes are
 * drifted instead, with the current P[].Vel, over the interval since the
 * previous walk, and its particles take the current P[].Pos.  Single MPI rank
 * per GPU.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "allvars.h"
#include "proto.h"

#include "gizmo_gravity_b200.h"

static gg_ctx *gg_tree_ctx = NULL;
static double *gg_soft = NULL, *gg_oldacc = NULL, *gg_acc = NULL, *gg_pot = NULL;
static int32_t *gg_active = NULL;
static long gg_cap = 0;
static integertime gg_tree_ti = 0;   /* integer time the device tree's positions belong to */

static void gg_fail(const char *what, gg_status st)
{
    printf("B200 gravity: %s failed: %s (%d)\n", what, gg_strerror(st), st);
    endrun(3131);
}

static void gg_reserve(long n)
{
    if (n <= gg_cap) return;
    gg_cap = n + n / 4 + 1024;
    gg_soft = (double *)realloc(gg_soft, gg_cap * sizeof(double));
    gg_oldacc = (double *)realloc(gg_oldacc, gg_cap * sizeof(double));
    gg_acc = (double *)realloc(gg_acc, 3 * gg_cap * sizeof(double));
    gg_pot = (double *)realloc(gg_pot, gg_cap * sizeof(double));
    gg_active = (int32_t *)realloc(gg_active, gg_cap * sizeof(int32_t));
    if (!gg_soft || !gg_oldacc || !gg_acc || !gg_pot || !gg_active) {
        printf("B200 gravity: host allocation of %ld entries failed\n", gg_cap);
        endrun(3132);
    }
}

/* Tree construction: replaces force_treebuild(NumPart, NULL) (gravtree.c:74). */
void gravtree_b200_build(void)
{
    gg_status st;
    int i;
    if (NTask != 1) {
        printf("B200 gravity: one MPI rank per GPU (NTask = %d)\n", NTask);
        endrun(3133);
    }
    if (!gg_tree_ctx) {
        gg_config cfg;
        gg_config_default(&cfg);
        if ((st = gg_create(&cfg, &gg_tree_ctx))) gg_fail("gg_create", st);
    }
    gg_reserve(NumPart);
    for (i = 0; i < NumPart; i++) gg_soft[i] = ForceSoftening_KernelRadius(i);
    int64_t count = NumPart;
    st = gg_load_particles(gg_tree_ctx, 1, &count, &P[0].Pos[0], (int64_t)sizeof(struct particle_data), &P[0].Mass,
                           (int64_t)sizeof(struct particle_data), gg_soft, (int64_t)sizeof(double));
    if (st) gg_fail("gg_load_particles", st);
    if ((st = gg_build(gg_tree_ctx, NULL))) gg_fail("gg_build", st);
    gg_tree_ti = All.Ti_Current;
}

/* Bring the resident tree to All.Ti_Current without a rebuild: nodes move by
 * force_drift_node (forcetree_update.c:265-338) with the current velocities,
 * and the particles take their current P[].Pos.  The reference's walk reads
 * P[].Pos, which drift_particle (predict.c:97-137) has already brought to the
 * current time -- by Vel*dt for most particles, but by each build's own rule
 * where there is one (advect_mesh_point for MFV cells, super-timestepped
 * binaries, frozen hydro) -- so the positions are taken from P[] rather than
 * drifted here.  Velocities do not change between two walks (kicks come after
 * the force computation), so one node drift per walk interval with the
 * current velocities follows the reference's lazy node drift. */
static void gravtree_b200_drift(void)
{
    gg_status st;
    if (All.Ti_Current == gg_tree_ti) return;
    double dt = All.ComovingIntegrationOn ? get_drift_factor(gg_tree_ti, All.Ti_Current)
                                          : (All.Ti_Current - gg_tree_ti) * All.Timebase_interval;
    st = gg_load_velocities(gg_tree_ctx, &P[0].Vel[0], (int64_t)sizeof(struct particle_data));
    if (st) gg_fail("gg_load_velocities", st);
    if ((st = gg_drift(gg_tree_ctx, dt))) gg_fail("gg_drift", st);
    st = gg_set_positions(gg_tree_ctx, &P[0].Pos[0], (int64_t)sizeof(struct particle_data));
    if (st) gg_fail("gg_set_positions", st);
    gg_tree_ti = All.Ti_Current;
}

/* Peano-Hilbert order of P[] on the GPU: replaces the sort of
 * peano_hilbert_order (system/peano.c:28-92), called from
 * domain_Decomposition (domain.c:275).  Gas cells [0, N_gas) and the other
 * particles are ordered separately, as there, by their key in GIZMO's domain
 * cube (DomainCorner, DomainLen); the library sorts the two blocks as two
 * systems that share that cube.  The permutation is then applied in place by
 * following its cycles, to P[] and, for gas, SphP[] (the reference's
 * reorder_particles / reorder_gas do the same moves with their own index
 * table).  Particles that share a 21-bit cell keep their relative order here
 * (the reference orders them by finer key bits).  Invalidates the device tree:
 * call it before the tree is built, as domain_Decomposition does. */
static void gg_apply_order(const int32_t *order, long first, long n, int with_sph, int *dest)
{
    long k;
    for (k = 0; k < n; k++) dest[order[first + k] - first] = (int)k;   /* new slot of each old slot */
    for (k = 0; k < n; k++) {
        while (dest[k] != k) {   /* send the record in slot k to its slot, take what was there */
            int d = dest[k];
            struct particle_data tp = P[first + d];
            P[first + d] = P[first + k];
            P[first + k] = tp;
            if (with_sph) {
                struct gas_cell_data ts = SphP[first + d];
                SphP[first + d] = SphP[first + k];
                SphP[first + k] = ts;
            }
            dest[k] = dest[d];
            dest[d] = d;
        }
    }
}

void peano_hilbert_order_b200(void)
{
    gg_status st;
    int i, k, S = 0;
    if (!gg_tree_ctx) {
        gg_config cfg;
        gg_config_default(&cfg);
        if ((st = gg_create(&cfg, &gg_tree_ctx))) gg_fail("gg_create", st);
    }
    gg_reserve(NumPart);
    for (i = 0; i < NumPart; i++) gg_soft[i] = ForceSoftening_KernelRadius(i);
    int64_t counts[2];
    long first[2];
    if (N_gas > 0) { counts[S] = N_gas; first[S] = 0; S++; }
    if (NumPart - N_gas > 0) { counts[S] = NumPart - N_gas; first[S] = N_gas; S++; }
    if (S == 0) return;
    st = gg_load_particles(gg_tree_ctx, S, counts, &P[0].Pos[0], (int64_t)sizeof(struct particle_data), &P[0].Mass,
                           (int64_t)sizeof(struct particle_data), gg_soft, (int64_t)sizeof(double));
    if (st) gg_fail("gg_load_particles", st);
    gg_domain dom[2];
    for (k = 0; k < S; k++) {
        int j;
        for (j = 0; j < 3; j++) {
            dom[k].center[j] = DomainCenter[j];
            dom[k].corner[j] = DomainCorner[j];
        }
        dom[k].len = DomainLen;
    }
    if ((st = gg_build(gg_tree_ctx, dom))) gg_fail("gg_build", st);
    int32_t *order = (int32_t *)malloc(sizeof(int32_t) * (NumPart ? NumPart : 1));
    int *dest = (int *)malloc(sizeof(int) * (NumPart ? NumPart : 1));
    if (!order || !dest) {
        printf("B200 gravity: host allocation for the Peano-Hilbert order failed\n");
        endrun(3134);
    }
    if ((st = gg_get_order(gg_tree_ctx, order))) gg_fail("gg_get_order", st);
    for (k = 0; k < S; k++) gg_apply_order(order, first[k], (long)counts[k], first[k] == 0 && N_gas > 0, dest);
    free(dest);
    free(order);
}

/* Local walk: replaces the force_treeevaluate loop over the active particles
 * (gravtree.c:138-457).  Leaves the pre-G force and potential in P[] like the
 * reference's walk does (forcetree.c:2661-2701) and returns the interaction
 * count (the reference's Costtotal). */
double gravtree_b200_walk(void)
{
    gg_status st;
    int i;
    long n = 0;
    gg_reserve(NumPart);
    gravtree_b200_drift();
    for (i = FirstActiveParticle; i >= 0; i = NextActiveParticle[i]) gg_active[n++] = i;
    for (i = 0; i < NumPart; i++) gg_oldacc[i] = P[i].OldAcc;
    gg_stats stats;
    st = gg_evaluate(gg_tree_ctx, gg_active, n, gg_oldacc, All.ErrTolForceAcc, All.ErrTolTheta, gg_acc, gg_pot, NULL,
                     &stats);
    if (st) gg_fail("gg_evaluate", st);
    for (long k = 0; k < n; k++) {
        i = gg_active[k];
        P[i].GravAccel[0] = gg_acc[3 * k];
        P[i].GravAccel[1] = gg_acc[3 * k + 1];
        P[i].GravAccel[2] = gg_acc[3 * k + 2];
#ifdef EVALPOTENTIAL
        P[i].Potential = gg_pot[k];
#endif
    }
    return (double)stats.interactions;
}
