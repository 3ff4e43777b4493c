/*
 * gg_oracle.c -- CPU oracle for GIZMO's tree-gravity force evaluation.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C and FP64, the
 * algorithm of the reference's tree-gravity path so that the CUDA library can
 * be checked against it.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the product path never links or calls it.
 *
 * What it restates (paths are within the GIZMO source tree):
 *   - domain_findExtent          domain.c:2518-2570  (root cube, len*1.001)
 *   - domain_double_to_int       domain.c:2504-2513  (mantissa quantisation)
 *   - peano_hilbert_key          system/peano.c:303-319, written here from the
 *                                curve's generator (base octant order and the
 *                                eight child orientations) instead of the
 *                                reference's 48x8 lookup tables
 *   - morton_key                 system/peano.c:323-335
 *   - force_treebuild_single     gravity/forcetree.c:152-342 (one particle per
 *                                leaf, Morton digits for the first 42 levels,
 *                                geometric comparisons below)
 *   - force_update_node_recursive gravity/forcetree.c:434-942 (mass, centre of
 *                                mass, maxsoft, multiple-particle flag)
 *   - force_treeevaluate         gravity/forcetree.c:1633-2807 (opening rules
 *                                :2026-2158, softened interaction :2258-2366)
 *   - kernel_gravity (cubic)     kernel.h:389-487
 *   - FP64 direct summation with the same pair rule (the reference declares
 *     force_treeevaluate_direct at gravity/forcetree.h:76 but defines none).
 *
 * Differences from the reference, none of which changes a force:
 *   - the domain's empty top-level nodes (force_create_empty_nodes,
 *     forcetree.c:353-400) are not created: empty nodes are skipped by the walk
 *     and a top node holding one particle is always opened, so the interaction
 *     set is the same;
 *   - near-coincident particles (node len < 1e-4 h, forcetree.c:219-231) get a
 *     hashed sub-node instead of a GSL random number.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ extent */

void oracle_find_extent(int64_t n, const double *pos, double *center, double *corner, double *len_out)
{
    double xmin[3], xmax[3], len = 0;
    for (int j = 0; j < 3; j++) { xmin[j] = 1e56; xmax[j] = -1e56; }
    for (int64_t i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) {
            double v = pos[3 * i + j];
            if (xmin[j] > v) xmin[j] = v;
            if (xmax[j] < v) xmax[j] = v;
        }
    for (int j = 0; j < 3; j++)
        if (xmax[j] - xmin[j] > len) len = xmax[j] - xmin[j];
    len *= 1.001;
    for (int j = 0; j < 3; j++) {
        center[j] = 0.5 * (xmin[j] + xmax[j]);
        corner[j] = 0.5 * (xmin[j] + xmax[j]) - 0.5 * len;
    }
    *len_out = len;
}

/* top `bits` bits of the mantissa of d, d in [1,2) */
uint64_t oracle_double_to_int(double d, int bits)
{
    uint64_t u;
    memcpy(&u, &d, 8);
    return (u & 0xFFFFFFFFFFFFFull) >> (52 - bits);
}

/* ------------------------------------------------------------- PH keys */

/* An orientation is a signed axis permutation acting on octant bits
 * (b0=x, b1=y, b2=z as the 4/2/1 bits of pix): out[i] = in[perm[i]] ^ flip[i]. */
typedef struct { int perm[3]; int flip[3]; } orient_t;

static const int ph_order0[8] = {0, 2, 6, 4, 5, 7, 3, 1};
static const orient_t ph_child[8] = {
    {{0, 2, 1}, {0, 0, 0}}, {{2, 1, 0}, {0, 0, 0}}, {{2, 1, 0}, {0, 0, 0}}, {{0, 1, 2}, {1, 1, 0}},
    {{0, 1, 2}, {1, 1, 0}}, {{2, 1, 0}, {1, 0, 1}}, {{2, 1, 0}, {1, 0, 1}}, {{0, 2, 1}, {0, 1, 1}}};

static int orient_apply(const orient_t *g, int pix)
{
    int b[3] = {(pix >> 2) & 1, (pix >> 1) & 1, pix & 1}, o[3];
    for (int i = 0; i < 3; i++) o[i] = b[g->perm[i]] ^ g->flip[i];
    return o[0] * 4 + o[1] * 2 + o[2];
}

/* (g o h): out = g(h(in)) */
static orient_t orient_compose(const orient_t *g, const orient_t *h)
{
    orient_t r;
    for (int i = 0; i < 3; i++) {
        r.perm[i] = h->perm[g->perm[i]];
        r.flip[i] = h->flip[g->perm[i]] ^ g->flip[i];
    }
    return r;
}

/* Peano-Hilbert key of integer coordinates with `bits` bits each (<=42):
 * returns the 3*bits-bit key, MSB-first like peano.c:309-316. */
static u128 ph_key128(uint64_t x, uint64_t y, uint64_t z, int bits)
{
    orient_t g = {{0, 1, 2}, {0, 0, 0}};
    u128 key = 0;
    for (int lev = bits - 1; lev >= 0; lev--) {
        int pix = (int)((((x >> lev) & 1) << 2) | (((y >> lev) & 1) << 1) | ((z >> lev) & 1));
        int k = 0;
        while (orient_apply(&g, ph_order0[k]) != pix) k++;
        key = (key << 3) | (u128)k;
        g = orient_compose(&g, &ph_child[k]);
    }
    return key;
}

/* keys for n positions in the given root cube; bits <= 42 per dimension.
 * key_hi/key_lo receive the high and low 64-bit words of the key. */
void oracle_ph_keys(int64_t n, const double *pos, const double *corner, double len, int bits, uint64_t *key_hi,
                    uint64_t *key_lo)
{
    for (int64_t i = 0; i < n; i++) {
        uint64_t q[3];
        for (int j = 0; j < 3; j++) q[j] = oracle_double_to_int(((pos[3 * i + j] - corner[j]) / len) + 1.0, bits);
        u128 k = ph_key128(q[0], q[1], q[2], bits);
        key_hi[i] = (uint64_t)(k >> 64);
        key_lo[i] = (uint64_t)k;
    }
}

/* ------------------------------------------------------ spline kernel */

/* cubic-spline softened gravity (kernel.h:452-470); mode 1 = force factor,
 * mode -1 = potential; u = r/h in [0,1). */
static double spline_gravity(double u, double hinv, double hinv3, int mode)
{
    if (u >= 1) {
        if (mode == 1) return hinv3 / (u * u * u);
        return -hinv / u;
    }
    if (mode == 1) {
        double w = (u < 0.5) ? (10.666666666667 + u * u * (32.0 * u - 38.4))
                             : (21.333333333333 - 48.0 * u + 38.4 * u * u - 10.666666666667 * u * u * u -
                                0.066666666667 / (u * u * u));
        return w * hinv3;
    } else {
        double w = (u < 0.5) ? (-2.8 + u * u * (5.333333333333 + u * u * (6.4 * u - 9.6)))
                             : (-3.2 + 0.066666666667 / u +
                                u * u * (10.666666666667 + u * (-16.0 + u * (9.6 - 2.133333333333 * u))));
        return w * hinv;
    }
}

double oracle_spline_gravity(double u, double hinv, double hinv3, int mode)
{
    return spline_gravity(u, hinv, hinv3, mode);
}

/* pair term shared by the tree walk and the direct sum (forcetree.c:2258-2283) */
static inline void pair_term(double dx, double dy, double dz, double r2, double mass, double h, double h_p,
                             double *ax, double *ay, double *az, double *pot)
{
    double r = sqrt(r2), fac, facpot;
    if (r >= h && r >= h_p) {
        fac = mass / (r2 * r);
        facpot = -mass / r;
    } else {
        double hg = h;
        if (h_p > hg) hg = h_p;
        double hinv = 1. / hg, h3inv = hinv * hinv * hinv, u = r * hinv;
        fac = mass * spline_gravity(u, hinv, h3inv, 1);
        facpot = mass * spline_gravity(u, hinv, h3inv, -1);
    }
    *pot += facpot;
    *ax += dx * fac;
    *ay += dy * fac;
    *az += dz * fac;
}

/* ------------------------------------------------------------ octree */

typedef struct {
    double center[3], len;
    double s[3], mass, maxsoft;
    double vs[3], vmax;   /* mass-weighted mean velocity, largest |velocity component| (drift only) */
    int suns[8];   /* <n: particle, >=n: node n+idx, -1: empty */
    int multiple;  /* more than one particle below */
} onode_t;

typedef struct {
    int64_t n;
    const double *pos, *mass, *h;
    const double *vel;    /* NULL unless the tree is drifted */
    onode_t *nodes;
    int64_t nnodes, cap;
} otree_t;

static int new_node(otree_t *t, const double *center, double len)
{
    if (t->nnodes == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->nodes = (onode_t *)realloc(t->nodes, sizeof(onode_t) * t->cap);
    }
    onode_t *nd = &t->nodes[t->nnodes];
    memset(nd, 0, sizeof(*nd));
    for (int j = 0; j < 3; j++) nd->center[j] = center[j];
    nd->len = len;
    for (int j = 0; j < 8; j++) nd->suns[j] = -1;
    return (int)(t->nnodes++);
}

static uint64_t hash64(uint64_t x)
{
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33; x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33;
    return x;
}

/* Morton digit of particle p at bit shift `shift` (x=bit0, y=bit1, z=bit2,
 * peano.c:323-335), or the geometric octant below 42 levels (forcetree.c:210-217). */
static int subnode_of(otree_t *t, const uint64_t *q, int64_t p, int node, int shift, int depth)
{
    int sub;
    if (shift >= 0) {
        sub = (int)(((q[3 * p] >> shift) & 1) | (((q[3 * p + 1] >> shift) & 1) << 1) | (((q[3 * p + 2] >> shift) & 1) << 2));
    } else {
        sub = 0;
        if (t->pos[3 * p] > t->nodes[node].center[0]) sub += 1;
        if (t->pos[3 * p + 1] > t->nodes[node].center[1]) sub += 2;
        if (t->pos[3 * p + 2] > t->nodes[node].center[2]) sub += 4;
    }
    if (t->nodes[node].len < 1.0e-4 * t->h[p]) sub = (int)(hash64((uint64_t)p * 131 + depth) & 7);
    return sub;
}

static void tree_build(otree_t *t, const double *center, const double *corner, double len)
{
    const int BITS = 42;
    int64_t n = t->n;
    uint64_t *q = (uint64_t *)malloc(sizeof(uint64_t) * 3 * (n ? n : 1));
    for (int64_t i = 0; i < n; i++)
        for (int j = 0; j < 3; j++) q[3 * i + j] = oracle_double_to_int(((t->pos[3 * i + j] - corner[j]) / len) + 1.0, BITS);
    new_node(t, center, len);
    for (int64_t i = 0; i < n; i++) {
        int th = 0, shift = BITS - 1, depth = 0;
        for (;;) {
            int sub = subnode_of(t, q, i, th, shift, depth);
            int nn = t->nodes[th].suns[sub];
            if (nn < 0) { t->nodes[th].suns[sub] = (int)i; break; }
            if (nn >= n) { th = (int)(nn - n); shift--; depth++; continue; }
            /* slot holds a particle: split (forcetree.c:250-303) */
            double c[3], lh = 0.25 * t->nodes[th].len;
            for (int j = 0; j < 3; j++) c[j] = t->nodes[th].center[j] + (((sub >> j) & 1) ? lh : -lh);
            int nw = new_node(t, c, 0.5 * t->nodes[th].len);
            t->nodes[th].suns[sub] = (int)(n + nw);
            int osub = subnode_of(t, q, nn, nw, shift - 1, depth + 1);
            t->nodes[nw].suns[osub] = nn;
            th = nw; shift--; depth++;
        }
    }
    free(q);
}

/* moments: Sigma m, centre of mass, maxsoft, multiple flag (forcetree.c:434-942),
 * children summed in sub-node order 0..7 like the reference's recursion */
static void tree_moments(otree_t *t, int node)
{
    onode_t *nd = &t->nodes[node];
    double mass = 0, s[3] = {0, 0, 0}, maxsoft = 0, vs[3] = {0, 0, 0}, vmax = 0;
    int count = 0;
    for (int j = 0; j < 8; j++) {
        int p = t->nodes[node].suns[j];
        if (p < 0) continue;
        if (p >= t->n) {
            int c = (int)(p - t->n);
            tree_moments(t, c);
            nd = &t->nodes[node];
            onode_t *cn = &t->nodes[c];
            mass += cn->mass;
            for (int k = 0; k < 3; k++) s[k] += cn->mass * cn->s[k];
            for (int k = 0; k < 3; k++) vs[k] += cn->mass * cn->vs[k];
            if (cn->vmax > vmax) vmax = cn->vmax;
            if (cn->mass > 0) count += cn->multiple ? 2 : 1;
            if (cn->maxsoft > maxsoft) maxsoft = cn->maxsoft;
        } else {
            count++;
            mass += t->mass[p];
            for (int k = 0; k < 3; k++) s[k] += t->mass[p] * t->pos[3 * p + k];
            if (t->h[p] > maxsoft) maxsoft = t->h[p];
            if (t->vel)
                for (int k = 0; k < 3; k++) {
                    vs[k] += t->mass[p] * t->vel[3 * p + k];
                    if (fabs(t->vel[3 * p + k]) > vmax) vmax = fabs(t->vel[3 * p + k]);
                }
        }
    }
    if (mass) for (int k = 0; k < 3; k++) { s[k] /= mass; vs[k] /= mass; }
    else for (int k = 0; k < 3; k++) { s[k] = nd->center[k]; vs[k] = 0; }
    nd->mass = mass;
    for (int k = 0; k < 3; k++) nd->vs[k] = vs[k];
    nd->vmax = vmax;
    for (int k = 0; k < 3; k++) nd->s[k] = s[k];
    nd->maxsoft = maxsoft;
    nd->multiple = count > 1;
}

/* one target's walk (forcetree.c:1823-2657); returns the interaction count.
 * pot_mode: the potential-only walk (force_treeevaluate_potential,
 * forcetree.c:3169-3474), which has the same opening rules but no r2 > 0 or
 * m > 0 condition on a pair: r = 0 pairs (the target itself, coincident
 * particles) add m kernel(0) like any other. */
static int64_t tree_walk(const otree_t *t, const double *pos, double soft, double aold, double theta, double *acc,
                         double *pot_out, int pot_mode)
{
    int64_t n = t->n, nint = 0;
    double ax = 0, ay = 0, az = 0, pot = 0;
    int stack_cap = 4096, sp = 0;
    int *stack = (int *)malloc(sizeof(int) * stack_cap);
    stack[sp++] = (int)n; /* root */
    while (sp > 0) {
        int no = stack[--sp];
        double dx, dy, dz, r2, mass, h = soft, h_p = -1;
        if (no < n) {
            dx = t->pos[3 * no] - pos[0];
            dy = t->pos[3 * no + 1] - pos[1];
            dz = t->pos[3 * no + 2] - pos[2];
            r2 = dx * dx + dy * dy + dz * dz;
            mass = t->mass[no];
            if ((r2 > 0 && mass > 0) || pot_mode) h_p = t->h[no];
        } else {
            const onode_t *nd = &t->nodes[no - n];
            int open = 0;
            mass = nd->mass;
            if (mass <= 0) continue;
            if (!nd->multiple) open = 1;
            if (!open) {
                dx = nd->s[0] - pos[0];
                dy = nd->s[1] - pos[1];
                dz = nd->s[2] - pos[2];
                r2 = dx * dx + dy * dy + dz * dz;
                if (h < nd->maxsoft && r2 < nd->maxsoft * nd->maxsoft) open = 1;
                else if (theta) {
                    if (nd->len * nd->len > r2 * theta * theta) open = 1;
                } else {
                    double a1 = soft + 0.6 * nd->len, a2 = nd->maxsoft + 0.6 * nd->len;
                    if (r2 < a1 * a1 || r2 < a2 * a2) open = 1;
                    else if (mass * nd->len * nd->len > r2 * r2 * aold) open = 1;
                    else if (fabs(nd->center[0] - pos[0]) < 0.60 * nd->len &&
                             fabs(nd->center[1] - pos[1]) < 0.60 * nd->len &&
                             fabs(nd->center[2] - pos[2]) < 0.60 * nd->len)
                        open = 1;
                }
            }
            if (open) {
                if (sp + 8 > stack_cap) { stack_cap *= 2; stack = (int *)realloc(stack, sizeof(int) * stack_cap); }
                for (int j = 7; j >= 0; j--)
                    if (nd->suns[j] >= 0) stack[sp++] = nd->suns[j];
                continue;
            }
            h_p = nd->maxsoft;
        }
        if ((r2 > 0 && mass > 0) || pot_mode) {
            pair_term(dx, dy, dz, r2, mass, h, h_p, &ax, &ay, &az, &pot);
            nint++;
        }
    }
    free(stack);
    acc[0] = ax; acc[1] = ay; acc[2] = az;
    *pot_out = pot;
    return nint;
}

/*
 * Full GIZMO-semantics tree force for the given targets.
 *   pos (n*3), mass (n), h (n, kernel radius = 2.8 * Plummer softening)
 *   old_acc (n): |a|/G from the previous pass (used only when err_tol_theta == 0)
 *   err_tol_theta > 0: Barnes-Hut pass; == 0: relative criterion
 * Outputs per target, pre-G like P[].GravAccel: acc (3), pot, ninter.
 * Returns the total interaction count (the reference's Costtotal).
 */
int64_t oracle_tree_gravity(int64_t n, const double *pos, const double *mass, const double *h, const double *old_acc,
                            double err_tol_force_acc, double err_tol_theta, int64_t n_targets, const int32_t *targets,
                            double *acc, double *pot, int64_t *ninter, int nthreads)
{
    double center[3], corner[3], len;
    oracle_find_extent(n, pos, center, corner, &len);
    otree_t t = {n, pos, mass, h, NULL, NULL, 0, 0};
    tree_build(&t, center, corner, len);
    tree_moments(&t, 0);
    int64_t total = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
#endif
    for (int64_t k = 0; k < n_targets; k++) {
        int64_t i = targets ? targets[k] : k;
        double aold = err_tol_force_acc * (old_acc ? old_acc[i] : 0.0);
        int64_t c = tree_walk(&t, &pos[3 * i], h[i], aold, err_tol_theta, &acc[3 * k], &pot[k], 0);
        if (ninter) ninter[k] = c;
        total += c;
    }
    free(t.nodes);
    return total;
}

/*
 * The same force after a drift of the resident tree without a rebuild: the
 * tree is built and its moments taken at the positions `pos`, then every
 * particle moves by vel*dt (drift_particle, predict.c:97-137) and every node
 * by force_drift_node (forcetree_update.c:265-338): centre of mass
 * s += vs*dt, side len += 2*vmax*dt, geometric centre unchanged, where vs is
 * the mass-weighted mean velocity and vmax the largest |velocity component|
 * of the node's particles (force_update_node_recursive, forcetree.c:558-560,
 * :629, :751, :764-781).  Targets are evaluated at their drifted positions.
 * pos_out (n*3, nullable) receives the drifted positions.
 */
int64_t oracle_tree_gravity_drift(int64_t n, const double *pos, const double *vel, const double *mass, const double *h,
                                  const double *old_acc, double err_tol_force_acc, double err_tol_theta, double dt,
                                  int64_t n_targets, const int32_t *targets, double *acc, double *pot, int64_t *ninter,
                                  double *pos_out, int nthreads)
{
    double center[3], corner[3], len;
    oracle_find_extent(n, pos, center, corner, &len);
    otree_t t = {n, pos, mass, h, vel, NULL, 0, 0};
    tree_build(&t, center, corner, len);
    tree_moments(&t, 0);
    for (int64_t k = 0; k < t.nnodes; k++) {
        onode_t *nd = &t.nodes[k];
        for (int j = 0; j < 3; j++) nd->s[j] += nd->vs[j] * dt;
        nd->len += 2 * nd->vmax * dt;
    }
    double *moved = (double *)malloc(sizeof(double) * 3 * (n ? n : 1));
    for (int64_t i = 0; i < 3 * n; i++) moved[i] = pos[i] + vel[i] * dt;
    t.pos = moved;
    int64_t total = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
#endif
    for (int64_t k = 0; k < n_targets; k++) {
        int64_t i = targets ? targets[k] : k;
        double aold = err_tol_force_acc * (old_acc ? old_acc[i] : 0.0);
        int64_t c = tree_walk(&t, &moved[3 * i], h[i], aold, err_tol_theta, &acc[3 * k], &pot[k], 0);
        if (ninter) ninter[k] = c;
        total += c;
    }
    if (pos_out) memcpy(pos_out, moved, sizeof(double) * 3 * n);
    free(moved);
    free(t.nodes);
    return total;
}

/*
 * compute_potential (gravity/potential.c:24-160) for an isolated tree-only
 * run: the potential-only walk of every target, then its self term removed,
 * m_i / h_i * kernel_gravity(0,1,1,-1) = -2.8 m_i / h_i (potential.c:137-145).
 * Pre-G like P[].Potential before the multiplication by G.
 */
void oracle_potential(int64_t n, const double *pos, const double *mass, const double *h, const double *old_acc,
                      double err_tol_force_acc, double err_tol_theta, int64_t n_targets, const int32_t *targets,
                      double *pot, int nthreads)
{
    double center[3], corner[3], len;
    oracle_find_extent(n, pos, center, corner, &len);
    otree_t t = {n, pos, mass, h, NULL, NULL, 0, 0};
    tree_build(&t, center, corner, len);
    tree_moments(&t, 0);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t k = 0; k < n_targets; k++) {
        int64_t i = targets ? targets[k] : k;
        double aold = err_tol_force_acc * (old_acc ? old_acc[i] : 0.0);
        double acc[3];
        tree_walk(&t, &pos[3 * i], h[i], aold, err_tol_theta, acc, &pot[k], 1);
        pot[k] -= mass[i] / h[i] * spline_gravity(0.0, 1.0, 1.0, -1);
    }
    free(t.nodes);
}

/* node count of the GIZMO octree (diagnostics) */
int64_t oracle_tree_nodes(int64_t n, const double *pos, const double *mass, const double *h)
{
    double center[3], corner[3], len;
    oracle_find_extent(n, pos, center, corner, &len);
    otree_t t = {n, pos, mass, h, NULL, NULL, 0, 0};
    tree_build(&t, center, corner, len);
    int64_t m = t.nnodes;
    free(t.nodes);
    return m;
}

/* FP64 direct summation over all sources with the tree's pair rule; self excluded */
void oracle_direct_sum(int64_t n, const double *pos, const double *mass, const double *h, int64_t n_targets,
                       const int32_t *targets, double *acc, double *pot, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int64_t k = 0; k < n_targets; k++) {
        int64_t i = targets ? targets[k] : k;
        double ax = 0, ay = 0, az = 0, p = 0;
        const double *xi = &pos[3 * i];
        for (int64_t j = 0; j < n; j++) {
            double dx = pos[3 * j] - xi[0], dy = pos[3 * j + 1] - xi[1], dz = pos[3 * j + 2] - xi[2];
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > 0 && mass[j] > 0) pair_term(dx, dy, dz, r2, mass[j], h[i], h[j], &ax, &ay, &az, &p);
        }
        acc[3 * k] = ax; acc[3 * k + 1] = ay; acc[3 * k + 2] = az;
        pot[k] = p;
    }
}
