/*
 * bd_oracle.c -- CPU oracle (TEST INFRASTRUCTURE, never linked into the
 * product).  A plain-C restatement of the reference's Brownian-dynamics
 * semantics; every function cites the reference code it follows.
 *
 * Compiled with -ffp-contract=off (no fused multiply-add) so that the
 * predicate arithmetic is bit-identical to the engine's non-contracted
 * __fadd_rn/__fmul_rn (__dadd_rn/__dmul_rn) sequences.
 */
#include "bd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MT RDGPU_MAX_TYPES

/* ------------------------------------------------------------------------ */
/* Pair potentials (Java semantics).                                        */
/* ------------------------------------------------------------------------ */

/* Scalar part of a pair potential: the force on particle 1 is
   pre * (x2 - x1) (Java "gradient", P2_Harmonic.java:157-196), energy e.
   r is the pair distance, r0 the resolved equilibrium distance.            */
static int pair_scalar(const rdgpu_pair_pot* p, double r0, double r,
                       double* pre, double* e)
{
    *pre = 0.0;
    *e = 0.0;
    if (p->kind == RDGPU_P2_HARMONIC) {
        /* P2_Harmonic.java:117-120: a distance of exactly 0 is set to 1e-6 */
        double rr = (r == 0.0) ? 1e-6 : r;
        const double k = p->k;
        int active;
        switch (p->subtype) {
        case RDGPU_SUB_SPRING:     active = 1; break;            /* :157-166 */
        case RDGPU_SUB_REPULSIVE:  active = (rr < r0); break;    /* :167-178 */
        case RDGPU_SUB_ATTRACTIVE: active = (rr > r0); break;    /* :179-190 */
        default: return -1;
        }
        if (active) {
            *pre = k * (-r0 + rr) / rr;
            *e = 0.5 * k * (-r0 + rr) * (-r0 + rr);              /* :208-228 */
        }
        return 0;
    }
    if (p->kind == RDGPU_P2_WEAK_PIECEWISE) {
        /* P2_WeakInteractionPiecewiseHarmonic.java:114-206 */
        const double k = p->k, d = p->depth, l = p->length;
        const double q = (1.0 / (0.5 * l)) * (1.0 / (0.5 * l));
        if (r < r0) {
            *pre = (r > 0.0) ? k * (r - r0) / r : 0.0;
            *e = k / 2 * (r - r0) * (r - r0) - d;
        } else if (r < r0 + 0.5 * l) {
            *pre = d * q * (r - r0) / r;
            *e = 0.5 * d * q * (r - r0) * (r - r0) - d;
        } else if (r < r0 + l) {
            *pre = -d * q * (r - r0 - l) / r;
            *e = -0.5 * d * q * (r - r0 - l) * (r - r0 - l);
        }
        return 0;
    }
    return -1;
}

int orc_pair_gradient(const rdgpu_pair_pot* p, double r0_pair,
                      const double x1[3], const double x2[3], double dist,
                      double grad[3], double* energy)
{
    double r0 = (p->r0 >= 0.0) ? p->r0 : r0_pair;   /* P2_Harmonic.java:124-128 */
    double pre, e;
    int rc = pair_scalar(p, r0, dist, &pre, &e);
    for (int k = 0; k < 3; ++k) grad[k] = pre * (x2[k] - x1[k]);
    if (energy) *energy = e;
    return rc;
}

double orc_pair_cutoff(const rdgpu_pair_pot* p, double r0_pair, double max_cutoff)
{
    double r0 = (p->r0 >= 0.0) ? p->r0 : r0_pair;
    if (p->kind == RDGPU_P2_HARMONIC) {
        if (p->subtype == RDGPU_SUB_REPULSIVE) return r0;
        return max_cutoff;          /* attractive/spring: reference maxCutoff */
    }
    if (p->kind == RDGPU_P2_WEAK_PIECEWISE) return r0 + p->length;
    return 0.0;
}

/* ------------------------------------------------------------------------ */
/* External potentials (Java semantics).                                    */
/* ------------------------------------------------------------------------ */

static double dot3(const double* a, const double* b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
static double norm3(const double* a) { return sqrt(dot3(a, a)); }

int orc_ext_gradient(const rdgpu_ext_pot* p, double p_radius, const double x[3],
                     double g[3], double* energy)
{
    const double k = p->k;
    double e = 0.0;
    g[0] = g[1] = g[2] = 0.0;
    if (p->kind == RDGPU_P1_DISK || p->kind == RDGPU_P1_CYLINDER) {
        /* normal normalised as in P1_Disk.java:170 (DoubleArrays.normalize) */
        double nn = norm3(p->normal);
        double n[3] = { p->normal[0] / nn, p->normal[1] / nn, p->normal[2] / nn };
        double nnorm = norm3(n);
        double s;
        if (p->kind == RDGPU_P1_DISK) {
            /* P1_Disk.java:118-125: dot(x,n)/|n| - dot(c,n)/|n| */
            s = dot3(x, n) / nnorm - dot3(p->center, n) / nnorm;
        } else {
            /* P1_Cylinder.java:115-120: dot(x-c, n)/|n| */
            double xc[3] = { x[0] - p->center[0], x[1] - p->center[1], x[2] - p->center[2] };
            s = dot3(xc, n) / nnorm;
        }
        double pp[3] = { x[0] - n[0] * s, x[1] - n[1] * s, x[2] - n[2] * s };
        double dplane = fabs(s);
        double cp[3] = { pp[0] - p->center[0], pp[1] - p->center[1], pp[2] - p->center[2] };
        double dinplane = norm3(cp);
        double r, r0, pre;
        if (p->kind == RDGPU_P1_DISK) {
            if (p->subtype == RDGPU_SUB_ATTRACTIVE) {           /* P1_Disk.java:213-240 */
                r = dplane; r0 = 0.0;
                if (r > r0) {
                    pre = k * (-r0 + r) / r;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                    e += 0.5 * k * (-r0 + r) * (-r0 + r);
                }
                r = dinplane + p_radius; r0 = p->radius;
                if (r > r0) {
                    pre = k * (-r0 + r) / r;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p->center[a] - pp[a]);
                    e += 0.5 * k * (-r0 + r) * (-r0 + r);
                }
            } else if (p->subtype == RDGPU_SUB_REPULSIVE) {     /* P1_Disk.java:241-258 */
                r = dplane; r0 = p_radius;
                double r1 = dinplane - p_radius, r01 = p->radius;
                if (r < r0 && r1 < r01) {
                    /* r == 0 (on the plane): direction undefined, no force */
                    pre = (r > 0.0) ? k * (-r0 + r) / r : 0.0;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                    e += 0.5 * k * (-r0 + r) * (-r0 + r);
                }
            } else {
                return -1;
            }
        } else {
            if (p->subtype == RDGPU_SUB_ATTRACTIVE) {           /* P1_Cylinder.java:212-240 */
                r = dplane + p_radius; r0 = 0.5 * p->height;
                if (r > r0) {
                    pre = k * (-r0 + r) / r;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                }
                r = dinplane + p_radius; r0 = p->radius;
                if (r > r0) {
                    pre = k * (-r0 + r) / r;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p->center[a] - pp[a]);
                }
                /* energy as P1_Cylinder.java:296-312 computes it (plane term
                   against the full height, without the particle radius)    */
                r = dplane; r0 = p->height;
                if (r > r0) e += 0.5 * k * (-r0 + r) * (-r0 + r);
                r = dinplane + p_radius; r0 = p->radius;
                if (r > r0) e += 0.5 * k * (-r0 + r) * (-r0 + r);
            } else if (p->subtype == RDGPU_SUB_REPULSIVE) {     /* P1_Cylinder.java:241-270 */
                r = dplane; r0 = p_radius + 0.5 * p->height;
                double r1 = dinplane - p_radius, r01 = p->radius;
                if (r1 < r01) {
                    pre = (r1 != 0.0) ? k * (-r01 + r1) / r1 : 0.0;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (p->center[a] - pp[a]);
                }
                if (r < r0) {
                    pre = (r > 0.0) ? k * (-r0 + r) / r : 0.0;
                    for (int a = 0; a < 3; ++a) g[a] += pre * (pp[a] - x[a]);
                }
                /* energy, P1_Cylinder.java:313-327 */
                r0 = p_radius + p->height;
                if (r < r0) e += 0.5 * k * (-r0 + r) * (-r0 + r);
                if (r1 < r01) e += 0.5 * k * (-r01 + r1) * (-r01 + r1);
            } else {
                return -1;
            }
        }
    } else if (p->kind == RDGPU_P1_SPHERE) {
        /* P1_Sphere.java:202-290 */
        double pr = p->consider_radius ? p_radius : 0.0;
        double xc[3] = { x[0] - p->center[0], x[1] - p->center[1], x[2] - p->center[2] };
        double d = norm3(xc);
        double r, r0, pre;
        int active;
        switch (p->subtype) {
        case RDGPU_SUB_ATTRACTIVE: r = d + pr; r0 = p->radius;      active = (r > r0);  break;
        case RDGPU_SUB_REPULSIVE:  r = d;      r0 = p->radius + pr; active = (r < r0);  break;
        case RDGPU_SUB_MEMBRANE:   r = d;      r0 = p->radius;      active = (r != r0); break;
        default: return -1;
        }
        if (active) {
            pre = (r != 0.0) ? k * (-r0 + r) / r : 0.0;
            for (int a = 0; a < 3; ++a) g[a] += pre * (p->center[a] - x[a]);
            e += 0.5 * k * (-r0 + r) * (-r0 + r);
        }
    } else if (p->kind == RDGPU_P1_CUBE) {
        /* P1_Cube.java:150-159 (min/max), 187-238 (gradient), 240-273 (energy) */
        double pr = p->consider_radius ? p_radius : 0.0;
        for (int a = 0; a < 3; ++a) {
            double lo = p->origin[a], hi = p->origin[a] + p->extension[a];
            if (!(lo < hi)) { double t = lo; lo = hi; hi = t; }
            double gi = 0.0;
            if (x[a] - pr >= lo && x[a] + pr <= hi) {
                gi = 0.0;
            } else if (x[a] - pr < lo) {
                double r = x[a] - pr;
                gi = k * (r - lo);
                e += 0.5 * k * (r - lo) * (r - lo);
            } else {
                double r = x[a] + pr;
                gi = k * (r - hi);
                e += 0.5 * k * (r - hi) * (r - hi);
            }
            if (p->subtype == RDGPU_SUB_ATTRACTIVE) gi = -gi;
            else if (p->subtype != RDGPU_SUB_REPULSIVE) return -1;
            g[a] = gi;
        }
    } else {
        return -1;
    }
    if (energy) *energy = e;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Derived per-system tables.                                               */
/* ------------------------------------------------------------------------ */

typedef struct {
    int S;
    double L[3], half[3];
    int per[3];
    double r0[MT * MT];        /* collision radius sum of the pair            */
    double rc[MT * MT];        /* neighbour cutoff of the pair (0: none)      */
    double rc2[MT * MT];
    float  rc2f[MT * MT];
    float  Lf[3], halff[3];
    double a[MT], b[MT];       /* D dt/(kB T), sqrt(2 D dt)                    */
    double ext_center[RDGPU_MAX_EXT_POTS][3]; /* box-relative centres          */
} tables_t;

/* f32box: use the FP32 box length (float)(hi-lo), widened, as the period --
   the FP32 engine's box                                                     */
static void make_tables_box(const rdgpu_system_desc* d, tables_t* t, int f32box)
{
    memset(t, 0, sizeof(*t));
    t->S = d->n_types;
    for (int a = 0; a < 3; ++a) {
        t->L[a] = d->hi[a] - d->lo[a];
        if (f32box) t->L[a] = (double)(float)t->L[a];
        t->half[a] = 0.5 * t->L[a];
        t->per[a] = d->periodic[a];
        t->Lf[a] = (float)t->L[a];
        t->halff[a] = 0.5f * t->Lf[a];
    }
    for (int i = 0; i < t->S; ++i) {
        for (int j = 0; j < t->S; ++j) {
            /* ParticleParametersFactory.java:167-170 */
            double r0 = d->coll_radius[i * MT + j] + d->coll_radius[j * MT + i];
            t->r0[i * MT + j] = r0;
            double rc = 0.0;
            for (int p = 0; p < d->n_pair; ++p) {
                if (!d->pair[p].pairs[i * MT + j] && !d->pair[p].pairs[j * MT + i]) continue;
                double c = orc_pair_cutoff(&d->pair[p], r0, d->max_cutoff);
                if (c > rc) rc = c;
            }
            t->rc[i * MT + j] = rc;
            t->rc2[i * MT + j] = rc * rc;
            t->rc2f[i * MT + j] = (float)(rc * rc);
        }
        /* ParticleParametersFactory.java:152-155 */
        t->a[i] = d->D[i] * d->dt / (d->kB * d->T);
        t->b[i] = sqrt(2.0 * d->D[i] * d->dt);
    }
}

static void make_tables(const rdgpu_system_desc* d, tables_t* t) { make_tables_box(d, t, 0); }

/* ------------------------------------------------------------------------ */
/* Coordinates.                                                             */
/* ------------------------------------------------------------------------ */

static double wrap_rel(double x, double L, int per)
{
    if (!per) return x;
    /* CudaSimulation.cu:1857-1858 wraps with while loops */
    while (x >= L) x -= L;
    while (x < 0.0) x += L;
    if (x >= L) x = 0.0;
    return x;
}

void orc_to_rel_f64(const rdgpu_system_desc* d, int64_t n, const double* xabs, double* xrel)
{
    for (int64_t i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a)
            xrel[3 * i + a] = wrap_rel(xabs[3 * i + a] - d->lo[a], d->hi[a] - d->lo[a], d->periodic[a]);
}

void orc_to_rel_f32(const rdgpu_system_desc* d, int64_t n, const double* xabs, float* hi, float* comp)
{
    for (int64_t i = 0; i < n; ++i) {
        for (int a = 0; a < 3; ++a) {
            double L = d->hi[a] - d->lo[a];
            float Lf = (float)L;
            double xr = wrap_rel(xabs[3 * i + a] - d->lo[a], (double)Lf, d->periodic[a]);
            float h = (float)xr;
            if (d->periodic[a] && h >= Lf) { h = 0.0f; xr -= (double)Lf; }
            hi[3 * i + a] = h;
            comp[3 * i + a] = (float)((double)h - xr);
        }
    }
}

/* Minimum-image displacement of one component (CudaSimulation.cu:996-1002):
   the image k in {-1, 0, +1} is chosen by comparing xi - xj with half a box,
   and the displacement is then formed as xi - (xj + k L).  Both the oracle
   and the engine round exactly this sequence; the engine's shared-memory
   stage applies the same image shift to the staged xj.                      */
static inline double mimg(double xi, double xj, double L, double half, int per)
{
    double d = xi - xj;
    if (per) {
        if (d > half) d = xi - (xj + L);
        else if (d < -half) d = xi - (xj - L);
    }
    return d;
}
static inline float mimgf(float xi, float xj, float L, float half, int per)
{
    float d = xi - xj;
    if (per) {
        if (d > half) d = xi - (xj + L);
        else if (d < -half) d = xi - (xj - L);
    }
    return d;
}

/* ------------------------------------------------------------------------ */
/* Cell list (acceleration only; the predicate defines the neighbour set).  */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n[3];
    double inv[3];
    int64_t ncells;
    int64_t* start;   /* ncells+1 */
    int64_t* list;    /* particle indices sorted by cell */
    int brute;        /* 1: fewer than 3 cells on a periodic axis */
} cells_t;

static int64_t cell_of(const cells_t* c, const double* x)
{
    int64_t id = 0, mul = 1;
    for (int a = 0; a < 3; ++a) {
        int k = (int)floor(x[a] * c->inv[a]);
        if (k < 0) k = 0;
        if (k >= c->n[a]) k = c->n[a] - 1;
        id += mul * k;
        mul *= c->n[a];
    }
    return id;
}

static void build_cells(const tables_t* t, double cut, int64_t n, const double* x, cells_t* c)
{
    memset(c, 0, sizeof(*c));
    c->ncells = 1;
    for (int a = 0; a < 3; ++a) {
        int k = (cut > 0.0) ? (int)floor(t->L[a] / cut) : 1;
        if (k < 1) k = 1;
        if (k > 1024) k = 1024;
        if (t->per[a] && k < 3) c->brute = 1;
        c->n[a] = k;
        c->inv[a] = (double)k / t->L[a];
        c->ncells *= k;
    }
    if (c->brute) return;
    c->start = (int64_t*)calloc((size_t)c->ncells + 1, sizeof(int64_t));
    c->list = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    int64_t* cid = (int64_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) { cid[i] = cell_of(c, x + 3 * i); c->start[cid[i] + 1]++; }
    for (int64_t k = 0; k < c->ncells; ++k) c->start[k + 1] += c->start[k];
    int64_t* fill = (int64_t*)malloc((size_t)c->ncells * sizeof(int64_t));
    memcpy(fill, c->start, (size_t)c->ncells * sizeof(int64_t));
    for (int64_t i = 0; i < n; ++i) c->list[fill[cid[i]]++] = i;
    free(fill);
    free(cid);
}

static void free_cells(cells_t* c) { free(c->start); free(c->list); }

/* Cell ranges of the (deduplicated) 27-cell neighbourhood of particle i.
   Returns the number of ranges; entries q in [st[r], en[r]) of c->list.
   Brute-force mode returns the single range [0, n) of the identity.        */
static int neighbour_ranges(const cells_t* c, const tables_t* t, const double* x,
                            int64_t i, int64_t n, int64_t st[27], int64_t en[27])
{
    if (c->brute) { st[0] = 0; en[0] = n; return 1; }
    int cc[3];
    int64_t id = cell_of(c, x + 3 * i);
    cc[0] = (int)(id % c->n[0]);
    cc[1] = (int)((id / c->n[0]) % c->n[1]);
    cc[2] = (int)(id / ((int64_t)c->n[0] * c->n[1]));
    int m = 0;
    for (int dz = -1; dz <= 1; ++dz) {
        int z = cc[2] + dz;
        if (z < 0 || z >= c->n[2]) { if (!t->per[2]) continue; z = (z + c->n[2]) % c->n[2]; }
        for (int dy = -1; dy <= 1; ++dy) {
            int y = cc[1] + dy;
            if (y < 0 || y >= c->n[1]) { if (!t->per[1]) continue; y = (y + c->n[1]) % c->n[1]; }
            for (int dx = -1; dx <= 1; ++dx) {
                int xx = cc[0] + dx;
                if (xx < 0 || xx >= c->n[0]) { if (!t->per[0]) continue; xx = (xx + c->n[0]) % c->n[0]; }
                int64_t nc = ((int64_t)z * c->n[1] + y) * c->n[0] + xx;
                st[m] = c->start[nc];
                en[m] = c->start[nc + 1];
                ++m;
            }
        }
    }
    return m;
}

#define NB_J(C, Q) ((C)->brute ? (Q) : (C)->list[(Q)])

static double max_rc(const tables_t* t)
{
    double m = 0.0;
    for (int i = 0; i < t->S; ++i)
        for (int j = 0; j < t->S; ++j)
            if (t->rc[i * MT + j] > m) m = t->rc[i * MT + j];
    return m;
}

/* ------------------------------------------------------------------------ */
/* Forces.                                                                  */
/* ------------------------------------------------------------------------ */

static void particle_force(const rdgpu_system_desc* d, const tables_t* t,
                           const cells_t* c, int64_t n, const double* x,
                           const int32_t* types, int64_t i, double F[3], double* E)
{
    const int ti = types[i];
    double f0 = 0.0, f1 = 0.0, f2 = 0.0, e = 0.0;
    int64_t st[27], en[27];
    int nr = neighbour_ranges(c, t, x, i, n, st, en);
    for (int rr = 0; rr < nr; ++rr) for (int64_t q = st[rr]; q < en[rr]; ++q) {
        const int64_t j = NB_J(c, q);
        if (j == i) continue;
        const int tj = types[j];
        double dx = mimg(x[3 * i + 0], x[3 * j + 0], t->L[0], t->half[0], t->per[0]);
        double dy = mimg(x[3 * i + 1], x[3 * j + 1], t->L[1], t->half[1], t->per[1]);
        double dz = mimg(x[3 * i + 2], x[3 * j + 2], t->L[2], t->half[2], t->per[2]);
        double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < t->rc2[ti * MT + tj]) {
            double r = sqrt(r2);
            for (int p = 0; p < d->n_pair; ++p) {
                const rdgpu_pair_pot* pp = &d->pair[p];
                if (!pp->pairs[ti * MT + tj] && !pp->pairs[tj * MT + ti]) continue;
                double r0 = (pp->r0 >= 0.0) ? pp->r0 : t->r0[ti * MT + tj];
                double pre, pe;
                pair_scalar(pp, r0, r, &pre, &pe);
                /* force on i = pre * (x_j - x_i) = -pre * dx */
                f0 -= pre * dx; f1 -= pre * dy; f2 -= pre * dz;
                e += 0.5 * pe;
            }
        }
    }
    /* external potentials act on box-relative coordinates with
       box-relative centres (same geometry, shifted frame)                   */
    double xa[3] = { x[3 * i] + d->lo[0], x[3 * i + 1] + d->lo[1], x[3 * i + 2] + d->lo[2] };
    for (int p = 0; p < d->n_ext; ++p) {
        if (!d->ext[p].types[ti]) continue;
        double g[3], pe;
        orc_ext_gradient(&d->ext[p], d->p_radius[ti], xa, g, &pe);
        f0 += g[0]; f1 += g[1]; f2 += g[2];
        e += pe;
    }
    F[0] = f0; F[1] = f1; F[2] = f2;
    *E = e;
}

int orc_forces_f64(const rdgpu_system_desc* d, int64_t n, const double* xrel,
                   const int32_t* types, double* forces, double* energy, int n_threads)
{
    tables_t t;
    make_tables(d, &t);
    double cut = d->cell_size > 0.0 ? d->cell_size : max_rc(&t);
    cells_t c;
    build_cells(&t, cut, n, xrel, &c);
    double etot = 0.0;
    if (n_threads < 1) n_threads = 1;
#pragma omp parallel for num_threads(n_threads) schedule(static) reduction(+:etot)
    for (int64_t i = 0; i < n; ++i) {
        double e;
        particle_force(d, &t, &c, n, xrel, types, i, forces + 3 * i, &e);
        etot += e;
    }
    free_cells(&c);
    if (energy) *energy = etot;
    return 0;
}

/* Adds the forces and energy of bonded pairs (ReaDDy particle groups): each
   bond applies one pair potential at any distance, minimum image, r0 from
   the potential or the collision-radius sum of the two types
   (group semantics of the Java core; the reference GPU's groups kernel,
   CudaSimulation.cu:1829-1836, passes particle 1's type twice).            */
int orc_bond_forces_f64(const rdgpu_system_desc* d, int64_t n, const double* x, const int32_t* types,
                        int64_t nb, const int32_t* ij, const int32_t* pot, int32_t npots,
                        const rdgpu_pair_pot* pots, double* forces, double* energy)
{
    tables_t t;
    make_tables(d, &t);
    double etot = 0.0;
    for (int64_t b = 0; b < nb; ++b) {
        const int64_t i = ij[2 * b], j = ij[2 * b + 1];
        if (i < 0 || j < 0 || i >= n || j >= n || pot[b] < 0 || pot[b] >= npots) return -1;
        const rdgpu_pair_pot* pp = &pots[pot[b]];
        const int ti = types[i], tj = types[j];
        double dx = mimg(x[3 * i + 0], x[3 * j + 0], t.L[0], t.half[0], t.per[0]);
        double dy = mimg(x[3 * i + 1], x[3 * j + 1], t.L[1], t.half[1], t.per[1]);
        double dz = mimg(x[3 * i + 2], x[3 * j + 2], t.L[2], t.half[2], t.per[2]);
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double r0 = (pp->r0 >= 0.0) ? pp->r0 : t.r0[ti * MT + tj];
        double pre, pe;
        if (pair_scalar(pp, r0, r, &pre, &pe)) return -1;
        /* force on i = pre * (x_j - x_i) = -pre * (x_i - x_j) */
        forces[3 * i + 0] -= pre * dx; forces[3 * i + 1] -= pre * dy; forces[3 * i + 2] -= pre * dz;
        forces[3 * j + 0] += pre * dx; forces[3 * j + 1] += pre * dy; forces[3 * j + 2] += pre * dz;
        etot += pe;
    }
    if (energy) *energy += etot;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Neighbour digests (bit-exact predicates).                                */
/* ------------------------------------------------------------------------ */

uint64_t orc_splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

void orc_neighbor_digest_f64(const rdgpu_system_desc* d, int64_t n, const double* x,
                             const int32_t* types, int32_t* counts, uint64_t* hashes)
{
    tables_t t;
    make_tables(d, &t);
    for (int64_t i = 0; i < n; ++i) {
        int32_t cnt = 0;
        uint64_t h = 0;
        const int ti = types[i];
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const int tj = types[j];
            double dx = mimg(x[3 * i + 0], x[3 * j + 0], t.L[0], t.half[0], t.per[0]);
            double dy = mimg(x[3 * i + 1], x[3 * j + 1], t.L[1], t.half[1], t.per[1]);
            double dz = mimg(x[3 * i + 2], x[3 * j + 2], t.L[2], t.half[2], t.per[2]);
            double r2 = (dx * dx + dy * dy) + dz * dz;
            if (r2 < t.rc2[ti * MT + tj]) { cnt++; h += orc_splitmix64((uint64_t)j); }
        }
        counts[i] = cnt;
        hashes[i] = h;
    }
}

void orc_neighbor_digest_f32(const rdgpu_system_desc* d, int64_t n, const float* x,
                             const int32_t* types, int32_t* counts, uint64_t* hashes)
{
    tables_t t;
    make_tables(d, &t);
    for (int64_t i = 0; i < n; ++i) {
        int32_t cnt = 0;
        uint64_t h = 0;
        const int ti = types[i];
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const int tj = types[j];
            float dx = mimgf(x[3 * i + 0], x[3 * j + 0], t.Lf[0], t.halff[0], t.per[0]);
            float dy = mimgf(x[3 * i + 1], x[3 * j + 1], t.Lf[1], t.halff[1], t.per[1]);
            float dz = mimgf(x[3 * i + 2], x[3 * j + 2], t.Lf[2], t.halff[2], t.per[2]);
            float r2 = (dx * dx + dy * dy) + dz * dz;
            if (r2 < t.rc2f[ti * MT + tj]) { cnt++; h += orc_splitmix64((uint64_t)j); }
        }
        counts[i] = cnt;
        hashes[i] = h;
    }
}

/* The same digests from a cell list, OpenMP over particles: for the
   benchmark configurations at their full sizes.  The cells (edge >= the
   largest cutoff x (1 + 1e-4), so that a pair that rounds under its FP32
   cutoff is still in adjacent cells) only select candidates; the predicate
   and its arithmetic are the brute-force functions' above.                  */
static void digest_cells(const rdgpu_system_desc* d, int64_t n, const double* xd, const float* xf,
                         const int32_t* types, int32_t* counts, uint64_t* hashes, int n_threads)
{
    tables_t t;
    make_tables(d, &t);
    double* xc = (double*)xd;
    if (xf) {
        xc = (double*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(double));
        for (int64_t i = 0; i < 3 * n; ++i) xc[i] = (double)xf[i];
    }
    cells_t c;
    build_cells(&t, max_rc(&t) * (1.0 + 1e-4), n, xc, &c);
    if (n_threads < 1) n_threads = 1;
#pragma omp parallel for num_threads(n_threads) schedule(dynamic, 4096)
    for (int64_t i = 0; i < n; ++i) {
        int32_t cnt = 0;
        uint64_t h = 0;
        const int ti = types[i];
        int64_t st[27], en[27];
        int nr = neighbour_ranges(&c, &t, xc, i, n, st, en);
        for (int rr = 0; rr < nr; ++rr) for (int64_t q = st[rr]; q < en[rr]; ++q) {
            const int64_t j = NB_J(&c, q);
            if (j == i) continue;
            const int tj = types[j];
            int in;
            if (xf) {
                float dx = mimgf(xf[3 * i + 0], xf[3 * j + 0], t.Lf[0], t.halff[0], t.per[0]);
                float dy = mimgf(xf[3 * i + 1], xf[3 * j + 1], t.Lf[1], t.halff[1], t.per[1]);
                float dz = mimgf(xf[3 * i + 2], xf[3 * j + 2], t.Lf[2], t.halff[2], t.per[2]);
                in = ((dx * dx + dy * dy) + dz * dz) < t.rc2f[ti * MT + tj];
            } else {
                double dx = mimg(xd[3 * i + 0], xd[3 * j + 0], t.L[0], t.half[0], t.per[0]);
                double dy = mimg(xd[3 * i + 1], xd[3 * j + 1], t.L[1], t.half[1], t.per[1]);
                double dz = mimg(xd[3 * i + 2], xd[3 * j + 2], t.L[2], t.half[2], t.per[2]);
                in = ((dx * dx + dy * dy) + dz * dz) < t.rc2[ti * MT + tj];
            }
            if (in) { cnt++; h += orc_splitmix64((uint64_t)j); }
        }
        counts[i] = cnt;
        hashes[i] = h;
    }
    free_cells(&c);
    if (xf) free(xc);
}

void orc_neighbor_digest_cells_f64(const rdgpu_system_desc* d, int64_t n, const double* xrel,
                                   const int32_t* types, int32_t* counts, uint64_t* hashes, int n_threads)
{
    digest_cells(d, n, xrel, NULL, types, counts, hashes, n_threads);
}

void orc_neighbor_digest_cells_f32(const rdgpu_system_desc* d, int64_t n, const float* xrel,
                                   const int32_t* types, int32_t* counts, uint64_t* hashes, int n_threads)
{
    digest_cells(d, n, NULL, xrel, types, counts, hashes, n_threads);
}

/* ------------------------------------------------------------------------ */
/* Euler-Maruyama step.                                                     */
/* ------------------------------------------------------------------------ */

/* x += a F + b xi, then wrap; CudaSimulation.cu:1852-1858 with the Java
   factors of ParticleParametersFactory.java:152-155                         */
static int em_update(const tables_t* t, int ti, double* x, const double F[3], const double xi[3])
{
    int rc = 0;
    for (int a = 0; a < 3; ++a) {
        double v = x[a] + (t->a[ti] * F[a] + t->b[ti] * xi[a]);
        if (t->per[a]) {
            if (v >= t->L[a]) v -= t->L[a];
            else if (v < 0.0) v += t->L[a];
            if (v >= t->L[a]) v = 0.0;
            if (v < 0.0 || v >= t->L[a]) rc = RDGPU_ERR_JUMP;
        }
        x[a] = v;
    }
    return rc;
}

int orc_step_f64(const rdgpu_system_desc* d, int64_t n, double* xrel,
                 const int32_t* types, const double* noise, int n_threads)
{
    tables_t t;
    make_tables(d, &t);
    double* F = (double*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(double));
    double e;
    orc_forces_f64(d, n, xrel, types, F, &e, n_threads);
    int rc = 0;
    for (int64_t i = 0; i < n; ++i) {
        int r = em_update(&t, types[i], xrel + 3 * i, F + 3 * i, noise + 3 * i);
        if (r) rc = r;
    }
    free(F);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* RDF counts.                                                              */
/* ------------------------------------------------------------------------ */

void orc_rdf_edges2(int32_t nbins, double rmax, double* edges2)
{
    double w = rmax / (double)nbins;
    for (int k = 0; k <= nbins; ++k) {
        double e = (double)k * w;
        edges2[k] = e * e;
    }
}

/* RDF displacement, symmetric in i and j: (xi - xj) -/+ L when |xi - xj| >
   L/2.  Swapping i and j negates every rounded intermediate, so both
   orientations of a pair land in the same bin (the engine evaluates each pair
   once and counts it for both, as CudaSimulation.cu:1815-1818 does).        */
static inline double mimg_sym(double xi, double xj, double L, double half, int per)
{
    double d = xi - xj;
    if (per) {
        if (d > half) d = d - L;
        else if (d < -half) d = d + L;
    }
    return d;
}

static int rdf_bin(const double* e2, int nbins, double w, double r2)
{
    int k = (int)(sqrt(r2) / w);
    if (k > nbins - 1) k = nbins - 1;
    if (k < 0) k = 0;
    while (k > 0 && e2[k] > r2) --k;
    while (k < nbins - 1 && e2[k + 1] <= r2) ++k;
    return k;
}

static void rdf_core(const rdgpu_system_desc* d, int64_t n, const double* x,
                     const int32_t* types, int32_t nbins, double rmax, uint64_t* counts,
                     int f32box)
{
    tables_t t;
    make_tables_box(d, &t, f32box);
    double* e2 = (double*)malloc((size_t)(nbins + 1) * sizeof(double));
    orc_rdf_edges2(nbins, rmax, e2);
    const double w = rmax / (double)nbins;
    const int S = d->n_types;
    cells_t c;
    build_cells(&t, rmax, n, x, &c);
    const int64_t H = (int64_t)S * S * nbins;
    /* per-thread histograms; integer sums, so the result does not depend on
       the number of threads                                                 */
#pragma omp parallel
    {
        uint64_t* h = (uint64_t*)calloc((size_t)H, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 1024)
        for (int64_t i = 0; i < n; ++i) {
            const int ti = types[i];
            int64_t st[27], en[27];
            int nr = neighbour_ranges(&c, &t, x, i, n, st, en);
            for (int rr = 0; rr < nr; ++rr) for (int64_t q = st[rr]; q < en[rr]; ++q) {
                const int64_t j = NB_J(&c, q);
                if (j == i) continue;
                const int tj = types[j];
                double dx = mimg_sym(x[3 * i + 0], x[3 * j + 0], t.L[0], t.half[0], t.per[0]);
                double dy = mimg_sym(x[3 * i + 1], x[3 * j + 1], t.L[1], t.half[1], t.per[1]);
                double dz = mimg_sym(x[3 * i + 2], x[3 * j + 2], t.L[2], t.half[2], t.per[2]);
                double r2 = (dx * dx + dy * dy) + dz * dz;
                if (r2 < e2[nbins]) {
                    int b = rdf_bin(e2, nbins, w, r2);
                    h[((int64_t)ti * S + tj) * nbins + b] += 1;
                }
            }
        }
#pragma omp critical
        for (int64_t q = 0; q < H; ++q) counts[q] += h[q];
        free(h);
    }
    free_cells(&c);
    free(e2);
}

void orc_rdf_counts_f64(const rdgpu_system_desc* d, int64_t n, const double* xrel,
                        const int32_t* types, int32_t nbins, double rmax, uint64_t* counts)
{
    rdf_core(d, n, xrel, types, nbins, rmax, counts, 0);
}

void orc_rdf_counts_f32(const rdgpu_system_desc* d, int64_t n, const float* xrel,
                        const int32_t* types, int32_t nbins, double rmax, uint64_t* counts)
{
    /* the FP32 engine runs its FP64 predicate on the widened stored floats,
       with the FP32 box length (widened) as the period                      */
    double* xd = (double*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(double));
    for (int64_t i = 0; i < 3 * n; ++i) xd[i] = (double)xrel[i];
    rdf_core(d, n, xd, types, nbins, rmax, counts, 1);
    free(xd);
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 and Gaussian draws.                                        */
/* ------------------------------------------------------------------------ */

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    /* multipliers and Weyl increments of Philox4x32 (Salmon et al. 2011) */
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += W0; k1 += W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* counter = (index lo, index hi, step lo, step hi), key = seed.  Box-Muller
   on the uniforms u = (w + 0.5) 2^-32 of the four words.                    */
void orc_bd_normals(uint64_t seed, int64_t step, int64_t index, double out[3])
{
    uint32_t ctr[4] = { (uint32_t)index, (uint32_t)((uint64_t)index >> 32),
                        (uint32_t)step, (uint32_t)((uint64_t)step >> 32) };
    uint32_t key[2] = { (uint32_t)seed, (uint32_t)(seed >> 32) };
    uint32_t w[4];
    orc_philox4x32_10(ctr, key, w);
    const double s = 2.3283064365386963e-10; /* 2^-32 */
    double u0 = ((double)w[0] + 0.5) * s, u1 = ((double)w[1] + 0.5) * s;
    double u2 = ((double)w[2] + 0.5) * s, u3 = ((double)w[3] + 0.5) * s;
    const double two_pi = 6.283185307179586;
    double ra = sqrt(-2.0 * log(u0)), rb = sqrt(-2.0 * log(u2));
    out[0] = ra * cos(two_pi * u1);
    out[1] = ra * sin(two_pi * u1);
    out[2] = rb * cos(two_pi * u3);
}

/* ------------------------------------------------------------------------ */
/* CPU baseline run.                                                        */
/* ------------------------------------------------------------------------ */

int orc_run_steps_f64(const rdgpu_system_desc* d, int64_t n, double* xrel,
                      const int32_t* types, uint64_t seed, int64_t first_step,
                      int64_t nsteps, int n_threads)
{
    tables_t t;
    make_tables(d, &t);
    if (n_threads < 1) n_threads = 1;
    double* F = (double*)malloc((size_t)(n > 0 ? n : 1) * 3 * sizeof(double));
    double cut = d->cell_size > 0.0 ? d->cell_size : max_rc(&t);
    int rc = 0;
    for (int64_t s = 0; s < nsteps && rc == 0; ++s) {
        cells_t c;
        build_cells(&t, cut, n, xrel, &c);
        int bad = 0;
#pragma omp parallel for num_threads(n_threads) schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            double e;
            particle_force(d, &t, &c, n, xrel, types, i, F + 3 * i, &e);
        }
#pragma omp parallel for num_threads(n_threads) schedule(static) reduction(|:bad)
        for (int64_t i = 0; i < n; ++i) {
            double xi[3];
            orc_bd_normals(seed, first_step + s, i, xi);
            if (em_update(&t, types[i], xrel + 3 * i, F + 3 * i, xi)) bad = 1;
        }
        free_cells(&c);
        if (bad) rc = RDGPU_ERR_JUMP;
    }
    free(F);
    return rc;
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Input generator of the config-3 workload for the benchmark's reference   */
/* arm: random sequential insertion of non-overlapping spheres, the same    */
/* proposals (SplitMix64 uniforms) and acceptance rule as the engine        */
/* package's generator, so both arms step identical coordinates.            */
/* ------------------------------------------------------------------------ */

static double orc_sm_uniform(uint64_t* s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int64_t orc_rsa_spheres(int64_t n, double L, double diam, uint64_t seed, int64_t max_attempts, double* xyz)
{
    int nc = (int)floor(L / diam);
    if (nc < 3) nc = 3 > (int)(L / diam) ? (int)(L / diam) : 3;
    if (nc < 1) nc = 1;
    const double c = L / nc;
    const int cap = 16;
    const size_t ncell = (size_t)nc * nc * nc;
    int32_t* cnt = (int32_t*)calloc(ncell, sizeof(int32_t));
    int64_t* slot = (int64_t*)malloc(ncell * cap * sizeof(int64_t));
    uint64_t rs = seed;
    const double d2 = diam * diam;
    int64_t placed = 0;
    for (int64_t att = 0; att < max_attempts && placed < n; ++att) {
        double p[3];
        for (int a = 0; a < 3; ++a) p[a] = orc_sm_uniform(&rs) * L;
        int ci[3];
        for (int a = 0; a < 3; ++a) {
            int k = (int)(p[a] / c);
            ci[a] = k >= nc ? nc - 1 : k;
        }
        int ok = 1;
        for (int dz = -1; dz <= 1 && ok; ++dz)
            for (int dy = -1; dy <= 1 && ok; ++dy)
                for (int dx = -1; dx <= 1 && ok; ++dx) {
                    int x = (ci[0] + dx + nc) % nc, y = (ci[1] + dy + nc) % nc, z = (ci[2] + dz + nc) % nc;
                    size_t cell = ((size_t)z * nc + y) * nc + x;
                    for (int q = 0; q < cnt[cell]; ++q) {
                        const double* o = xyz + 3 * slot[cell * cap + q];
                        double r2 = 0.0;
                        for (int a = 0; a < 3; ++a) {
                            double dd = p[a] - o[a];
                            if (dd > 0.5 * L) dd -= L;
                            else if (dd < -0.5 * L) dd += L;
                            r2 += dd * dd;
                        }
                        if (r2 < d2) { ok = 0; break; }
                    }
                }
        if (!ok) continue;
        size_t cell = ((size_t)ci[2] * nc + ci[1]) * nc + ci[0];
        if (cnt[cell] >= cap) continue;
        slot[cell * cap + cnt[cell]++] = placed;
        for (int a = 0; a < 3; ++a) xyz[3 * placed + a] = p[a];
        ++placed;
    }
    free(cnt);
    free(slot);
    return placed;
}
