/*
 * C/OpenMP restatement of Genesis's MLS-MPM substep -- TEST INFRASTRUCTURE ONLY.
 *
 * Used as (a) the timed CPU baseline of bench.py (the reference itself runs on
 * gstaichi, which is not installed, so this port stands in for the reference's CPU
 * backend; "kind": "port") and (b) a second checker beside the numpy oracle
 * (oracle/mpm_ref.py).  Never linked into the product.
 *
 * Follows, in the reference:
 *   compute_F_tmp  genesis/engine/solvers/mpm_solver.py:261-267
 *   svd            mpm_solver.py:269-275 (ti.svd; restated as Jacobi eigen-analysis of
 *                  A^T A + Givens QR, the McAdams et al. 2011 structure)
 *   p2g            mpm_solver.py:290-389 (return mappings and stress of materials/MPM/)
 *   grid op        genesis/engine/couplers/legacy_coupler.py:364-375, 495-496
 *   g2p            mpm_solver.py:391-449
 *   boundary       genesis/engine/boundaries/boundaries.py:23-33
 *
 * Parity is unpinned (no reference outputs exist for this path); see mpm_ref.py.
 * Compiled twice: REAL=float (f32) and REAL=double (f64).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif

#if defined(REAL_IS_FLOAT)
#define R_SQRT(x) sqrtf(x)
#define RLOG(x) logf(x)
#define REXP(x) expf(x)
#define RPOW(x, y) powf(x, y)
#define RFLOOR(x) floorf(x)
#define RABS(x) fabsf(x)
#define RMAX(a, b) fmaxf(a, b)
#define RMIN(a, b) fminf(a, b)
#define R_SIN(x) sinf(x)
#define R_FLOOR(x) floorf(x)
#define R_COS(x) cosf(x)
#else
#define R_SQRT(x) sqrt(x)
#define RLOG(x) log(x)
#define REXP(x) exp(x)
#define RPOW(x, y) pow(x, y)
#define RFLOOR(x) floor(x)
#define RABS(x) fabs(x)
#define RMAX(a, b) fmax(a, b)
#define RMIN(a, b) fmin(a, b)
#define R_SIN(x) sin(x)
#define R_FLOOR(x) floor(x)
#define R_COS(x) cos(x)
#endif

typedef struct {
    int32_t res[3];
    int32_t lower_cell[3];
    REAL dx, inv_dx, dt, eps;
    REAL gravity[3];
    REAL bnd_lo[3], bnd_hi[3];
    REAL stress_scale; /* -dt * p_vol * 4 * inv_dx^2 */
    REAL c_scale;      /* 4 * inv_dx */
} ref_params;

typedef struct {
    int32_t kind; /* 0 elastic 1 elastoplastic 2 liquid 3 sand 4 snow */
    int32_t flags; /* 1 neohookean, 2 von mises, 4 muscle */
    REAL mu, lam, mass;
    REAL clamp_lo, clamp_hi, vm_threshold, sand_c1, sand_alpha;
    REAL muscle_stiffness; /* muscle.py:54 (E) */
} ref_material;

/* kinematic rigid collider of the grid op (legacy_coupler.py:131-343); kind 0 sphere
 * (data[0] radius), 1 plane (data = unit normal, geom frame), 2 box (data = half extents) */
typedef struct {
    int32_t kind; /* 0 sphere, 1 plane, 2 box, 3 tool (voxel signed-distance grid) */
    REAL pos[3], rot[9], data[3], lin_vel[3], ang_vel[3];
    REAL friction, softness, restitution;
    const REAL* sdf;    /* tool: [sdf_res]^3 voxels, x-major */
    int32_t sdf_res;
    REAL sdf_scale[3];  /* tool, sampled geom: voxel = sdf_scale * (geom-frame point) + (res - 1) / 2 */
    REAL floor;         /* tool: floor height of the tool solver */
    int32_t sdf_res3[3];/* sampled geom (kind 4): voxels per axis; sdf holds the values, then [n][3] gradients */
    REAL sdf_cell;      /* sampled geom: cell size */
    REAL sdf_max;       /* sampled geom: largest sampled distance */
} ref_collider;

/* ---------------------------------------------------------------- SVD */

static void jacobi(REAL a[3][3], REAL v[3][3], int P, int Q) {
    int R = 3 - P - Q;
    REAL apq = a[P][Q], app = a[P][P], aqq = a[Q][Q];
    REAL t = 0, c = 1, s = 0;
    if (RABS(apq) > (REAL)1e-30) {
        REAL tau = (aqq - app) / (2 * apq);
        REAL at = RABS(tau);
        t = at > (REAL)1e15 ? (REAL)0.5 / tau : (tau >= 0 ? 1 : -1) / (at + R_SQRT(1 + tau * tau));
        c = 1 / R_SQRT(1 + t * t);
        s = t * c;
    }
    a[P][P] = app - t * apq;
    a[Q][Q] = aqq + t * apq;
    a[P][Q] = a[Q][P] = 0;
    REAL arp = a[R][P], arq = a[R][Q];
    a[R][P] = a[P][R] = c * arp - s * arq;
    a[R][Q] = a[Q][R] = s * arp + c * arq;
    for (int i = 0; i < 3; ++i) {
        REAL vip = v[i][P], viq = v[i][Q];
        v[i][P] = c * vip - s * viq;
        v[i][Q] = s * vip + c * viq;
    }
}

static void givens(REAL a, REAL b, REAL* c, REAL* s) {
    REAL r = R_SQRT(a * a + b * b);
    if (r > (REAL)1e-30) {
        *c = a / r;
        *s = b / r;
    } else {
        *c = 1;
        *s = 0;
    }
}

static void swap_neg(REAL b[3][3], REAL v[3][3], REAL* n, int I, int J) {
    for (int r = 0; r < 3; ++r) {
        REAL tb = b[r][I];
        b[r][I] = b[r][J];
        b[r][J] = -tb;
        REAL tv = v[r][I];
        v[r][I] = v[r][J];
        v[r][J] = -tv;
    }
    REAL t = n[I];
    n[I] = n[J];
    n[J] = t;
}

static void rot_rows(REAL b[3][3], REAL u[3][3], int I, int J, REAL c, REAL s) {
    for (int j = 0; j < 3; ++j) {
        REAL t0 = b[I][j], t1 = b[J][j];
        b[I][j] = c * t0 + s * t1;
        b[J][j] = -s * t0 + c * t1;
    }
    for (int i = 0; i < 3; ++i) {
        REAL t0 = u[i][I], t1 = u[i][J];
        u[i][I] = c * t0 + s * t1;
        u[i][J] = -s * t0 + c * t1;
    }
}

void ref_svd3(const REAL* A, REAL* U, REAL* S, REAL* V) {
    REAL a[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, b[3][3], u[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) a[i][j] = A[0 * 3 + i] * A[0 * 3 + j] + A[1 * 3 + i] * A[1 * 3 + j] + A[2 * 3 + i] * A[2 * 3 + j];
    int sweeps = sizeof(REAL) == 4 ? 4 : 8;
    for (int sw = 0; sw < sweeps; ++sw) {
        jacobi(a, v, 0, 1);
        jacobi(a, v, 0, 2);
        jacobi(a, v, 1, 2);
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) b[i][j] = A[i * 3 + 0] * v[0][j] + A[i * 3 + 1] * v[1][j] + A[i * 3 + 2] * v[2][j];
    REAL n[3];
    for (int j = 0; j < 3; ++j) n[j] = b[0][j] * b[0][j] + b[1][j] * b[1][j] + b[2][j] * b[2][j];
    if (n[0] < n[1]) swap_neg(b, v, n, 0, 1);
    if (n[0] < n[2]) swap_neg(b, v, n, 0, 2);
    if (n[1] < n[2]) swap_neg(b, v, n, 1, 2);
    REAL c, s;
    givens(b[0][0], b[1][0], &c, &s);
    rot_rows(b, u, 0, 1, c, s);
    givens(b[0][0], b[2][0], &c, &s);
    rot_rows(b, u, 0, 2, c, s);
    givens(b[1][1], b[2][1], &c, &s);
    rot_rows(b, u, 1, 2, c, s);
    S[0] = b[0][0];
    S[1] = b[1][1];
    S[2] = b[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            U[i * 3 + j] = u[i][j];
            V[i * 3 + j] = v[i][j];
        }
}

/* ---------------------------------------------------------------- materials */

static void usvt(const REAL* U, const REAL* s, const REAL* V, REAL* M) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            M[i * 3 + j] = U[i * 3 + 0] * s[0] * V[j * 3 + 0] + U[i * 3 + 1] * s[1] * V[j * 3 + 1] + U[i * 3 + 2] * s[2] * V[j * 3 + 2];
}

static void corot(REAL mu, REAL lam, REAL J, const REAL* F, const REAL* U, const REAL* V, REAL* out) {
    REAL R[9];
    REAL one[3] = {1, 1, 1};
    usvt(U, one, V, R);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            REAL acc = 0;
            for (int k = 0; k < 3; ++k) acc += (F[i * 3 + k] - R[i * 3 + k]) * F[j * 3 + k];
            out[i * 3 + j] = 2 * mu * acc + (i == j ? lam * J * (J - 1) : 0);
        }
}

static void constitutive(const ref_material* m, REAL eps, REAL J, const REAL* Ft, const REAL* U, const REAL* S,
                         const REAL* V, REAL Jp, REAL* Fn, REAL* Jpn, REAL* st) {
    REAL mu = m->mu, lam = m->lam, Sn[3];
    switch (m->kind) {
        case 0: /* elastic.py:62-83 */
            memcpy(Fn, Ft, 9 * sizeof(REAL));
            *Jpn = Jp;
            if (m->flags & 1) {
                REAL d = lam * RLOG(J) - mu;
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) {
                        REAL acc = Ft[i * 3 + 0] * Ft[j * 3 + 0] + Ft[i * 3 + 1] * Ft[j * 3 + 1] + Ft[i * 3 + 2] * Ft[j * 3 + 2];
                        st[i * 3 + j] = mu * acc + (i == j ? d : 0);
                    }
            } else {
                corot(mu, lam, J, Fn, U, V, st);
            }
            break;
        case 2: { /* liquid.py:50-64 */
            REAL c = RPOW(J, (REAL)(1.0 / 3.0));
            for (int k = 0; k < 9; ++k) Fn[k] = (k % 4 == 0) ? c : 0;
            *Jpn = Jp;
            corot(mu, lam, J, Ft, U, V, st);
            break;
        }
        case 1: /* elasto_plastic.py:66-93 */
            if (m->flags & 2) {
                REAL e[3], eh[3];
                for (int d = 0; d < 3; ++d) e[d] = RLOG(RMAX(S[d], (REAL)0.05));
                REAL mean = (e[0] + e[1] + e[2]) / 3;
                for (int d = 0; d < 3; ++d) eh[d] = e[d] - mean;
                REAL ehn = R_SQRT(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
                REAL dg = ehn - m->vm_threshold;
                if (dg > 0) {
                    for (int d = 0; d < 3; ++d) Sn[d] = REXP(e[d] - (dg / ehn) * eh[d]);
                    usvt(U, Sn, V, Fn);
                } else {
                    memcpy(Fn, Ft, 9 * sizeof(REAL));
                }
            } else {
                for (int d = 0; d < 3; ++d) Sn[d] = RMIN(RMAX(S[d], m->clamp_lo), m->clamp_hi);
                usvt(U, Sn, V, Fn);
            }
            *Jpn = Jp;
            corot(mu, lam, J, Fn, U, V, st);
            break;
        case 4: { /* snow.py:62-81 */
            REAL jp = Jp;
            for (int d = 0; d < 3; ++d) {
                Sn[d] = RMIN(RMAX(S[d], m->clamp_lo), m->clamp_hi);
                jp = jp * (S[d] / Sn[d]);
            }
            *Jpn = jp;
            usvt(U, Sn, V, Fn);
            REAL h = REXP(10 * (1 - Jp));
            corot(mu * h, lam * h, J, Fn, U, V, st);
            break;
        }
        default: { /* sand.py:51-89 */
            REAL e[3], eh[3];
            for (int d = 0; d < 3; ++d) e[d] = RLOG(RMAX(RABS(S[d]), (REAL)1e-4));
            REAL tr = e[0] + e[1] + e[2] + Jp;
            for (int d = 0; d < 3; ++d) eh[d] = e[d] - tr / 3;
            REAL ehn = R_SQRT(eh[0] * eh[0] + eh[1] * eh[1] + eh[2] * eh[2] + eps);
            if (tr >= 0) {
                *Jpn = tr;
                Sn[0] = Sn[1] = Sn[2] = 1;
            } else {
                *Jpn = 0;
                REAL dg = ehn + m->sand_c1 * tr * m->sand_alpha;
                for (int d = 0; d < 3; ++d) Sn[d] = REXP(e[d] - RMAX(0, dg) / ehn * eh[d]);
            }
            usvt(U, Sn, V, Fn);
            REAL l[3], center[3], M[9];
            for (int d = 0; d < 3; ++d) l[d] = RLOG(Sn[d]);
            REAL ls = l[0] + l[1] + l[2];
            for (int d = 0; d < 3; ++d) center[d] = 2 * mu * l[d] * (1 / Sn[d]) + lam * ls * (1 / Sn[d]);
            usvt(U, center, V, M);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                    st[i * 3 + j] = M[i * 3 + 0] * Fn[j * 3 + 0] + M[i * 3 + 1] * Fn[j * 3 + 1] + M[i * 3 + 2] * Fn[j * 3 + 2];
            break;
        }
    }
}

/* Branch margins (test instrumentation, off unless ref_set_branch_margin gave a buffer):
 * for each particle, the smallest distance seen so far to the switch of its return
 * mapping's branch -- Sand |tr| (sand.py:60-62), von Mises |delta_gamma|
 * (elasto_plastic.py:76-78), clamp / Snow min over d of |S_d - (1 - yield_lower)| and
 * |S_d - (1 + yield_higher)| (elasto_plastic.py:89, snow.py:67).  A float32 run can take the
 * other branch where this is within its rounding.  One buffer for the whole library: not
 * for concurrent calls. */
static REAL* g_branch_margin = NULL;

void ref_set_branch_margin(REAL* buf) { g_branch_margin = buf; }

static void record_branch_margin(const ref_material* m, REAL eps, const REAL* S, REAL Jp, REAL* out) {
    REAL d = *out;
    if (m->kind == 3) {
        REAL tr = Jp;
        for (int k = 0; k < 3; ++k) tr += RLOG(RMAX(RABS(S[k]), (REAL)1e-4));
        d = RMIN(d, RABS(tr));
    } else if (m->kind == 1 && (m->flags & 2)) {
        REAL e[3];
        for (int k = 0; k < 3; ++k) e[k] = RLOG(RMAX(S[k], (REAL)0.05));
        REAL mean = (e[0] + e[1] + e[2]) / 3, q = eps;
        for (int k = 0; k < 3; ++k) q += (e[k] - mean) * (e[k] - mean);
        d = RMIN(d, RABS(R_SQRT(q) - m->vm_threshold));
    } else if (m->kind == 1 || m->kind == 4) {
        for (int k = 0; k < 3; ++k) d = RMIN(d, RMIN(RABS(S[k] - m->clamp_lo), RABS(S[k] - m->clamp_hi)));
    }
    *out = d;
}

static REAL bc_vel(REAL pos, REAL vel, REAL lo, REAL hi) {
    if (pos >= hi && vel >= 0) return vel * (REAL)-0.0;
    if (pos <= lo && vel <= 0) return vel * (REAL)-0.0;
    return vel;
}

static inline int64_t gidx(const ref_params* p, int i, int j, int k) {
    return ((int64_t)i * p->res[1] + j) * p->res[2] + k;
}

/*
 * n_substeps full substeps in place.  State arrays (API order): x,v [n*3], C,F [n*9], Jp [n];
 * mat [n] material index, active [n] (0/1).  grid: caller scratch of 4*res^3 (momentum.xyz, mass)
 * and vel 3*res^3.  Returns 0, or 1 if a stencil left the grid, 2 if a position became NaN.
 */
int ref_substeps_lame(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p);
int ref_substeps_ext(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                     REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                     int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir);
int ref_substeps_full(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir,
                      ref_collider* colliders, int n_colliders, REAL* forces);
int ref_substeps_cpic(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir,
                      ref_collider* colliders, int n_colliders, REAL* forces, REAL* rnormal);

int ref_substeps(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F, REAL* Jp,
                 const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel, int n_threads) {
    return ref_substeps_lame(p, mats, n, x, v, C, F, Jp, mat, active, n_substeps, grid, gvel, n_threads, NULL, NULL);
}

/* as ref_substeps, with optional per-particle Lame parameters (NULL: the material's) */
int ref_substeps_lame(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p) {
    return ref_substeps_ext(p, mats, n, x, v, C, F, Jp, mat, active, n_substeps, grid, gvel, n_threads, mu_p, lam_p,
                            NULL, NULL);
}

/* as ref_substeps_lame, with optional per-particle muscle actuation actu[n] and fibre
 * direction mdir[n*3] (NULL: no actuation) */
int ref_substeps_ext(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                     REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                     int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir) {
    return ref_substeps_full(p, mats, n, x, v, C, F, Jp, mat, active, n_substeps, grid, gvel, n_threads, mu_p, lam_p,
                             actu, mdir, NULL, 0, NULL);
}

/* signed distance sd and (unnormalised) world gradient g of the collider at pos, q = pos -
 * collider centre (utils/sdf_decomp.py: the analytic sphere/plane/box SDFs) */
static void sdf_grad(const ref_collider* c, REAL eps, const REAL* pos, REAL* sd_out, REAL* g, REAL* q) {
    REAL sd;
    for (int i = 0; i < 3; ++i) q[i] = pos[i] - c->pos[i];
    if (c->kind == 0) {
        sd = R_SQRT(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) - c->data[0];
        REAL nn = R_SQRT(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + eps);
        for (int i = 0; i < 3; ++i) g[i] = q[i] / nn;
    } else {
        REAL l[3], gl[3];
        for (int i = 0; i < 3; ++i) l[i] = c->rot[0 * 3 + i] * q[0] + c->rot[1 * 3 + i] * q[1] + c->rot[2 * 3 + i] * q[2];
        if (c->kind == 1) {
            sd = l[0] * c->data[0] + l[1] * c->data[1] + l[2] * c->data[2];
            for (int i = 0; i < 3; ++i) gl[i] = c->data[i];
        } else if (c->kind == 4) {
            /* sampled geom: sdf_func_sdf / sdf_func_grad (utils/sdf_decomp.py:102-276) */
            const int32_t* r = c->sdf_res3;
            REAL ps[3], dc[3];
            int outside = 0;
            for (int i = 0; i < 3; ++i) {
                REAL half = (REAL)0.5 * (REAL)(r[i] - 1);
                ps[i] = c->sdf_scale[i] * (l[i] - c->data[i]) + half; /* data: the grid's centre, geom frame */
                dc[i] = ps[i] - half;
                if (ps[i] >= (REAL)(r[i] - 1) || ps[i] <= 0) outside = 1;
            }
            if (outside) {
                REAL d2 = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2];
                sd = R_SQRT(d2) / c->sdf_cell + c->sdf_max;
                REAL nn = R_SQRT(d2 + eps);
                for (int i = 0; i < 3; ++i) gl[i] = dc[i] / nn;
            } else {
                int b[3];
                for (int i = 0; i < 3; ++i) {
                    b[i] = (int)RFLOOR(ps[i]);
                    if (b[i] > r[i] - 2) b[i] = r[i] - 2;
                }
                const int64_t N = (int64_t)r[0] * r[1] * r[2];
                sd = 0;
                gl[0] = gl[1] = gl[2] = 0;
                for (int o = 0; o < 8; ++o) {
                    int cx = b[0] + (o >> 2), cy = b[1] + ((o >> 1) & 1), cz = b[2] + (o & 1);
                    REAL w = (1 - RABS(ps[0] - cx)) * (1 - RABS(ps[1] - cy)) * (1 - RABS(ps[2] - cz));
                    int64_t idx = ((int64_t)cx * r[1] + cy) * r[2] + cz;
                    sd += w * c->sdf[idx];
                    for (int i = 0; i < 3; ++i) gl[i] += w * c->sdf[N + 3 * idx + i];
                }
            }
        } else {
            REAL d[3], o[3];
            for (int i = 0; i < 3; ++i) {
                d[i] = (l[i] < 0 ? -l[i] : l[i]) - c->data[i];
                o[i] = d[i] > 0 ? d[i] : 0;
            }
            REAL out = R_SQRT(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            REAL dm = d[0] > d[1] ? (d[0] > d[2] ? d[0] : d[2]) : (d[1] > d[2] ? d[1] : d[2]);
            sd = out + (dm < 0 ? dm : 0);
            if (out > 0) {
                for (int i = 0; i < 3; ++i) gl[i] = (l[i] < 0 ? -o[i] : o[i]) / out;
            } else {
                int a = (d[0] >= d[1] && d[0] >= d[2]) ? 0 : (d[1] >= d[2] ? 1 : 2);
                for (int i = 0; i < 3; ++i) gl[i] = (i == a) ? (l[i] < 0 ? -1 : 1) : 0;
            }
        }
        for (int i = 0; i < 3; ++i) g[i] = c->rot[i * 3 + 0] * gl[0] + c->rot[i * 3 + 1] * gl[1] + c->rot[i * 3 + 2] * gl[2];
    }
    *sd_out = sd;
}

/* sdf_func_normal_world: the unit outward normal of the collider at pos */
static void sdf_normal(const ref_collider* c, REAL eps, const REAL* pos, REAL* n) {
    REAL sd, g[3], q[3];
    sdf_grad(c, eps, pos, &sd, g, q);
    REAL gn = R_SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + eps);
    for (int i = 0; i < 3; ++i) n[i] = g[i] / gn;
}

/* the collision response of legacy_coupler.py:297-341 (_func_collide_in_rigid_geom) for a
 * point at q from the collider centre with outward normal n and influence infl; adds the
 * reaction force and torque (about the centre) to f[6] */
static void rigid_respond(const ref_collider* c, REAL eps, REAL dt, REAL mass, const REAL* q, const REAL* n, REAL infl,
                          REAL* v, REAL* f) {
    const REAL* w = c->ang_vel;
    REAL vr[3] = {c->lin_vel[0] + w[1] * q[2] - w[2] * q[1], c->lin_vel[1] + w[2] * q[0] - w[0] * q[2],
                  c->lin_vel[2] + w[0] * q[1] - w[1] * q[0]};
    REAL rv[3] = {v[0] - vr[0], v[1] - vr[1], v[2] - vr[2]};
    REAL rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    if (!(rn < 0)) return;
    REAL rt[3] = {rv[0] - rn * n[0], rv[1] - rn * n[1], rv[2] - rn * n[2]};
    REAL rtn = R_SQRT(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] + eps);
    REAL sc = rtn + rn * c->friction;
    sc = (sc > 0 ? sc : 0) / rtn;
    REAL dv[3];
    for (int i = 0; i < 3; ++i) {
        REAL rnew = rt[i] * sc - n[i] * rn * c->restitution;
        REAL nv = vr[i] + rnew * infl + rv[i] * (1 - infl);
        dv[i] = nv - v[i];
        v[i] = nv;
    }
    if (f) {
        REAL fo[3] = {-mass * dv[0] / dt, -mass * dv[1] / dt, -mass * dv[2] / dt};
        REAL to[3] = {q[1] * fo[2] - q[2] * fo[1], q[2] * fo[0] - q[0] * fo[2], q[0] * fo[1] - q[1] * fo[0]};
        for (int i = 0; i < 3; ++i) {
#pragma omp atomic
            f[i] += fo[i];
#pragma omp atomic
            f[3 + i] += to[i];
        }
    }
}

/* legacy_coupler.py:166-343 for one node against one collider (the grid op's coupling):
 * influence min(exp(-sd / softness), 1), acting above 0.1 */
static void collide_rigid(const ref_collider* c, REAL eps, REAL dt, REAL mass, const REAL* pos, REAL* v, REAL* f) {
    REAL sd, g[3], q[3];
    sdf_grad(c, eps, pos, &sd, g, q);
    REAL soft = c->softness > (REAL)1e-10 ? c->softness : (REAL)1e-10;
    REAL infl = RMIN(REXP(-sd / soft), (REAL)1);
    if (!(infl > (REAL)0.1)) return;
    REAL gn = R_SQRT(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + eps);
    REAL n[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
    rigid_respond(c, eps, dt, mass, q, n, infl, v, f);
}

/* ---- tools (engine/entities/tool_entity/mesh.py:80-176) ---- */

/* mesh.py:89-104: trilinear sample at voxel coordinate pv, 1 outside the grid */
static REAL tool_sdf_at(const ref_collider* c, const REAL* pv) {
    int res = c->sdf_res;
    REAL f0 = R_FLOOR(pv[0]), f1 = R_FLOOR(pv[1]), f2 = R_FLOOR(pv[2]);
    if (!(f0 >= 0 && f1 >= 0 && f2 >= 0 && f0 < res - 1 && f1 < res - 1 && f2 < res - 1)) return 1;
    int b[3] = {(int)f0, (int)f1, (int)f2};
    REAL sd = 0;
    for (int o = 0; o < 8; ++o) {
        int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        REAL w = (1 - RABS(pv[0] - (b[0] + i))) * (1 - RABS(pv[1] - (b[1] + j))) * (1 - RABS(pv[2] - (b[2] + k)));
        sd += w * c->sdf[((int64_t)(b[0] + i) * res + (b[1] + j)) * res + (b[2] + k)];
    }
    return sd;
}

/* Tool.collide (mesh.py:147-176) for a grid node at pos: influence min(exp(-sd / softness), 1);
 * the body point's velocity from the pose one substep later (mesh.py:139-145), the normal by
 * central differences of 1e-2 voxel (mesh.py:107-137), friction on the tangential part */
static void collide_tool(const ref_collider* c, REAL eps, REAL dt, const REAL* pos, REAL* v) {
    if (!c->sdf || c->sdf_res < 2) return;
    REAL q[3] = {pos[0] - c->pos[0], pos[1] - c->pos[1], pos[2] - c->pos[2]};
    REAL pv[3], half = (REAL)0.5 * (c->sdf_res - 1);
    for (int i = 0; i < 3; ++i)
        pv[i] = c->sdf_scale[i] * (c->rot[0 * 3 + i] * q[0] + c->rot[1 * 3 + i] * q[1] + c->rot[2 * 3 + i] * q[2]) + half;
    REAL sd = tool_sdf_at(c, pv);
    REAL soft = c->softness > eps ? c->softness : eps;
    REAL infl = RMIN(REXP(-sd / soft), (REAL)1);
    if (!(sd <= 0 || infl > (REAL)0.1)) return;
    /* ((E - I) q + dpos) / dt, E the rotation by ang dt */
    REAL d[3] = {0, 0, 0};
    REAL wx = c->ang_vel[0] * dt, wy = c->ang_vel[1] * dt, wz = c->ang_vel[2] * dt;
    REAL th = R_SQRT(wx * wx + wy * wy + wz * wz);
    if (th > 0) {
        REAL k[3] = {wx / th, wy / th, wz / th};
        REAL kq[3] = {k[1] * q[2] - k[2] * q[1], k[2] * q[0] - k[0] * q[2], k[0] * q[1] - k[1] * q[0]};
        REAL kkq[3] = {k[1] * kq[2] - k[2] * kq[1], k[2] * kq[0] - k[0] * kq[2], k[0] * kq[1] - k[1] * kq[0]};
        REAL sh = R_SIN(th / 2), s = R_SIN(th), t = 2 * sh * sh;
        for (int i = 0; i < 3; ++i) d[i] = s * kq[i] + t * kkq[i];
    }
    REAL dz = c->lin_vel[2] * dt;
    if (c->pos[2] + dz < c->floor) dz = c->floor - c->pos[2];
    REAL vc[3] = {(d[0] + c->lin_vel[0] * dt) / dt, (d[1] + c->lin_vel[1] * dt) / dt, (d[2] + dz) / dt};
    REAL rv[3] = {v[0] - vc[0], v[1] - vc[1], v[2] - vc[2]};
    REAL nv[3];
    for (int i = 0; i < 3; ++i) {
        REAL a[3] = {pv[0], pv[1], pv[2]}, b[3] = {pv[0], pv[1], pv[2]};
        a[i] += (REAL)1e-2;
        b[i] -= (REAL)1e-2;
        nv[i] = (tool_sdf_at(c, a) - tool_sdf_at(c, b)) / (REAL)2e-2;
    }
    REAL nn = R_SQRT(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2] + eps);
    REAL nm[3] = {nv[0] / nn / c->sdf_scale[0], nv[1] / nn / c->sdf_scale[1], nv[2] / nn / c->sdf_scale[2]};
    REAL n[3];
    for (int i = 0; i < 3; ++i) n[i] = c->rot[i * 3 + 0] * nm[0] + c->rot[i * 3 + 1] * nm[1] + c->rot[i * 3 + 2] * nm[2];
    nn = R_SQRT(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + eps);
    for (int i = 0; i < 3; ++i) n[i] /= nn;
    REAL rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    if (!(rn < 0)) return;
    REAL rt[3] = {rv[0] - rn * n[0], rv[1] - rn * n[1], rv[2] - rn * n[2]};
    REAL rtn = R_SQRT(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] + eps);
    REAL sc = rtn + rn * c->friction;
    sc = (sc > 0 ? sc : 0) / rtn;
    for (int i = 0; i < 3; ++i) v[i] = vc[i] + rt[i] * sc * infl + rv[i] * (1 - infl);
}

/* constant-velocity kinematic motion over one substep */
static void advance_collider(ref_collider* c, REAL dt) {
    for (int d = 0; d < 3; ++d) c->pos[d] += c->lin_vel[d] * dt;
    if (c->kind == 3 && c->pos[2] < c->floor) c->pos[2] = c->floor; /* FloorBoundary.impose_pos */
    REAL wx = c->ang_vel[0] * dt, wy = c->ang_vel[1] * dt, wz = c->ang_vel[2] * dt;
    REAL th = R_SQRT(wx * wx + wy * wy + wz * wz);
    if (th > 0) {
        REAL kx = wx / th, ky = wy / th, kz = wz / th, s = R_SIN(th), co = R_COS(th), t = 1 - co;
        REAL E[9] = {co + t * kx * kx, t * kx * ky - s * kz, t * kx * kz + s * ky, t * kx * ky + s * kz, co + t * ky * ky,
                     t * ky * kz - s * kx, t * kx * kz - s * ky, t * ky * kz + s * kx, co + t * kz * kz};
        REAL R[9];
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                R[a * 3 + b] = E[a * 3 + 0] * c->rot[0 * 3 + b] + E[a * 3 + 1] * c->rot[1 * 3 + b] + E[a * 3 + 2] * c->rot[2 * 3 + b];
        memcpy(c->rot, R, sizeof(R));
    }
}

/* as ref_substeps_ext, with kinematic rigid colliders coupled in the grid op
 * (legacy_coupler.py:385-397); forces (optional, [n_colliders][6]) accumulate the
 * reaction force and torque over all substeps; the colliders' poses advance in place */
int ref_substeps_full(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir,
                      ref_collider* colliders, int n_colliders, REAL* forces) {
    return ref_substeps_cpic(p, mats, n, x, v, C, F, Jp, mat, active, n_substeps, grid, gvel, n_threads, mu_p, lam_p,
                             actu, mdir, colliders, n_colliders, forces, NULL);
}

/* as ref_substeps_full, with CPIC (mpm_solver.py:357-379, 412-427; legacy_coupler.py:498-525)
 * when rnormal ([n_colliders][n][3], the particles' remembered collider-side normals, zero
 * at the start) is given: at the start of each substep every active particle takes the
 * collider's normal at its position unless that points against the one it remembers (it has
 * crossed the collider); p2g skips the stencil nodes whose normal points against the
 * particle's for some collider (the first such collider separates them), and g2p takes for
 * those nodes, instead of the grid velocity, the particle's own velocity after the rigid
 * response along its remembered normal (influence 1; the reaction goes to forces).  The
 * normals and p2g see the colliders' poses at the start of the substep, g2p the advanced
 * ones. */
int ref_substeps_cpic(const ref_params* p, const ref_material* mats, int n, REAL* x, REAL* v, REAL* C, REAL* F,
                      REAL* Jp, const int32_t* mat, const uint8_t* active, int n_substeps, REAL* grid, REAL* gvel,
                      int n_threads, const REAL* mu_p, const REAL* lam_p, const REAL* actu, const REAL* mdir,
                      ref_collider* colliders, int n_colliders, REAL* forces, REAL* rnormal) {
    signed char* sep = NULL;
    if (rnormal && n_colliders > 0) {
        sep = (signed char*)malloc((size_t)n * 27);
        if (!sep) return 4;
    } else {
        rnormal = NULL;
    }
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#endif
    const int64_t G = (int64_t)p->res[0] * p->res[1] * p->res[2];
    int status = 0;
    for (int step = 0; step < n_substeps; ++step) {
#pragma omp parallel for schedule(static)
        for (int64_t g = 0; g < G; ++g) {
            grid[4 * g + 0] = grid[4 * g + 1] = grid[4 * g + 2] = grid[4 * g + 3] = 0;
        }
        if (rnormal) {
            /* coupler.preprocess -> mpm_surface_to_particle (legacy_coupler.py:498-525) */
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) {
                if (!active[i]) continue;
                for (int k = 0; k < n_colliders; ++k) {
                    if (colliders[k].kind == 3) continue; /* CPIC: rigid geoms only */
                    REAL nn[3];
                    REAL* o = rnormal + 3 * ((int64_t)k * n + i);
                    sdf_normal(&colliders[k], p->eps, x + 3 * i, nn);
                    if (nn[0] * o[0] + nn[1] * o[1] + nn[2] * o[2] >= 0) {
                        o[0] = nn[0];
                        o[1] = nn[1];
                        o[2] = nn[2];
                    }
                }
            }
        }
        /* p2g (mpm_solver.py:290-389) */
#pragma omp parallel for schedule(static) reduction(| : status)
        for (int i = 0; i < n; ++i) {
            if (!active[i]) continue;
            const REAL* Ci = C + 9 * i;
            REAL* Fi = F + 9 * i;
            REAL Ft[9], U[9], S[3], V[9], Fn[9], st[9], Jpn;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    REAL acc = Fi[a * 3 + b];
                    for (int k = 0; k < 3; ++k) acc += p->dt * Ci[a * 3 + k] * Fi[k * 3 + b];
                    Ft[a * 3 + b] = acc;
                }
            ref_svd3(Ft, U, S, V);
            REAL J = S[0] * (S[1] * S[2]);
            const ref_material* m = &mats[mat[i]];
            ref_material mp;
            if (mu_p) {
                mp = *m;
                mp.mu = mu_p[i];
                mp.lam = lam_p[i];
                m = &mp;
            }
            if (g_branch_margin) record_branch_margin(m, p->eps, S, Jp[i], &g_branch_margin[i]);
            constitutive(m, p->eps, J, Ft, U, S, V, Jp[i], Fn, &Jpn, st);
            if ((m->flags & 4) && actu) {
                /* muscle.py:57-65: stress += stiffness * actu * F_tmp (d d^T) F_tmp^T */
                const REAL* d = mdir + 3 * i;
                REAL fd[3];
                for (int a = 0; a < 3; ++a) fd[a] = Ft[a * 3] * d[0] + Ft[a * 3 + 1] * d[1] + Ft[a * 3 + 2] * d[2];
                const REAL k = m->muscle_stiffness * actu[i];
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) st[a * 3 + b] += k * fd[a] * fd[b];
            }
            memcpy(Fi, Fn, 9 * sizeof(REAL));
            Jp[i] = Jpn;
            REAL A[9];
            for (int k = 0; k < 9; ++k) A[k] = p->stress_scale * st[k] + m->mass * Ci[k];
            int base[3];
            REAL fx[3], w[3][3];
            for (int d = 0; d < 3; ++d) {
                REAL xi = x[3 * i + d] * p->inv_dx;
                REAL bf = RFLOOR(xi - (REAL)0.5);
                base[d] = (int)bf - p->lower_cell[d];
                fx[d] = xi - bf;
                w[0][d] = (REAL)0.5 * ((REAL)1.5 - fx[d]) * ((REAL)1.5 - fx[d]);
                w[1][d] = (REAL)0.75 - (fx[d] - 1) * (fx[d] - 1);
                w[2][d] = (REAL)0.5 * (fx[d] - (REAL)0.5) * (fx[d] - (REAL)0.5);
            }
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c) {
                        int gi = base[0] + a, gj = base[1] + b, gk = base[2] + c;
                        if (gi < 0 || gj < 0 || gk < 0 || gi >= p->res[0] || gj >= p->res[1] || gk >= p->res[2]) {
                            status |= 1;
                            continue;
                        }
                        if (sep) {
                            /* mpm_solver.py:357-379: is the node on the other side of a collider? */
                            const REAL cp[3] = {(REAL)(gi + p->lower_cell[0]) * p->dx,
                                                (REAL)(gj + p->lower_cell[1]) * p->dx,
                                                (REAL)(gk + p->lower_cell[2]) * p->dx};
                            int sg = -1;
                            for (int k = 0; k < n_colliders && sg < 0; ++k) {
                                if (colliders[k].kind == 3) continue;
                                REAL nc[3];
                                const REAL* np_ = rnormal + 3 * ((int64_t)k * n + i);
                                sdf_normal(&colliders[k], p->eps, cp, nc);
                                if (np_[0] * nc[0] + np_[1] * nc[1] + np_[2] * nc[2] < 0) sg = k;
                            }
                            sep[(int64_t)i * 27 + a * 9 + b * 3 + c] = (signed char)sg;
                            if (sg >= 0) continue;
                        }
                        REAL wt = w[a][0] * w[b][1] * w[c][2];
                        REAL dp[3] = {(a - fx[0]) * p->dx, (b - fx[1]) * p->dx, (c - fx[2]) * p->dx};
                        REAL* cell = grid + 4 * gidx(p, gi, gj, gk);
                        for (int d = 0; d < 3; ++d) {
                            REAL q = wt * (m->mass * v[3 * i + d] + A[d * 3 + 0] * dp[0] + A[d * 3 + 1] * dp[1] + A[d * 3 + 2] * dp[2]);
#pragma omp atomic
                            cell[d] += q;
                        }
#pragma omp atomic
                        cell[3] += wt * m->mass;
                    }
        }
        /* grid op (legacy_coupler.py:364-375, 495-496) */
#pragma omp parallel for schedule(static)
        for (int64_t g = 0; g < G; ++g) {
            REAL* cell = grid + 4 * g;
            REAL* out = gvel + 3 * g;
            out[0] = out[1] = out[2] = 0;
            if (cell[3] > p->eps) {
                int k = (int)(g % p->res[2]);
                int j = (int)((g / p->res[2]) % p->res[1]);
                int ii = (int)(g / ((int64_t)p->res[1] * p->res[2]));
                int I[3] = {ii, j, k};
                REAL inv = 1 / cell[3];
                REAL vel[3], pos[3];
                for (int d = 0; d < 3; ++d) {
                    vel[d] = inv * cell[d] + p->dt * p->gravity[d];
                    pos[d] = (REAL)(I[d] + p->lower_cell[d]) * p->dx;
                }
                /* MPM <-> rigid (legacy_coupler.py:385-397), node mass without the 1e3 volume scale */
                /* MPM <-> Tool first (legacy_coupler.py:381-383) */
                for (int k = 0; k < n_colliders; ++k)
                    if (colliders[k].kind == 3) collide_tool(&colliders[k], p->eps, p->dt, pos, vel);
                for (int k = 0; k < n_colliders; ++k)
                    if (colliders[k].kind != 3)
                        collide_rigid(&colliders[k], p->eps, p->dt, cell[3] / (REAL)1e3, pos, vel,
                                      forces ? forces + 6 * k : NULL);
                for (int d = 0; d < 3; ++d) out[d] = bc_vel(pos[d], vel[d], p->bnd_lo[d], p->bnd_hi[d]);
            }
        }
        for (int k = 0; k < n_colliders; ++k) advance_collider(&colliders[k], p->dt);
        /* g2p (mpm_solver.py:391-449) */
#pragma omp parallel for schedule(static) reduction(| : status)
        for (int i = 0; i < n; ++i) {
            if (!active[i]) continue;
            int base[3];
            REAL fx[3], w[3][3];
            for (int d = 0; d < 3; ++d) {
                REAL xi = x[3 * i + d] * p->inv_dx;
                REAL bf = RFLOOR(xi - (REAL)0.5);
                base[d] = (int)bf - p->lower_cell[d];
                fx[d] = xi - bf;
                w[0][d] = (REAL)0.5 * ((REAL)1.5 - fx[d]) * ((REAL)1.5 - fx[d]);
                w[1][d] = (REAL)0.75 - (fx[d] - 1) * (fx[d] - 1);
                w[2][d] = (REAL)0.5 * (fx[d] - (REAL)0.5) * (fx[d] - (REAL)0.5);
            }
            REAL nv[3] = {0, 0, 0}, nC[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c) {
                        int gi = base[0] + a, gj = base[1] + b, gk = base[2] + c;
                        if (gi < 0 || gj < 0 || gk < 0 || gi >= p->res[0] || gj >= p->res[1] || gk >= p->res[2]) {
                            status |= 1;
                            continue;
                        }
                        REAL wt = w[a][0] * w[b][1] * w[c][2];
                        const REAL* gv = gvel + 3 * gidx(p, gi, gj, gk);
                        REAL vs[3];
                        const int sg = sep ? sep[(int64_t)i * 27 + a * 9 + b * 3 + c] : -1;
                        if (sg >= 0) {
                            /* mpm_solver.py:412-427: the particle's own velocity after the rigid
                             * response along its remembered normal, mass m w / 1e3 */
                            const ref_collider* cs = &colliders[sg];
                            REAL q[3];
                            for (int d = 0; d < 3; ++d) {
                                q[d] = x[3 * i + d] - cs->pos[d];
                                vs[d] = v[3 * i + d];
                            }
                            rigid_respond(cs, p->eps, p->dt, mats[mat[i]].mass * wt / (REAL)1e3, q,
                                          rnormal + 3 * ((int64_t)sg * n + i), 1, vs, forces ? forces + 6 * sg : NULL);
                            gv = vs;
                        }
                        REAL dp[3] = {a - fx[0], b - fx[1], c - fx[2]};
                        for (int d = 0; d < 3; ++d) {
                            nv[d] += wt * gv[d];
                            for (int e = 0; e < 3; ++e) nC[d * 3 + e] += p->c_scale * wt * gv[d] * dp[e];
                        }
                    }
            for (int d = 0; d < 3; ++d) {
                REAL nx = x[3 * i + d] + p->dt * nv[d];
                REAL vv = bc_vel(nx, nv[d], p->bnd_lo[d], p->bnd_hi[d]);
                nx = RMAX(RMIN(nx, p->bnd_hi[d]), p->bnd_lo[d]);
                if (nx != nx) status |= 2;
                x[3 * i + d] = nx;
                v[3 * i + d] = vv;
            }
            memcpy(C + 9 * i, nC, 9 * sizeof(REAL));
        }
    }
    free(sep);
    return status;
}

int ref_sizeof_params(void) { return (int)sizeof(ref_params); }
int ref_sizeof_material(void) { return (int)sizeof(ref_material); }
int ref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
