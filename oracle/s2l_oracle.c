/*
 * s2l_oracle.c - CPU restatement of the reference's solve phase.  TEST INFRASTRUCTURE ONLY.
 *
 * This file is the oracle the GPU path is checked against: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it, and only as the checker or the timed CPU baseline.
 * It is never part of the product path.
 *
 * It restates, in plain sequential C, the algorithm of the reference (fraBuffoli/
 * Algebraic-Multilevel-Preconditioner) on one process holding every subdomain:
 *   - DistributedMatrix::apply          include/linalg/distributed_matrix.hpp:33-38
 *   - HaloExchange::forward/reverseAdd   src/linalg/halo_exchange.cpp:34-53, 86-107
 *   - LocalSolver::solve                src/linalg/local_solver.cpp:119-126 (Eigen triangular solves)
 *   - OneLevelSchwarz::apply            src/preconditioner/one_level_schwarz.cpp:80-99
 *   - CoarseSpace::restrict/prolong     src/preconditioner/coarse_space.cpp:208-230
 *   - CoarseSolver::solve (root)        src/preconditioner/coarse_solver.cpp:166-179 (direct solve of E)
 *   - TwoLevelSchwarz::apply            src/preconditioner/two_level_schwarz.cpp:134-163
 *   - Gmres::solve                      src/solver/gmres.cpp:18-161 (L2 and OpenFOAM stopping tests)
 *   - BiCgStab::solve                   src/solver/bicgstab.cpp:15-154 (L2 and OpenFOAM stopping tests)
 *   - detail::openfoamNormFactor        src/solver/krylov.cpp:48-58
 * The factors, coarse basis and coarse matrix are inputs (the setup phase produces them), in the
 * same conventions as include/s2l_gpu.h.  Parity of this restatement with the reference itself is
 * pinned by the golden fixtures under tests/golden/ (generated by running the reference).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int64_t begin;
    int n_owned, n_local;
    int64_t *l2g;       /* local -> global */
    double *D;
    int kind;           /* 0 LU, 1 LLT, 2 LDLT */
    int32_t *pin, *pout;
    int64_t *Lp, *Up;
    int32_t *Li, *Ui;
    double *Lx, *Ux, *d; /* values widened to double (float factors are exact in double) */
    int single;          /* 1: the solve runs in float, as the reference's float factors do */
    int m;
    double *V;           /* n_local x m column-major */
    double *rloc, *yloc; /* work */
    void *amg;           /* AMG local solver (oracle_add_subdomain_amg) instead of factors, or NULL */
} OSub;

typedef struct {
    int64_t n;
    int nsub, one_level, coarse, pou;
    int64_t *Ap, *Ai;
    double *Ax;
    OSub *sub;
    int64_t n0;
    int64_t *coff;
    double *ELU;   /* LU of E (row-major, partial pivoting) */
    int *piv;
    double *c, *y, *x0, *w, *z1, *tmp;
} OSetup;

static void amg_local(const void *h, const double *b, double *x);
static void amg_free(void *h);

/* ---------------------------------------------------------------------------------------- */
OSetup *oracle_setup_create(int64_t n, int nsub, int one_level, int coarse, int pou)
{
    OSetup *s = (OSetup *)calloc(1, sizeof(OSetup));
    s->n = n;
    s->nsub = nsub;
    s->one_level = one_level;
    s->coarse = coarse;
    s->pou = pou;
    s->sub = (OSub *)calloc((size_t)nsub, sizeof(OSub));
    s->x0 = (double *)calloc((size_t)n, sizeof(double));
    s->w = (double *)calloc((size_t)n, sizeof(double));
    s->z1 = (double *)calloc((size_t)n, sizeof(double));
    s->tmp = (double *)calloc((size_t)n, sizeof(double));
    return s;
}

void oracle_setup_destroy(OSetup *s)
{
    if (!s) return;
    for (int i = 0; i < s->nsub; ++i) {
        OSub *q = &s->sub[i];
        free(q->l2g); free(q->D); free(q->pin); free(q->pout); free(q->Lp); free(q->Up); free(q->Li);
        free(q->Ui); free(q->Lx); free(q->Ux); free(q->d); free(q->V); free(q->rloc); free(q->yloc);
        amg_free(q->amg);
    }
    free(s->sub); free(s->Ap); free(s->Ai); free(s->Ax); free(s->coff); free(s->ELU); free(s->piv);
    free(s->c); free(s->y); free(s->x0); free(s->w); free(s->z1); free(s->tmp);
    free(s);
}

void oracle_set_matrix(OSetup *s, const int64_t *rp, const int64_t *ci, const double *v)
{
    int64_t nnz = rp[s->n];
    s->Ap = (int64_t *)malloc((size_t)(s->n + 1) * sizeof(int64_t));
    s->Ai = (int64_t *)malloc((size_t)(nnz ? nnz : 1) * sizeof(int64_t));
    s->Ax = (double *)malloc((size_t)(nnz ? nnz : 1) * sizeof(double));
    memcpy(s->Ap, rp, (size_t)(s->n + 1) * sizeof(int64_t));
    memcpy(s->Ai, ci, (size_t)nnz * sizeof(int64_t));
    memcpy(s->Ax, v, (size_t)nnz * sizeof(double));
}

static double *dup_vals(const void *v, int64_t count, int single)
{
    double *o = (double *)malloc((size_t)(count ? count : 1) * sizeof(double));
    for (int64_t k = 0; k < count; ++k) o[k] = single ? (double)((const float *)v)[k] : ((const double *)v)[k];
    return o;
}

void oracle_add_subdomain(OSetup *s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t *ghosts,
                          const double *D, int kind, int single, const int32_t *pin, const int32_t *pout,
                          const int64_t *Lp, const int32_t *Li, const void *Lx, const int64_t *Up, const int32_t *Ui,
                          const void *Ux, const void *d, int m, const double *V)
{
    OSub *q = &s->sub[i];
    int nl = n_owned + n_ghost;
    q->begin = begin;
    q->n_owned = n_owned;
    q->n_local = nl;
    q->l2g = (int64_t *)malloc((size_t)nl * sizeof(int64_t));
    for (int j = 0; j < n_owned; ++j) q->l2g[j] = begin + j;
    for (int j = 0; j < n_ghost; ++j) q->l2g[n_owned + j] = ghosts[j];
    q->D = (double *)malloc((size_t)nl * sizeof(double));
    memcpy(q->D, D, (size_t)nl * sizeof(double));
    q->kind = kind;
    q->single = single;
    q->pin = (int32_t *)malloc((size_t)nl * sizeof(int32_t));
    q->pout = (int32_t *)malloc((size_t)nl * sizeof(int32_t));
    memcpy(q->pin, pin, (size_t)nl * sizeof(int32_t));
    memcpy(q->pout, pout, (size_t)nl * sizeof(int32_t));
    q->Lp = (int64_t *)malloc((size_t)(nl + 1) * sizeof(int64_t));
    memcpy(q->Lp, Lp, (size_t)(nl + 1) * sizeof(int64_t));
    q->Li = (int32_t *)malloc((size_t)(Lp[nl] ? Lp[nl] : 1) * sizeof(int32_t));
    memcpy(q->Li, Li, (size_t)Lp[nl] * sizeof(int32_t));
    q->Lx = dup_vals(Lx, Lp[nl], single);
    if (kind == 0) {
        q->Up = (int64_t *)malloc((size_t)(nl + 1) * sizeof(int64_t));
        memcpy(q->Up, Up, (size_t)(nl + 1) * sizeof(int64_t));
        q->Ui = (int32_t *)malloc((size_t)(Up[nl] ? Up[nl] : 1) * sizeof(int32_t));
        memcpy(q->Ui, Ui, (size_t)Up[nl] * sizeof(int32_t));
        q->Ux = dup_vals(Ux, Up[nl], single);
    }
    if (kind == 2) q->d = dup_vals(d, nl, single);
    q->m = m;
    if (m) {
        q->V = (double *)malloc((size_t)nl * m * sizeof(double));
        memcpy(q->V, V, (size_t)nl * m * sizeof(double));
    }
    q->rloc = (double *)calloc((size_t)nl, sizeof(double));
    q->yloc = (double *)calloc((size_t)nl, sizeof(double));
}

/* LU with partial pivoting of the coarse matrix (the root solver factorizes E once,
   src/preconditioner/coarse_solver.cpp:113-139).  Returns 0 if E is singular. */
int oracle_set_coarse(OSetup *s, int64_t n0, const int64_t *offsets, const double *E)
{
    int n = (int)n0;
    s->n0 = n0;
    s->coff = (int64_t *)malloc((size_t)(s->nsub + 1) * sizeof(int64_t));
    memcpy(s->coff, offsets, (size_t)(s->nsub + 1) * sizeof(int64_t));
    s->ELU = (double *)malloc((size_t)(n ? n : 1) * (n ? n : 1) * sizeof(double));
    memcpy(s->ELU, E, (size_t)n * n * sizeof(double));
    s->piv = (int *)malloc((size_t)(n ? n : 1) * sizeof(int));
    s->c = (double *)calloc((size_t)(n ? n : 1), sizeof(double));
    s->y = (double *)calloc((size_t)(n ? n : 1), sizeof(double));
    double *A = s->ELU;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[(size_t)i * n + k]) > best) { best = fabs(A[(size_t)i * n + k]); p = i; }
        if (best == 0.0) return 0;
        s->piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) { double t = A[(size_t)k * n + j]; A[(size_t)k * n + j] = A[(size_t)p * n + j]; A[(size_t)p * n + j] = t; }
        for (int i = k + 1; i < n; ++i) {
            double l = A[(size_t)i * n + k] / A[(size_t)k * n + k];
            A[(size_t)i * n + k] = l;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
        }
    }
    return 1;
}

/* ------------------------------------------------------------------------ building blocks */
/* y = A x (or y = b - A x) */
void oracle_spmv(const OSetup *s, const double *x, double *y)
{
    for (int64_t r = 0; r < s->n; ++r) {
        double t = 0.0;
        for (int64_t e = s->Ap[r]; e < s->Ap[r + 1]; ++e) t += s->Ax[e] * x[s->Ai[e]];
        y[r] = t;
    }
}

/* A_ii x = b with the factors: t = b[perm_in]; L u = t; U v = u; x = v[perm_out] */
static void local_solve_d(const OSub *q, const double *b, double *x, double *t)
{
    int n = q->n_local;
    for (int k = 0; k < n; ++k) t[k] = b[q->pin[k]];
    /* forward: L lower (unit for LU/LDLT) */
    for (int r = 0; r < n; ++r) {
        double acc = t[r], dg = 1.0;
        for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e) {
            int c = q->Li[e];
            if (c < r) acc -= q->Lx[e] * t[c];
            else if (c == r) dg = q->Lx[e];
        }
        t[r] = (q->kind == 1) ? acc / dg : acc;
    }
    if (q->kind == 0) { /* U upper */
        for (int r = n - 1; r >= 0; --r) {
            double acc = t[r], dg = 1.0;
            for (int64_t e = q->Up[r]; e < q->Up[r + 1]; ++e) {
                int c = q->Ui[e];
                if (c > r) acc -= q->Ux[e] * t[c];
                else if (c == r) dg = q->Ux[e];
            }
            t[r] = acc / dg;
        }
    } else { /* U = L^T (LLT) or diag(d) L^T (LDLT): column sweep over the rows of L */
        if (q->kind == 2)
            for (int r = 0; r < n; ++r) t[r] /= q->d[r];
        for (int r = n - 1; r >= 0; --r) {
            double dg = 1.0;
            if (q->kind == 1)
                for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e)
                    if (q->Li[e] == r) dg = q->Lx[e];
            t[r] /= dg;
            for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e) {
                int c = q->Li[e];
                if (c < r) t[c] -= q->Lx[e] * t[r];
            }
        }
    }
    for (int j = 0; j < n; ++j) x[j] = t[q->pout[j]];
}

/* the same solve with float arithmetic (factors stored in float, rhs rounded to float,
   src/linalg/local_solver.cpp:76-84) */
static void local_solve_f(const OSub *q, const double *b, double *x, float *t)
{
    int n = q->n_local;
    for (int k = 0; k < n; ++k) t[k] = (float)b[q->pin[k]];
    for (int r = 0; r < n; ++r) {
        float acc = t[r], dg = 1.0f;
        for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e) {
            int c = q->Li[e];
            if (c < r) acc -= (float)q->Lx[e] * t[c];
            else if (c == r) dg = (float)q->Lx[e];
        }
        t[r] = (q->kind == 1) ? acc / dg : acc;
    }
    if (q->kind == 0) {
        for (int r = n - 1; r >= 0; --r) {
            float acc = t[r], dg = 1.0f;
            for (int64_t e = q->Up[r]; e < q->Up[r + 1]; ++e) {
                int c = q->Ui[e];
                if (c > r) acc -= (float)q->Ux[e] * t[c];
                else if (c == r) dg = (float)q->Ux[e];
            }
            t[r] = acc / dg;
        }
    } else {
        if (q->kind == 2)
            for (int r = 0; r < n; ++r) t[r] /= (float)q->d[r];
        for (int r = n - 1; r >= 0; --r) {
            float dg = 1.0f;
            if (q->kind == 1)
                for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e)
                    if (q->Li[e] == r) dg = (float)q->Lx[e];
            t[r] /= dg;
            for (int64_t e = q->Lp[r]; e < q->Lp[r + 1]; ++e) {
                int c = q->Li[e];
                if (c < r) t[c] -= (float)q->Lx[e] * t[r];
            }
        }
    }
    for (int j = 0; j < n; ++j) x[j] = (double)t[q->pout[j]];
}

void oracle_local_solve(const OSetup *s, int i, const double *b, double *x)
{
    const OSub *q = &s->sub[i];
    if (q->amg) {
        amg_local(q->amg, b, x);
        return;
    }
    if (q->single) {
        float *t = (float *)malloc((size_t)q->n_local * sizeof(float));
        local_solve_f(q, b, x, t);
        free(t);
    } else {
        double *t = (double *)malloc((size_t)q->n_local * sizeof(double));
        local_solve_d(q, b, x, t);
        free(t);
    }
}

/* z = M1^-1 r: halo forward, A_ii^-1, D (RAS), reverse accumulation (one_level_schwarz.cpp:80-99) */
void oracle_one_level(OSetup *s, const double *r, double *z)
{
    int boolean = s->pou == 0, ras = s->one_level == 0;
    for (int64_t g = 0; g < s->n; ++g) z[g] = 0.0;
    for (int i = 0; i < s->nsub; ++i) {
        OSub *q = &s->sub[i];
        for (int j = 0; j < q->n_local; ++j) q->rloc[j] = r[q->l2g[j]]; /* R_i r (owned + forward) */
        oracle_local_solve(s, i, q->rloc, q->yloc);
        if (ras)
            for (int j = 0; j < q->n_local; ++j) q->yloc[j] *= q->D[j];
    }
    /* z = sum_i R_i^T y_i: own rows, then the ghost copies of the other subdomains in order */
    for (int i = 0; i < s->nsub; ++i) {
        OSub *q = &s->sub[i];
        for (int j = 0; j < q->n_owned; ++j) z[q->begin + j] += q->yloc[j];
    }
    if (!(ras && boolean))
        for (int i = 0; i < s->nsub; ++i) {
            OSub *q = &s->sub[i];
            for (int j = q->n_owned; j < q->n_local; ++j) z[q->l2g[j]] += q->yloc[j];
        }
}

/* x0 = R0^T E^-1 R0 r (coarse_space.cpp:208-246) */
void oracle_coarse_apply(OSetup *s, const double *r, double *x0)
{
    int n0 = (int)s->n0;
    for (int i = 0; i < s->nsub; ++i) { /* restrict: c_i = V_i^T R_i r */
        OSub *q = &s->sub[i];
        for (int a = 0; a < q->m; ++a) {
            double t = 0.0;
            for (int j = 0; j < q->n_local; ++j) t += q->V[(size_t)a * q->n_local + j] * r[q->l2g[j]];
            s->c[s->coff[i] + a] = t;
        }
    }
    /* solve E y = c with the LU */
    for (int k = 0; k < n0; ++k) s->y[k] = s->c[k];
    for (int k = 0; k < n0; ++k) { double t = s->y[k]; s->y[k] = s->y[s->piv[k]]; s->y[s->piv[k]] = t; }
    for (int i = 0; i < n0; ++i) {
        double t = s->y[i];
        for (int k = 0; k < i; ++k) t -= s->ELU[(size_t)i * n0 + k] * s->y[k];
        s->y[i] = t;
    }
    for (int i = n0 - 1; i >= 0; --i) {
        double t = s->y[i];
        for (int k = i + 1; k < n0; ++k) t -= s->ELU[(size_t)i * n0 + k] * s->y[k];
        s->y[i] = t / s->ELU[(size_t)i * n0 + i];
    }
    /* prolong: x = sum_j R_j^T V_j y_j */
    for (int64_t g = 0; g < s->n; ++g) x0[g] = 0.0;
    for (int i = 0; i < s->nsub; ++i) {
        OSub *q = &s->sub[i];
        for (int j = 0; j < q->n_local; ++j) {
            double t = 0.0;
            for (int a = 0; a < q->m; ++a) t += q->V[(size_t)a * q->n_local + j] * s->y[s->coff[i] + a];
            if (j < q->n_owned || s->pou != 0) x0[q->l2g[j]] += t;
        }
    }
}

/* two_level_schwarz.cpp:134-163 */
void oracle_apply(OSetup *s, const double *r, double *z)
{
    if (s->coarse == 0 || s->n0 == 0) { oracle_one_level(s, r, z); return; }
    oracle_coarse_apply(s, r, s->x0);
    if (s->coarse == 1) {
        oracle_one_level(s, r, z);
        for (int64_t g = 0; g < s->n; ++g) z[g] += s->x0[g];
    } else {
        oracle_spmv(s, s->x0, s->w);
        for (int64_t g = 0; g < s->n; ++g) s->w[g] = r[g] - s->w[g];
        oracle_one_level(s, s->w, s->z1);
        for (int64_t g = 0; g < s->n; ++g) z[g] = s->x0[g] + s->z1[g];
    }
}

/* ------------------------------------------------------------------------ Krylov */
typedef struct {
    int converged, breakdown, iterations, restarts;
    double rel_residual, true_rel_residual;
    double initial_residual_of, final_residual_of; /* OpenFOAM test only (include/solver/krylov.hpp:51-52) */
    int history_len;
    double *history;
} OResult;

static double dotv(int64_t n, const double *a, const double *b)
{
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) t += a[i] * b[i];
    return t;
}

static double norm1v(int64_t n, const double *a)
{
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) t += fabs(a[i]);
    return t;
}

/* sum |a - alpha c| */
static double norm1_diff(int64_t n, const double *a, double alpha, const double *c)
{
    double t = 0.0;
    for (int64_t i = 0; i < n; ++i) t += fabs(a[i] - alpha * c[i]);
    return t;
}

/* OpenFOAM normalisation factor of x0 (krylov.cpp:48-58), Ax0 = A x0 */
static double of_norm_factor(OSetup *s, const double *b, const double *x0, const double *Ax0)
{
    int64_t n = s->n;
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) sum += x0[i];
    double xm = n > 0 ? sum / (double)n : 0.0;
    if (xm == 0.0) return norm1v(n, Ax0) + norm1v(n, b) + 1e-20;
    double *ones = (double *)malloc((size_t)n * sizeof(double)), *rs = (double *)malloc((size_t)n * sizeof(double));
    for (int64_t i = 0; i < n; ++i) ones[i] = 1.0;
    oracle_spmv(s, ones, rs);
    double F = norm1_diff(n, Ax0, xm, rs) + norm1_diff(n, b, xm, rs) + 1e-20;
    free(ones);
    free(rs);
    return F;
}

static void hpush(OResult *res, int cap, double v)
{
    if (res->history && res->history_len < cap) res->history[res->history_len] = v;
    if (res->history_len < cap) res->history_len++;
}

/* gmres.cpp:18-161; flexible = 1 keeps Z_j (not in the reference), strict = 1 accepts only a true
   residual <= rtol (the reference accepts 1.1 rtol, gmres.cpp:148-156); stop_norm 1 = OpenFOAM test
   with absolute tolerance atol (gmres.cpp:41-56, 106-123, 145-150) */
int oracle_gmres(OSetup *s, const double *b, double *x, int m, double rtol, int maxit, int flexible, int strict,
                 int hist_cap, int stop_norm, double atol, OResult *res)
{
    const int of = stop_norm == 1;
    int64_t n = s->n;
    memset(res, 0, sizeof(*res) - sizeof(double *));
    res->history_len = 0;
    double bnorm = sqrt(dotv(n, b, b));
    if (bnorm == 0.0) {
        memset(x, 0, (size_t)n * sizeof(double));
        res->converged = 1;
        hpush(res, hist_cap, 0.0);
        return 0;
    }
    double *V = (double *)malloc((size_t)n * (m + 1) * sizeof(double));
    double *Z = flexible ? (double *)malloc((size_t)n * m * sizeof(double)) : NULL;
    double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
    double *cs = (double *)calloc((size_t)m, sizeof(double)), *sn = (double *)calloc((size_t)m, sizeof(double));
    double *g = (double *)calloc((size_t)m + 1, sizeof(double)), *h = (double *)calloc((size_t)m + 1, sizeof(double));
    double *h2 = (double *)calloc((size_t)m + 1, sizeof(double)), *yv = (double *)calloc((size_t)m + 1, sizeof(double));
    double *r = (double *)malloc((size_t)n * sizeof(double)), *w = (double *)malloc((size_t)n * sizeof(double));
    double *zz = (double *)malloc((size_t)n * sizeof(double)), *u = (double *)malloc((size_t)n * sizeof(double));
#define HH(i, j) H[(size_t)(j) * (m + 1) + (i)]
    oracle_spmv(s, x, r);
    double normF = 1.0, l1 = 0.0, thr = 0.0;
    if (of) normF = of_norm_factor(s, b, x, r);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double beta = sqrt(dotv(n, r, r));
    hpush(res, hist_cap, beta / bnorm);
    res->rel_residual = beta / bnorm;
    int converged;
    if (of) {
        l1 = norm1v(n, r);
        res->initial_residual_of = l1 / normF;
        thr = fmax(rtol * l1, atol * normF);
        converged = l1 <= thr;
    } else {
        converged = beta <= rtol * bnorm;
    }
    while (!converged && res->iterations < maxit) {
        for (int64_t i = 0; i < n; ++i) V[i] = r[i] / beta;
        memset(g, 0, (size_t)(m + 1) * sizeof(double));
        g[0] = beta;
        memset(H, 0, (size_t)(m + 1) * m * sizeof(double));
        int k = 0, breakdown = 0;
        for (int j = 0; j < m && res->iterations < maxit; ++j) {
            double *zj = flexible ? Z + (size_t)j * n : zz;
            oracle_apply(s, V + (size_t)j * n, zj);
            oracle_spmv(s, zj, w);
            for (int i = 0; i <= j; ++i) h[i] = dotv(n, V + (size_t)i * n, w);
            for (int i = 0; i <= j; ++i) { double c = h[i]; const double *vi = V + (size_t)i * n; for (int64_t t = 0; t < n; ++t) w[t] -= c * vi[t]; }
            for (int i = 0; i <= j; ++i) h2[i] = dotv(n, V + (size_t)i * n, w);
            for (int i = 0; i <= j; ++i) { double c = h2[i]; const double *vi = V + (size_t)i * n; for (int64_t t = 0; t < n; ++t) w[t] -= c * vi[t]; }
            double hn = sqrt(dotv(n, w, w));
            for (int i = 0; i <= j; ++i) HH(i, j) = h[i] + h2[i];
            HH(j + 1, j) = hn;
            if (hn > 0.0)
                for (int64_t t = 0; t < n; ++t) V[(size_t)(j + 1) * n + t] = w[t] / hn;
            for (int i = 0; i < j; ++i) {
                double t = cs[i] * HH(i, j) + sn[i] * HH(i + 1, j);
                HH(i + 1, j) = -sn[i] * HH(i, j) + cs[i] * HH(i + 1, j);
                HH(i, j) = t;
            }
            double den = hypot(HH(j, j), HH(j + 1, j));
            cs[j] = den > 0.0 ? HH(j, j) / den : 1.0;
            sn[j] = den > 0.0 ? HH(j + 1, j) / den : 0.0;
            HH(j, j) = den;
            HH(j + 1, j) = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++k;
            ++res->iterations;
            res->rel_residual = fabs(g[j + 1]) / bnorm;
            hpush(res, hist_cap, res->rel_residual);
            int done;
            if (of) {
                /* r_j = g_{j+1} V_{j+2} Q^T e_{j+1} (gmres.cpp:106-123) */
                if (hn == 0.0 || g[j + 1] == 0.0) {
                    l1 = 0.0;
                } else {
                    double *q = (double *)calloc((size_t)j + 2, sizeof(double));
                    q[j + 1] = 1.0;
                    for (int i = j; i >= 0; --i) {
                        double qa = q[i], qc = q[i + 1];
                        q[i] = cs[i] * qa - sn[i] * qc;
                        q[i + 1] = sn[i] * qa + cs[i] * qc;
                    }
                    double acc1 = 0.0;
                    for (int64_t t = 0; t < n; ++t) {
                        double v = 0.0;
                        for (int c = 0; c < j + 2; ++c) v += V[(size_t)c * n + t] * q[c];
                        acc1 += fabs(v);
                    }
                    l1 = fabs(g[j + 1]) * acc1;
                    free(q);
                }
                done = l1 <= thr;
            } else {
                done = res->rel_residual <= rtol;
            }
            if (done) { converged = 1; break; }
            if (hn == 0.0) { breakdown = 1; break; }
        }
        for (int i = k - 1; i >= 0; --i) {
            double t = g[i];
            for (int c = i + 1; c < k; ++c) t -= HH(i, c) * yv[c];
            yv[i] = t / HH(i, i);
        }
        const double *B = flexible ? Z : V;
        for (int64_t t = 0; t < n; ++t) {
            double acc = 0.0;
            for (int c = 0; c < k; ++c) acc += B[(size_t)c * n + t] * yv[c];
            u[t] = acc;
        }
        if (flexible) {
            for (int64_t t = 0; t < n; ++t) x[t] += u[t];
        } else {
            oracle_apply(s, u, zz);
            for (int64_t t = 0; t < n; ++t) x[t] += zz[t];
        }
        oracle_spmv(s, x, r);
        for (int64_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
        beta = sqrt(dotv(n, r, r));
        if (of) l1 = norm1v(n, r);
        double slack = strict ? 1.0 : 1.1;
        int within = of ? l1 <= thr : beta <= rtol * bnorm;
        int within_slack = of ? l1 <= slack * thr : beta <= slack * rtol * bnorm;
        if (breakdown) converged = within || converged;
        if (converged && !within_slack) converged = 0;
        if (beta == 0.0) converged = 1;
        if (!converged) res->restarts++;
    }
#undef HH
    res->converged = converged;
    res->true_rel_residual = beta / bnorm;
    if (of) res->final_residual_of = l1 / normF;
    free(V); free(Z); free(H); free(cs); free(sn); free(g); free(h); free(h2); free(yv); free(r); free(w); free(zz); free(u);
    return 0;
}

/* bicgstab.cpp:15-154; stop_norm 1 = OpenFOAM test with absolute tolerance atol (bicgstab.cpp:33-66) */
int oracle_bicgstab(OSetup *s, const double *b, double *x, double rtol, int maxit, int strict, int hist_cap,
                    int stop_norm, double atol, OResult *res)
{
    const int of = stop_norm == 1;
    int64_t n = s->n;
    memset(res, 0, sizeof(*res) - sizeof(double *));
    double bnorm = sqrt(dotv(n, b, b));
    if (bnorm == 0.0) {
        memset(x, 0, (size_t)n * sizeof(double));
        res->converged = 1;
        hpush(res, hist_cap, 0.0);
        return 0;
    }
    size_t sz = (size_t)n * sizeof(double);
    double *r = (double *)malloc(sz), *rh = (double *)malloc(sz), *p = (double *)calloc((size_t)n, sizeof(double));
    double *v = (double *)calloc((size_t)n, sizeof(double)), *y = (double *)malloc(sz), *sv = (double *)malloc(sz);
    double *z = (double *)malloc(sz), *t = (double *)malloc(sz);
    oracle_spmv(s, x, r);
    double normF = 1.0, l1 = 0.0, thr = 0.0;
    if (of) normF = of_norm_factor(s, b, x, r);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - r[i];
    double rn = sqrt(dotv(n, r, r));
    if (of) {
        l1 = norm1v(n, r);
        res->initial_residual_of = l1 / normF;
        thr = fmax(rtol * l1, atol * normF);
    }
#define SATISFIED(slack) (of ? l1 <= (slack) * thr : rn <= (slack) * rtol * bnorm)
    hpush(res, hist_cap, rn / bnorm);
    res->rel_residual = rn / bnorm;
    for (;;) {
        if (SATISFIED(1.0)) { res->converged = 1; break; }
        if (res->iterations >= maxit) break;
        memcpy(rh, r, sz);
        double rhn = rn, rho = rn * rn, rho_old = 1.0, alpha = 1.0, omega = 1.0;
        int first = 1, candidate = 0;
        while (res->iterations < maxit) {
            if (first) memcpy(p, r, sz);
            else {
                double beta = (rho / rho_old) * (alpha / omega);
                for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
            }
            first = 0;
            oracle_apply(s, p, y);
            oracle_spmv(s, y, v);
            ++res->iterations;
            double rhv = dotv(n, rh, v);
            if (rhv == 0.0 || !isfinite(rhv)) { res->breakdown = 1; break; }
            alpha = rho / rhv;
            for (int64_t i = 0; i < n; ++i) sv[i] = r[i] - alpha * v[i];
            rn = sqrt(dotv(n, sv, sv));
            if (of) l1 = norm1v(n, sv);
            res->rel_residual = rn / bnorm;
            hpush(res, hist_cap, res->rel_residual);
            if (SATISFIED(1.0) || res->iterations >= maxit) {
                for (int64_t i = 0; i < n; ++i) x[i] += alpha * y[i];
                memcpy(r, sv, sz);
                candidate = SATISFIED(1.0);
                break;
            }
            oracle_apply(s, sv, z);
            oracle_spmv(s, z, t);
            ++res->iterations;
            double tt = dotv(n, t, t), ts = dotv(n, t, sv);
            omega = tt > 0.0 ? ts / tt : 0.0;
            for (int64_t i = 0; i < n; ++i) { x[i] += alpha * y[i] + omega * z[i]; r[i] = sv[i] - omega * t[i]; }
            rho_old = rho;
            rn = sqrt(dotv(n, r, r));
            rho = dotv(n, rh, r);
            if (of) l1 = norm1v(n, r);
            res->rel_residual = rn / bnorm;
            hpush(res, hist_cap, res->rel_residual);
            if (SATISFIED(1.0)) { candidate = 1; break; }
            if (omega == 0.0 || fabs(rho) < 1e-14 * rhn * rn) break;
        }
        oracle_spmv(s, x, t);
        for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
        rn = sqrt(dotv(n, r, r));
        if (of) l1 = norm1v(n, r);
        if (res->breakdown) break;
        if (candidate && SATISFIED(strict ? 1.0 : 1.1)) { res->converged = 1; break; }
        if (res->iterations >= maxit) break;
        res->restarts++;
    }
#undef SATISFIED
    res->true_rel_residual = rn / bnorm;
    if (of) res->final_residual_of = l1 / normF;
    free(r); free(rh); free(p); free(v); free(y); free(sv); free(z); free(t);
    return 0;
}

/* ---------------------------------------------------------------------------------------- */
/* Numeric refactorization on a kept factor pattern.
 *
 * The reference's UpdateLevel::Refactorize (include/preconditioner/preconditioner.hpp:15-30,
 * src/preconditioner/two_level_schwarz.cpp:30-41) refills A_ii from the new matrix
 * (Subdomain::refillValues, src/partition/subdomain.cpp:107-127) and calls
 * LocalSolver::refactorize (src/linalg/local_solver.cpp:111-118): Eigen's factorize() with the
 * ordering and elimination tree of analyzePattern() kept.  This restates that numeric step on the
 * factor pattern of include/s2l_gpu.h: the input is the permuted local matrix Ahat = P_in A_ii Q
 * (CSC, its pattern inside the factor's), with Ahat(p, q) = A_ii(perm_in[p], j) for
 * perm_out[j] = q.
 *   kind 0 (LU): left-looking LU with the setup's row order kept (no new pivoting); L unit lower
 *                with its diagonal stored, U upper.
 *   kind 1 (LL^T): left-looking Cholesky.
 * New values go to Lx (and Ux), in the CSR order of Lp/Li (Up/Ui).  Returns 0; -(j + 1) for a zero
 * (LU) or non-positive (LL^T) pivot in column j; -(n + 1) when an entry of Ahat lies outside the
 * factor pattern.
 */
int oracle_refactor(int n, int kind, const int64_t *Ap, const int32_t *Ai, const double *Ax, const int64_t *Lp,
                    const int32_t *Li, double *Lx, const int64_t *Up, const int32_t *Ui, double *Ux)
{
    /* column views of the CSR factors: per column, (row, CSR position) in increasing row order */
    int64_t *lcp = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t *ucp = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    const int64_t lnz = Lp[n], unz = kind == 0 ? Up[n] : 0;
    int32_t *lrow = (int32_t *)malloc((size_t)(lnz ? lnz : 1) * sizeof(int32_t));
    int64_t *lpos = (int64_t *)malloc((size_t)(lnz ? lnz : 1) * sizeof(int64_t));
    int32_t *urow = (int32_t *)malloc((size_t)(unz ? unz : 1) * sizeof(int32_t));
    int64_t *upos = (int64_t *)malloc((size_t)(unz ? unz : 1) * sizeof(int64_t));
    double *x = (double *)calloc((size_t)n + 1, sizeof(double));
    char *in = (char *)calloc((size_t)n + 1, 1);
    int rc = 0;
    for (int64_t e = 0; e < lnz; ++e) ++lcp[Li[e] + 1];
    for (int j = 0; j < n; ++j) lcp[j + 1] += lcp[j];
    for (int64_t e = 0; e < unz; ++e) ++ucp[Ui[e] + 1];
    for (int j = 0; j < n; ++j) ucp[j + 1] += ucp[j];
    {
        int64_t *nx = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
        memcpy(nx, lcp, ((size_t)n + 1) * sizeof(int64_t));
        for (int r = 0; r < n; ++r) /* rows in increasing order: each column's rows come out sorted */
            for (int64_t e = Lp[r]; e < Lp[r + 1]; ++e) {
                const int64_t q = nx[Li[e]]++;
                lrow[q] = r;
                lpos[q] = e;
            }
        if (kind == 0) {
            memcpy(nx, ucp, ((size_t)n + 1) * sizeof(int64_t));
            for (int r = 0; r < n; ++r)
                for (int64_t e = Up[r]; e < Up[r + 1]; ++e) {
                    const int64_t q = nx[Ui[e]]++;
                    urow[q] = r;
                    upos[q] = e;
                }
        }
        free(nx);
    }
    for (int j = 0; j < n && rc == 0; ++j) {
        /* work column on the pattern of column j */
        for (int64_t q = lcp[j]; q < lcp[j + 1]; ++q) {
            x[lrow[q]] = 0.0;
            in[lrow[q]] = 1;
        }
        for (int64_t q = ucp[j]; q < ucp[j + 1]; ++q) {
            x[urow[q]] = 0.0;
            in[urow[q]] = 1;
        }
        for (int64_t e = Ap[j]; e < Ap[j + 1]; ++e) {
            const int i = Ai[e];
            if (kind == 1 && i < j) continue; /* LL^T reads the lower triangle */
            if (!in[i]) {
                rc = -(n + 1);
                break;
            }
            x[i] += Ax[e];
        }
        if (rc) break;
        if (kind == 0) {
            /* U(:, j) by a sparse triangular solve with the finished columns of L, in row order */
            for (int64_t q = ucp[j]; q < ucp[j + 1]; ++q) {
                const int k = urow[q];
                if (k >= j) break;
                const double u = x[k];
                for (int64_t t = lcp[k]; t < lcp[k + 1]; ++t)
                    if (lrow[t] > k) x[lrow[t]] -= Lx[lpos[t]] * u;
            }
            const double piv = x[j];
            if (piv == 0.0 || !isfinite(piv)) {
                rc = -(j + 1);
                break;
            }
            for (int64_t q = ucp[j]; q < ucp[j + 1]; ++q) Ux[upos[q]] = x[urow[q]];
            for (int64_t q = lcp[j]; q < lcp[j + 1]; ++q) Lx[lpos[q]] = lrow[q] == j ? 1.0 : x[lrow[q]] / piv;
        } else {
            /* column j of L: Ahat(j:n, j) - sum_k L(j:n, k) L(j, k) over the finished columns k < j */
            for (int64_t e = Lp[j]; e < Lp[j + 1]; ++e) {
                const int k = Li[e];
                if (k >= j) break;
                const double ljk = Lx[e];
                for (int64_t t = lcp[k]; t < lcp[k + 1]; ++t)
                    if (lrow[t] >= j) x[lrow[t]] -= Lx[lpos[t]] * ljk;
            }
            const double d = x[j];
            if (!(d > 0.0) || !isfinite(d)) {
                rc = -(j + 1);
                break;
            }
            const double ljj = sqrt(d);
            for (int64_t q = lcp[j]; q < lcp[j + 1]; ++q) Lx[lpos[q]] = lrow[q] == j ? ljj : x[lrow[q]] / ljj;
        }
        for (int64_t q = lcp[j]; q < lcp[j + 1]; ++q) in[lrow[q]] = 0;
        for (int64_t q = ucp[j]; q < ucp[j + 1]; ++q) in[urow[q]] = 0;
    }
    free(lcp);
    free(ucp);
    free(lrow);
    free(lpos);
    free(urow);
    free(upos);
    free(x);
    free(in);
    return rc;
}

/* ---------------------------------------------------------------------------------------- */
/* One AMG V-cycle from x = 0: the reference's inexact local solve (--local-approx amg,
 * src/linalg/inexact_solver.cpp:89-95, AMGCL amg::apply / amg::cycle with serial Gauss-Seidel,
 * relaxation/gauss_seidel.hpp).  Levels 0 .. nlev-1 carry A_l (CSR, sorted columns) and, except a
 * last smoothed-only level, P_l (n_l x n_{l+1}) and R_l; the coarsest operator, when present, is
 * solved with its LU (row-major, partial pivoting, from oracle_dense_lu).
 *   level l: `sweeps` forward Gauss-Seidel sweeps on A_l x = f (x_i = (f_i - sum_{j != i} a_ij x_j)
 *            / a_ii in increasing i, updated values used at once), t = f - A_l x, f_{l+1} = R_l t,
 *            x_{l+1} = cycle(l + 1), x += P_l x_{l+1}, `sweeps` backward sweeps (decreasing i);
 *   coarsest: x = A_c^-1 f;  a last level without coarse solve: forward then backward sweeps.
 * Arrays: Ap/Ai/Ax[l], Pp/Pi/Px[l], Rp/Ri/Rx[l], nrow[l] (nlev + 1 sizes: nrow[nlev] = coarse
 * size, 0 without a coarse solve). */
typedef struct {
    int nlev, sweeps;
    const int *nrow;
    const int64_t *const *Ap, *const *Pp, *const *Rp;
    const int32_t *const *Ai, *const *Pi, *const *Ri;
    const double *const *Ax, *const *Px, *const *Rx;
    const double *CLU; /* coarse LU, row-major, partial pivoting */
    const int *Cpiv;
} OAmg;

static void gs_sweep(int n, const int64_t *p, const int32_t *ci, const double *v, const double *f, double *x,
                     int forward)
{
    for (int q = 0; q < n; ++q) {
        const int i = forward ? q : n - 1 - q;
        double D = 1.0, X = f[i];
        for (int64_t e = p[i]; e < p[i + 1]; ++e) {
            if (ci[e] == i) D = v[e];
            else X -= v[e] * x[ci[e]];
        }
        x[i] = (1.0 / D) * X;
    }
}

static void lu_solve(int n, const double *LU, const int *piv, const double *b, double *x)
{
    for (int i = 0; i < n; ++i) x[i] = b[i];
    for (int k = 0; k < n; ++k) {
        const int p = piv[k];
        if (p != k) {
            const double t = x[k];
            x[k] = x[p];
            x[p] = t;
        }
    }
    for (int i = 0; i < n; ++i) {
        double s = x[i];
        for (int k = 0; k < i; ++k) s -= LU[(size_t)i * n + k] * x[k];
        x[i] = s;
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (int k = i + 1; k < n; ++k) s -= LU[(size_t)i * n + k] * x[k];
        x[i] = s / LU[(size_t)i * n + i];
    }
}

static void amg_cycle(const OAmg *h, int l, const double *f, double *x)
{
    if (l == h->nlev) { /* coarsest, solved directly */
        lu_solve(h->nrow[l], h->CLU, h->Cpiv, f, x);
        return;
    }
    const int n = h->nrow[l];
    const int last_smoothed = (l == h->nlev - 1) && h->nrow[h->nlev] == 0;
    for (int s = 0; s < h->sweeps; ++s) gs_sweep(n, h->Ap[l], h->Ai[l], h->Ax[l], f, x, 1);
    if (last_smoothed) {
        for (int s = 0; s < h->sweeps; ++s) gs_sweep(n, h->Ap[l], h->Ai[l], h->Ax[l], f, x, 0);
        return;
    }
    const int nc = h->nrow[l + 1];
    double *t = (double *)malloc((size_t)(n ? n : 1) * sizeof(double));
    double *fc = (double *)malloc((size_t)(nc ? nc : 1) * sizeof(double));
    double *xc = (double *)calloc((size_t)(nc ? nc : 1), sizeof(double));
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t e = h->Ap[l][i]; e < h->Ap[l][i + 1]; ++e) s += h->Ax[l][e] * x[h->Ai[l][e]];
        t[i] = f[i] - s;
    }
    for (int i = 0; i < nc; ++i) {
        double s = 0.0;
        for (int64_t e = h->Rp[l][i]; e < h->Rp[l][i + 1]; ++e) s += h->Rx[l][e] * t[h->Ri[l][e]];
        fc[i] = s;
    }
    amg_cycle(h, l + 1, fc, xc);
    for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int64_t e = h->Pp[l][i]; e < h->Pp[l][i + 1]; ++e) s += h->Px[l][e] * xc[h->Pi[l][e]];
        x[i] += s;
    }
    for (int s = 0; s < h->sweeps; ++s) gs_sweep(n, h->Ap[l], h->Ai[l], h->Ax[l], f, x, 0);
    free(t);
    free(fc);
    free(xc);
}

/* LU with partial pivoting of a dense row-major n x n matrix, in place; 0 if singular. */
int oracle_dense_lu(int n, double *A, int *piv)
{
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[(size_t)i * n + k]) > best) {
                best = fabs(A[(size_t)i * n + k]);
                p = i;
            }
        if (best == 0.0) return 0;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                const double t = A[(size_t)k * n + j];
                A[(size_t)k * n + j] = A[(size_t)p * n + j];
                A[(size_t)p * n + j] = t;
            }
        for (int i = k + 1; i < n; ++i) {
            const double l = A[(size_t)i * n + k] / A[(size_t)k * n + k];
            A[(size_t)i * n + k] = l;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
        }
    }
    return 1;
}

void oracle_amg_apply(int nlev, int sweeps, const int *nrow, const int64_t *const *Ap, const int32_t *const *Ai,
                      const double *const *Ax, const int64_t *const *Pp, const int32_t *const *Pi,
                      const double *const *Px, const int64_t *const *Rp, const int32_t *const *Ri,
                      const double *const *Rx, const double *CLU, const int *Cpiv, const double *b, double *x)
{
    OAmg h = {nlev, sweeps, nrow, Ap, Pp, Rp, Ai, Pi, Ri, Ax, Px, Rx, CLU, Cpiv};
    const int n = nlev > 0 ? nrow[0] : nrow[0];
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    amg_cycle(&h, 0, b, x);
}

/* An owned copy of a hierarchy, for a subdomain of an OSetup (the reference's --local-approx amg). */
typedef struct {
    int nlev, sweeps;
    int *nrow; /* nlev + 1 entries, the last the coarse size (0: none) */
    int64_t **Ap, **Pp, **Rp;
    int32_t **Ai, **Pi, **Ri;
    double **Ax, **Px, **Rx;
    double *CLU;
    int *Cpiv;
} OAmgOwn;

static void *dupb(const void *p, size_t bytes)
{
    void *q = malloc(bytes ? bytes : 1);
    if (bytes) memcpy(q, p, bytes);
    return q;
}

static void amg_local(const void *hv, const double *b, double *x)
{
    const OAmgOwn *h = (const OAmgOwn *)hv;
    oracle_amg_apply(h->nlev, h->sweeps, h->nrow, (const int64_t *const *)h->Ap, (const int32_t *const *)h->Ai,
                     (const double *const *)h->Ax, (const int64_t *const *)h->Pp, (const int32_t *const *)h->Pi,
                     (const double *const *)h->Px, (const int64_t *const *)h->Rp, (const int32_t *const *)h->Ri,
                     (const double *const *)h->Rx, h->CLU, h->Cpiv, b, x);
}

static void amg_free(void *hv)
{
    OAmgOwn *h = (OAmgOwn *)hv;
    if (!h) return;
    for (int l = 0; l < h->nlev; ++l) {
        free(h->Ap[l]); free(h->Ai[l]); free(h->Ax[l]);
        free(h->Pp[l]); free(h->Pi[l]); free(h->Px[l]);
        free(h->Rp[l]); free(h->Ri[l]); free(h->Rx[l]);
    }
    free(h->Ap); free(h->Ai); free(h->Ax); free(h->Pp); free(h->Pi); free(h->Px);
    free(h->Rp); free(h->Ri); free(h->Rx); free(h->nrow); free(h->CLU); free(h->Cpiv);
    free(h);
}

/* Subdomain i with the AMG local solver (arguments as s2l_gpu_add_subdomain_amg).  Returns 0 if the
   coarsest operator is singular. */
int oracle_add_subdomain_amg(OSetup *s, int i, int64_t begin, int n_owned, int n_ghost, const int64_t *ghosts,
                             const double *D, int nlev, int sweeps, const int32_t *nrow,
                             const int64_t *const *Ap, const int32_t *const *Ai, const double *const *Ax,
                             const int64_t *const *Pp, const int32_t *const *Pi, const double *const *Px,
                             const int64_t *const *Rp, const int32_t *const *Ri, const double *const *Rx, int nc,
                             const double *C, int m, const double *V)
{
    OSub *q = &s->sub[i];
    const int nl = n_owned + n_ghost;
    memset(q, 0, sizeof(*q));
    q->begin = begin;
    q->n_owned = n_owned;
    q->n_local = nl;
    q->l2g = (int64_t *)malloc((size_t)nl * sizeof(int64_t));
    for (int j = 0; j < n_owned; ++j) q->l2g[j] = begin + j;
    for (int j = 0; j < n_ghost; ++j) q->l2g[n_owned + j] = ghosts[j];
    q->D = (double *)dupb(D, (size_t)nl * sizeof(double));
    q->m = m;
    if (m) q->V = (double *)dupb(V, (size_t)nl * m * sizeof(double));
    q->rloc = (double *)calloc((size_t)nl, sizeof(double));
    q->yloc = (double *)calloc((size_t)nl, sizeof(double));
    OAmgOwn *h = (OAmgOwn *)calloc(1, sizeof(OAmgOwn));
    h->nlev = nlev;
    h->sweeps = sweeps;
    h->nrow = (int *)malloc((size_t)(nlev + 1) * sizeof(int));
    for (int l = 0; l < nlev; ++l) h->nrow[l] = nrow[l];
    h->nrow[nlev] = nc;
    const int L = nlev ? nlev : 1;
    h->Ap = (int64_t **)calloc((size_t)L, sizeof(void *));
    h->Pp = (int64_t **)calloc((size_t)L, sizeof(void *));
    h->Rp = (int64_t **)calloc((size_t)L, sizeof(void *));
    h->Ai = (int32_t **)calloc((size_t)L, sizeof(void *));
    h->Pi = (int32_t **)calloc((size_t)L, sizeof(void *));
    h->Ri = (int32_t **)calloc((size_t)L, sizeof(void *));
    h->Ax = (double **)calloc((size_t)L, sizeof(void *));
    h->Px = (double **)calloc((size_t)L, sizeof(void *));
    h->Rx = (double **)calloc((size_t)L, sizeof(void *));
    for (int l = 0; l < nlev; ++l) {
        const int n = nrow[l];
        const int next = l + 1 < nlev ? nrow[l + 1] : nc;
        h->Ap[l] = (int64_t *)dupb(Ap[l], (size_t)(n + 1) * sizeof(int64_t));
        h->Ai[l] = (int32_t *)dupb(Ai[l], (size_t)Ap[l][n] * sizeof(int32_t));
        h->Ax[l] = (double *)dupb(Ax[l], (size_t)Ap[l][n] * sizeof(double));
        if (next > 0) {
            h->Pp[l] = (int64_t *)dupb(Pp[l], (size_t)(n + 1) * sizeof(int64_t));
            h->Pi[l] = (int32_t *)dupb(Pi[l], (size_t)Pp[l][n] * sizeof(int32_t));
            h->Px[l] = (double *)dupb(Px[l], (size_t)Pp[l][n] * sizeof(double));
            h->Rp[l] = (int64_t *)dupb(Rp[l], (size_t)(next + 1) * sizeof(int64_t));
            h->Ri[l] = (int32_t *)dupb(Ri[l], (size_t)Rp[l][next] * sizeof(int32_t));
            h->Rx[l] = (double *)dupb(Rx[l], (size_t)Rp[l][next] * sizeof(double));
        }
    }
    h->CLU = (double *)dupb(C ? C : D, C ? (size_t)nc * nc * sizeof(double) : 0);
    h->Cpiv = (int *)calloc((size_t)(nc ? nc : 1), sizeof(int));
    q->amg = h;
    if (nc && !oracle_dense_lu(nc, h->CLU, h->Cpiv)) return 0;
    return 1;
}
