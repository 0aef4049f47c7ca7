/*
 * CPU port of the FIT-TD step -- TEST INFRASTRUCTURE AND CPU BASELINE ONLY.
 *
 * A C + OpenMP restatement of one leapfrog step of the reference's CPU path:
 *   - the fused Numba kernels update_E_fused / update_H_fused
 *     (src/magnelio/_operators/numba_kernels.py:36-127), conditional dual
 *     curl accumulated in double as the Numba kernels do (curl = 0.0);
 *   - CPMLBoundary.update_E / update_H (src/magnelio/boundaries/cpml.py
 *     :343-516), element order b*psi, + c*d, * air, then E +-= beta*(ck*d+psi);
 *   - the series-R lumped port update_e
 *     (src/magnelio/ports/_lumped/operator.py:134-166);
 *   - running-DFT monitors with complex128 accumulation
 *     (src/magnelio/monitors/field_frequency.py:249-294, base.py:51-168,
 *     _dft.py:37-52).
 * REAL is float (the reference's default single precision) or double; the
 * file is compiled once per type with -DREAL=... -DSFX=... .
 * Nothing in the engine links or calls this code.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#define SFX f32
#endif
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

typedef struct {
    int axis, side, n;
    const REAL *b, *c, *ck;   /* [n] */
    REAL *psi[4];             /* reference psi shapes E1, E2, H1, H2 */
    const REAL *air[4];       /* same shapes, or NULL */
} fitc_face;

typedef struct {
    int n_edges;
    const int64_t *idx;
    const double *sign, *beta;
    double R, beta_sum, rec_scale;
    const double *vsrc;
    int64_t n_src;
    double i_prev;
    double *V, *I;            /* [steps] recorder output */
} fitc_lumped;

typedef struct {
    int i0, i1, j0, j1, k0, k1;
    int ncomp, comps[6];
    int nf;
    const double *omega;
    int stride;
    double *re, *im;          /* [ncomp][nf][cells] */
} fitc_mon;

typedef struct {
    int nx, ny, nz;
    REAL *e, *h;
    const REAL *aE, *bE, *aH, *bH;
    int nfaces;
    fitc_face faces[6];
    int nlumped;
    fitc_lumped lumped[4];
    int nmon;
    fitc_mon mon[4];
    const double *dx, *dy, *dz;
    double dt;
    int64_t n;
} fitc_problem;

#define IDX(i, j, k, NJ, NK) (((int64_t)(i) * (NJ) + (j)) * (NK) + (k))

static void update_E(fitc_problem *p) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int64_t nEx = (int64_t)nx * (ny + 1) * (nz + 1), nEy = (int64_t)(nx + 1) * ny * (nz + 1);
    const int64_t nHx = (int64_t)(nx + 1) * ny * nz, nHy = (int64_t)nx * (ny + 1) * nz;
    REAL *Ex = p->e, *Ey = p->e + nEx, *Ez = p->e + nEx + nEy;
    const REAL *Hx = p->h, *Hy = p->h + nHx, *Hz = p->h + nHx + nHy;
    const REAL *aEx = p->aE, *aEy = p->aE + nEx, *aEz = p->aE + nEx + nEy;
    const REAL *bEx = p->bE, *bEy = p->bE + nEx, *bEz = p->bE + nEx + nEy;
    int ni, nj, nk;
    /* Ex (nx, ny+1, nz+1): dHz/dy - dHy/dz */
    ni = nx; nj = ny + 1; nk = nz + 1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j)
            for (int k = 0; k < nk; ++k) {
                double c = 0.0;
                if (j < nj - 1) c += Hz[IDX(i, j, k, ny, nz + 1)];
                if (j > 0) c -= Hz[IDX(i, j - 1, k, ny, nz + 1)];
                if (k < nk - 1) c -= Hy[IDX(i, j, k, ny + 1, nz)];
                if (k > 0) c += Hy[IDX(i, j, k - 1, ny + 1, nz)];
                int64_t o = IDX(i, j, k, nj, nk);
                Ex[o] = (REAL)((double)(aEx[o] * Ex[o]) + (double)bEx[o] * c);
            }
    /* Ey (nx+1, ny, nz+1): dHx/dz - dHz/dx */
    ni = nx + 1; nj = ny; nk = nz + 1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j)
            for (int k = 0; k < nk; ++k) {
                double c = 0.0;
                if (k < nk - 1) c += Hx[IDX(i, j, k, ny, nz)];
                if (k > 0) c -= Hx[IDX(i, j, k - 1, ny, nz)];
                if (i < ni - 1) c -= Hz[IDX(i, j, k, ny, nz + 1)];
                if (i > 0) c += Hz[IDX(i - 1, j, k, ny, nz + 1)];
                int64_t o = IDX(i, j, k, nj, nk);
                Ey[o] = (REAL)((double)(aEy[o] * Ey[o]) + (double)bEy[o] * c);
            }
    /* Ez (nx+1, ny+1, nz): dHy/dx - dHx/dy */
    ni = nx + 1; nj = ny + 1; nk = nz;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < ni; ++i)
        for (int j = 0; j < nj; ++j)
            for (int k = 0; k < nk; ++k) {
                double c = 0.0;
                if (i < ni - 1) c += Hy[IDX(i, j, k, ny + 1, nz)];
                if (i > 0) c -= Hy[IDX(i - 1, j, k, ny + 1, nz)];
                if (j < nj - 1) c -= Hx[IDX(i, j, k, ny, nz)];
                if (j > 0) c += Hx[IDX(i, j - 1, k, ny, nz)];
                int64_t o = IDX(i, j, k, nj, nk);
                Ez[o] = (REAL)((double)(aEz[o] * Ez[o]) + (double)bEz[o] * c);
            }
}

static void update_H(fitc_problem *p) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    const int64_t nEx = (int64_t)nx * (ny + 1) * (nz + 1), nEy = (int64_t)(nx + 1) * ny * (nz + 1);
    const int64_t nHx = (int64_t)(nx + 1) * ny * nz, nHy = (int64_t)nx * (ny + 1) * nz;
    const REAL *Ex = p->e, *Ey = p->e + nEx, *Ez = p->e + nEx + nEy;
    REAL *Hx = p->h, *Hy = p->h + nHx, *Hz = p->h + nHx + nHy;
    const REAL *aHx = p->aH, *aHy = p->aH + nHx, *aHz = p->aH + nHx + nHy;
    const REAL *bHx = p->bH, *bHy = p->bH + nHx, *bHz = p->bH + nHx + nHy;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx + 1; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                double c = (double)Ez[IDX(i, j + 1, k, ny + 1, nz)] - Ez[IDX(i, j, k, ny + 1, nz)] -
                           Ey[IDX(i, j, k + 1, ny, nz + 1)] + Ey[IDX(i, j, k, ny, nz + 1)];
                int64_t o = IDX(i, j, k, ny, nz);
                Hx[o] = (REAL)((double)(aHx[o] * Hx[o]) - (double)bHx[o] * c);
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny + 1; ++j)
            for (int k = 0; k < nz; ++k) {
                double c = (double)Ex[IDX(i, j, k + 1, ny + 1, nz + 1)] - Ex[IDX(i, j, k, ny + 1, nz + 1)] -
                           Ez[IDX(i + 1, j, k, ny + 1, nz)] + Ez[IDX(i, j, k, ny + 1, nz)];
                int64_t o = IDX(i, j, k, ny + 1, nz);
                Hy[o] = (REAL)((double)(aHy[o] * Hy[o]) - (double)bHy[o] * c);
            }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz + 1; ++k) {
                double c = (double)Ey[IDX(i + 1, j, k, ny, nz + 1)] - Ey[IDX(i, j, k, ny, nz + 1)] -
                           Ex[IDX(i, j + 1, k, ny + 1, nz + 1)] + Ex[IDX(i, j, k, ny + 1, nz + 1)];
                int64_t o = IDX(i, j, k, ny, nz + 1);
                Hz[o] = (REAL)((double)(aHz[o] * Hz[o]) - (double)bHz[o] * c);
            }
}

/* Reference shape of component c (0..5 = Ex..Hz). */
static void shape_of(const fitc_problem *p, int c, int *a, int *b, int *d) {
    *a = p->nx + ((c == 1 || c == 2 || c == 3) ? 1 : 0);
    *b = p->ny + ((c == 0 || c == 2 || c == 4) ? 1 : 0);
    *d = p->nz + ((c == 0 || c == 1 || c == 5) ? 1 : 0);
}

static REAL *comp_ptr(const fitc_problem *p, int c) {
    int64_t off = 0;
    for (int q = (c < 3 ? 0 : 3); q < c; ++q) {
        int a, b, d;
        shape_of(p, q, &a, &b, &d);
        off += (int64_t)a * b * d;
    }
    return (c < 3 ? p->e : p->h) + off;
}

static const REAL *coef_ptr(const fitc_problem *p, const REAL *base, int c) {
    int64_t off = 0;
    for (int q = (c < 3 ? 0 : 3); q < c; ++q) {
        int a, b, d;
        shape_of(p, q, &a, &b, &d);
        off += (int64_t)a * b * d;
    }
    return base + off;
}

/* One CPML face, E side (phase 0) or H side (phase 1). */
static void cpml(fitc_problem *p, const fitc_face *f, int phase) {
    static const int tgt[3][4] = {{1, 2, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 4}};
    static const int src[3][4] = {{5, 4, 2, 1}, {5, 3, 2, 0}, {4, 3, 1, 0}};
    static const int sgn[3][4] = {{+1, -1, -1, +1}, {-1, +1, +1, -1}, {+1, -1, -1, +1}};
    const int ax = f->axis, n = f->n;
    const int N = ax == 0 ? p->nx : (ax == 1 ? p->ny : p->nz);
    const int k0 = f->side == 0 ? 0 : N - n;
    for (int q = 2 * phase; q < 2 * phase + 2; ++q) {
        const int tc = tgt[ax][q], sc = src[ax][q];
        REAL *T = comp_ptr(p, tc);
        const REAL *S = comp_ptr(p, sc);
        const REAL *beta = coef_ptr(p, tc < 3 ? p->bE : p->bH, tc);
        int ta, tb, td, sa, sb, sd;
        shape_of(p, tc, &ta, &tb, &td);
        shape_of(p, sc, &sa, &sb, &sd);
        int pa = ta, pb = tb, pd = td;
        if (ax == 0) pa = n;
        if (ax == 1) pb = n;
        if (ax == 2) pd = n;
        REAL *psi = f->psi[q];
        const REAL *air = f->air[q];
#pragma omp parallel for schedule(static)
        for (int a = 0; a < pa; ++a)
            for (int b = 0; b < pb; ++b)
                for (int d = 0; d < pd; ++d) {
                    const int l = ax == 0 ? a : (ax == 1 ? b : d);
                    int ia = a, ib = b, id = d;
                    if (ax == 0) ia = k0 + l;
                    if (ax == 1) ib = k0 + l;
                    if (ax == 2) id = k0 + l;
                    REAL dv;
                    if (phase == 0) { /* backward H difference, none at the min-side first layer */
                        REAL cur = S[IDX(ia, ib, id, sb, sd)];
                        REAL prv = 0;
                        int pa_ = ia, pb_ = ib, pd_ = id;
                        if (ax == 0) pa_ -= 1;
                        if (ax == 1) pb_ -= 1;
                        if (ax == 2) pd_ -= 1;
                        if ((ax == 0 ? pa_ : (ax == 1 ? pb_ : pd_)) >= 0) prv = S[IDX(pa_, pb_, pd_, sb, sd)];
                        dv = (f->side == 0 && l == 0) ? cur : (REAL)(cur - prv);
                    } else { /* forward E difference */
                        int na = ia, nb = ib, nd = id;
                        if (ax == 0) na += 1;
                        if (ax == 1) nb += 1;
                        if (ax == 2) nd += 1;
                        dv = (REAL)(S[IDX(na, nb, nd, sb, sd)] - S[IDX(ia, ib, id, sb, sd)]);
                    }
                    const int64_t s = IDX(a, b, d, pb, pd);
                    REAL ps = psi[s] * f->b[l];
                    ps = ps + f->c[l] * dv;
                    if (air) ps = ps * air[s];
                    psi[s] = ps;
                    const int64_t o = IDX(ia, ib, id, tb, td);
                    const REAL corr = beta[o] * (f->ck[l] * dv + ps);
                    T[o] = sgn[ax][q] > 0 ? (REAL)(T[o] + corr) : (REAL)(T[o] - corr);
                }
    }
}

static void lumped(fitc_problem *p, fitc_lumped *L) {
    double v_total = 0.0;
    for (int q = 0; q < L->n_edges; ++q) v_total += L->sign[q] * (double)p->e[L->idx[q]];
    const double v_src = p->n < L->n_src ? L->vsrc[p->n] : 0.0;
    const double i_port = (v_src - 0.0 - v_total) / (L->R + L->beta_sum);
    for (int q = 0; q < L->n_edges; ++q) {
        const int64_t o = L->idx[q];
        p->e[o] = (REAL)((double)p->e[o] + L->sign[q] * L->beta[q] * i_port);
    }
    L->i_prev = i_port;
    double v = 0.0;
    for (int q = 0; q < L->n_edges; ++q) v += L->sign[q] * (double)p->e[L->idx[q]];
    if (L->V) L->V[p->n] = v * L->rec_scale;
    if (L->I) L->I[p->n] = i_port * L->rec_scale;
}

static double dual_w(const double *d, int n, int q) {
    if (q == 0) return d[0];
    if (q >= n) return d[n - 1];
    return 0.5 * (d[q - 1] + d[q]);
}

static void monitor(fitc_problem *p, fitc_mon *m) {
    if (m->stride > 1 && (p->n % m->stride)) return;
    const double t = (double)p->n * p->dt, w = m->stride * p->dt;
    const int ni = m->i1 - m->i0, nj = m->j1 - m->j0, nk = m->k1 - m->k0;
    const int64_t cells = (int64_t)ni * nj * nk;
    double *val = malloc(sizeof(double) * (size_t)cells);
    double *cs = malloc(sizeof(double) * 2 * m->nf);
    for (int ci = 0; ci < m->ncomp; ++ci) {
        const int c = m->comps[ci];
        const REAL *A = comp_ptr(p, c);
        int sa, sb, sd;
        shape_of(p, c, &sa, &sb, &sd);
        const double tc = c < 3 ? t : t + 0.5 * p->dt;
        for (int f = 0; f < m->nf; ++f) {
            cs[2 * f] = cos(m->omega[f] * tc) * w;
            cs[2 * f + 1] = sin(m->omega[f] * tc) * w;
        }
        /* cell-centre samples first, then one contiguous pass per frequency
           (the per-bin arithmetic is the same in either loop order) */
#pragma omp parallel for schedule(static)
        for (int64_t cell = 0; cell < cells; ++cell) {
            const int kk = (int)(cell % nk), jj = (int)((cell / nk) % nj), ii = (int)(cell / ((int64_t)nk * nj));
            const int i = m->i0 + ii, j = m->j0 + jj, k = m->k0 + kk;
            double v;
#define AT(a, b, d) ((double)A[IDX(a, b, d, sb, sd)])
            switch (c) {
                case 0: v = (double)((REAL)0.25 * (REAL)(((A[IDX(i, j, k, sb, sd)] + A[IDX(i, j + 1, k, sb, sd)]) + A[IDX(i, j, k + 1, sb, sd)]) + A[IDX(i, j + 1, k + 1, sb, sd)])) / p->dx[i]; break;
                case 1: v = (double)((REAL)0.25 * (REAL)(((A[IDX(i, j, k, sb, sd)] + A[IDX(i + 1, j, k, sb, sd)]) + A[IDX(i, j, k + 1, sb, sd)]) + A[IDX(i + 1, j, k + 1, sb, sd)])) / p->dy[j]; break;
                case 2: v = (double)((REAL)0.25 * (REAL)(((A[IDX(i, j, k, sb, sd)] + A[IDX(i + 1, j, k, sb, sd)]) + A[IDX(i, j + 1, k, sb, sd)]) + A[IDX(i + 1, j + 1, k, sb, sd)])) / p->dz[k]; break;
                case 3: v = 0.5 * (AT(i, j, k) / dual_w(p->dx, p->nx, i) + AT(i + 1, j, k) / dual_w(p->dx, p->nx, i + 1)); break;
                case 4: v = 0.5 * (AT(i, j, k) / dual_w(p->dy, p->ny, j) + AT(i, j + 1, k) / dual_w(p->dy, p->ny, j + 1)); break;
                default: v = 0.5 * (AT(i, j, k) / dual_w(p->dz, p->nz, k) + AT(i, j, k + 1) / dual_w(p->dz, p->nz, k + 1)); break;
            }
#undef AT
            val[cell] = v;
        }
        double *re0 = m->re + (int64_t)ci * m->nf * cells, *im0 = m->im + (int64_t)ci * m->nf * cells;
#pragma omp parallel for schedule(static) collapse(2)
        for (int f = 0; f < m->nf; ++f)
            for (int64_t cell = 0; cell < cells; ++cell) {
                re0[(int64_t)f * cells + cell] += cs[2 * f] * val[cell];
                im0[(int64_t)f * cells + cell] += cs[2 * f + 1] * val[cell];
            }
    }
    free(cs);
    free(val);
}

void FN(fitc_step)(fitc_problem *p, int64_t n_steps) {
    for (int64_t s = 0; s < n_steps; ++s) {
        update_E(p);
        for (int q = 0; q < p->nfaces; ++q) cpml(p, &p->faces[q], 0);
        for (int q = 0; q < p->nlumped; ++q) lumped(p, &p->lumped[q]);
        update_H(p);
        for (int q = 0; q < p->nfaces; ++q) cpml(p, &p->faces[q], 1);
        for (int q = 0; q < p->nmon; ++q) monitor(p, &p->mon[q]);
        p->n += 1;
    }
}

int FN(fitc_sizeof_problem)(void) { return (int)sizeof(fitc_problem); }
