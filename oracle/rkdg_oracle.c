/*
 * rkdg_oracle.c -- plain-C CPU restatement of the reference RKDG algorithm
 * (see rkdg_oracle.h).  TEST INFRASTRUCTURE ONLY: used by tests/ and
 * bench.py's CPU leg as the checker, never by the product.
 *
 * Paths cited are relative to the reference's multi_gpuRkdg/ directory.
 */
#include "rkdg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXNB 6
#define MAXNQ 7
#define MAXNG 3

static int g_threads = 1;
void oracle_set_threads(int n) { g_threads = n > 0 ? n : 1; }

/* ---------------------------------------------------------------- rules -- */

/* Volume rules as barycentric (l0, l1, l2) and weights normalised to 1.
 * The 7-point degree-5 rule keeps the reference's decimal constants
 * (src/triangleinfo.cpp:159-163, 199-205, 219-225). */
static void volume_rule(int nq, double l[][3], double* w) {
    if (nq == 7) {
        const double w1 = 0.797426985353087, w2 = 0.101286507323456;
        const double w3 = 0.059715871789770, w4 = 0.470142064105115;
        const double L[7][3] = {{1.0 / 3, 1.0 / 3, 1.0 / 3}, {w1, w2, w2}, {w2, w1, w2},
                                {w2, w2, w1}, {w3, w4, w4}, {w4, w3, w4}, {w4, w4, w3}};
        const double W[7] = {0.225, 0.125939180544827, 0.125939180544827, 0.125939180544827,
                             0.132394152788506, 0.132394152788506, 0.132394152788506};
        memcpy(l, L, sizeof(L));
        memcpy(w, W, sizeof(W));
    } else if (nq == 6) {
        /* Dunavant (1985) degree-4 six-point rule */
        const double a = 0.44594849091596488631832925388305, wa = 0.22338158967801146569500700843312;
        const double b = 0.09157621350977074345957146340220, wb = 0.10995174365532186763832632490021;
        const double L[6][3] = {{1 - 2 * a, a, a}, {a, 1 - 2 * a, a}, {a, a, 1 - 2 * a},
                                {1 - 2 * b, b, b}, {b, 1 - 2 * b, b}, {b, b, 1 - 2 * b}};
        const double W[6] = {wa, wa, wa, wb, wb, wb};
        memcpy(l, L, sizeof(L));
        memcpy(w, W, sizeof(W));
    } else { /* nq == 3: Strang-Fix degree-2 interior rule */
        const double L[3][3] = {{2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6},
                                {1.0 / 6, 1.0 / 6, 2.0 / 3}};
        const double W[3] = {1.0 / 3, 1.0 / 3, 1.0 / 3};
        memcpy(l, L, sizeof(L));
        memcpy(w, W, sizeof(W));
    }
}

/* Gauss-Legendre points as fractions s along an edge from its start vertex,
 * weights normalised to 1.  The 3-point rule keeps the reference's constants
 * (src/triangleinfo.cpp:165, 209-217, 227-232). */
static void edge_rule(int ng, double* s, double* w) {
    if (ng == 3) {
        const double cp = 0.5 + sqrt(15.0) / 10.0;
        s[0] = 1 - cp;
        s[1] = 0.5;
        s[2] = cp;
        w[0] = 0.55555555555556 * 0.5;
        w[1] = 0.88888888888889 * 0.5;
        w[2] = 0.55555555555556 * 0.5;
    } else {
        s[0] = 0.5 - sqrt(3.0) / 6.0;
        s[1] = 0.5 + sqrt(3.0) / 6.0;
        w[0] = 0.5;
        w[1] = 0.5;
    }
}

/* 13-point degree-7 rule used for the basis Gram matrix
 * (src/triangleinfo.cpp:287-298): barycentric points and weights. */
static void gram_rule(double l[13][3], double w[13]) {
    const double A = 0.065130102902216, B = 0.869739794195568, C = 0.312865496004875;
    const double D = 0.638444188569809, E = 0.048690315425316, F = 0.260345966079038;
    const double G = 0.479308067841923;
    const double w1 = -0.149570044467670, w2 = 0.053347235608839, w3 = 0.175615257433204,
                 w4 = 0.077113760890257;
    const double L[13][3] = {{1.0 / 3, 1.0 / 3, 1.0 / 3}, {B, A, A}, {A, B, A}, {A, A, B},
                             {G, F, F}, {F, G, F}, {F, F, G}, {C, D, E}, {D, C, E},
                             {D, E, C}, {E, D, C}, {E, C, D}, {C, E, D}};
    const double W[13] = {w1, w2, w2, w2, w3, w3, w3, w4, w4, w4, w4, w4, w4};
    memcpy(l, L, sizeof(L));
    memcpy(w, W, sizeof(W));
}

/* ------------------------------------------------------------ case data -- */

struct oracle_case {
    int T, nb, nq, ng;
    oracle_params p;
    int* nbr;     /* [T][3] */
    int* bc;      /* [T][3] */
    int* shared;  /* [T][3] neighbour-local index of the shared edge */
    double* xy;   /* [T][3][2] */
    /* per-triangle geometry */
    double* area;
    double* perim;
    double* normal; /* [T][3][2] unit outward normals */
    double* len;    /* [T][3] */
    double* bary;   /* [T][2] */
    double* coeff;  /* [T][6][6] basis coefficients on 1,dx,dy,dx2,dxdy,dy2 */
    double* mass;   /* [T][6] */
    double* vphi;   /* [T][nq][nb] */
    double* vdx;    /* [T][nq][nb] */
    double* vdy;    /* [T][nq][nb] */
    double* vw;     /* [T][nq] physical weights */
    double* ephi;   /* [T][3][ng][nb] */
    double* ew;     /* [T][3][ng] physical weights */
    /* limiter geometry */
    double* lim_ab;   /* [T][3][2] alpha, beta */
    int* lim_j;       /* [T][3] second neighbour slot */
    double* lim_dir;  /* [T][3][2] unit direction barycentre -> midpoint */
    double* lim_h2;   /* [T][3] (2 |m - b|)^2 */
    double* lim_mphi; /* [T][3][2] phi_1, phi_2 at edge midpoints */
    /* state */
    double* U;  /* [4][nb][T] */
    double* U0; /* [4][nb][T] */
    double* R;  /* [4][nb][T] */
};

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

/* Partial-pivot Gaussian elimination of A (n x n, row-major) x = b, in place
 * on b.  Same method as the reference's Gauss() (src/gauss.cpp:3-107). */
static void solve_dense(int n, double* A, double* b) {
    for (int k = 0; k < n - 1; ++k) {
        int piv = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(A[i * n + k]) > fabs(A[piv * n + k])) piv = i;
        if (piv != k) {
            for (int j = 0; j < n; ++j) {
                double t = A[k * n + j];
                A[k * n + j] = A[piv * n + j];
                A[piv * n + j] = t;
            }
            double t = b[k];
            b[k] = b[piv];
            b[piv] = t;
        }
        for (int i = k + 1; i < n; ++i) {
            double m = A[i * n + k] / A[k * n + k];
            for (int j = k + 1; j < n; ++j) A[i * n + j] -= m * A[k * n + j];
            b[i] -= m * b[k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = 0;
        for (int j = i + 1; j < n; ++j) s += A[i * n + j] * b[j];
        b[i] = (b[i] - s) / A[i * n + i];
    }
}

static inline void monomials(double dx, double dy, double m[6]) {
    m[0] = 1;
    m[1] = dx;
    m[2] = dy;
    m[3] = dx * dx;
    m[4] = dx * dy;
    m[5] = dy * dy;
}

static inline double basis_val(const double* cf, double dx, double dy) {
    return cf[0] + cf[1] * dx + cf[2] * dy + cf[3] * dx * dx + cf[4] * dx * dy + cf[5] * dy * dy;
}
static inline double basis_ddx(const double* cf, double dx, double dy) {
    return cf[1] + 2 * cf[3] * dx + cf[4] * dy; /* src/triangleinfo.cpp:111-116 */
}
static inline double basis_ddy(const double* cf, double dx, double dy) {
    return cf[2] + cf[4] * dx + 2 * cf[5] * dy; /* src/triangleinfo.cpp:118-120 */
}

/* Per-element orthogonal basis of the reference: Gram-Schmidt of the scaled
 * monomials 1, X, Y, X^2, XY, Y^2 (X = (x-xc)/sqrt(A), Y = (y-yc)/sqrt(A)),
 * each basis function monic in its leading monomial and orthogonal to all
 * earlier ones under the area average, the moments taken with the 13-point
 * rule (src/triangleinfo.cpp:281-602).  Coefficients are returned on the
 * unscaled monomials 1, dx, dy, dx^2, dxdy, dy^2. */
static void reference_basis(const double x[3], const double y[3], double area, double xc,
                            double yc, double cf[6][6]) {
    double gl[13][3], gw[13];
    gram_rule(gl, gw);
    const double s = 1.0 / sqrt(area);
    double G[6][6] = {{0}};
    for (int q = 0; q < 13; ++q) {
        double px = gl[q][0] * x[0] + gl[q][1] * x[1] + gl[q][2] * x[2];
        double py = gl[q][0] * y[0] + gl[q][1] * y[1] + gl[q][2] * y[2];
        double m[6];
        monomials((px - xc) * s, (py - yc) * s, m);
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) G[i][j] += gw[q] * m[i] * m[j];
    }
    double c[6][6] = {{0}}; /* coefficients on scaled monomials */
    c[0][0] = 1;
    for (int k = 1; k < 6; ++k) {
        double A[36], b[6];
        for (int i = 0; i < k; ++i) {
            for (int j = 0; j < k; ++j) A[i * k + j] = G[i][j];
            b[i] = -G[i][k];
        }
        solve_dense(k, A, b);
        for (int j = 0; j < k; ++j) c[k][j] = b[j];
        c[k][k] = 1;
    }
    const double sc[6] = {1, s, s, s * s, s * s, s * s};
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) cf[i][j] = c[i][j] * sc[j];
}

oracle_case* oracle_create(int T, const double* xy, const int* nbr, const int* bc,
                           const oracle_params* p) {
    if (T <= 0 || !xy || !nbr || !bc || !p) return NULL;
    if (p->order != 1 && p->order != 2) return NULL;
    if (p->nq != 3 && p->nq != 6 && p->nq != 7) return NULL;
    if (p->ng != 2 && p->ng != 3) return NULL;
    if (p->rk != 2 && p->rk != 3) return NULL;
    oracle_case* c = (oracle_case*)calloc(1, sizeof(oracle_case));
    c->T = T;
    c->p = *p;
    c->nb = p->order == 1 ? 3 : 6;
    c->nq = p->nq;
    c->ng = p->ng;
    const int nb = c->nb, nq = c->nq, ng = c->ng;
    c->nbr = (int*)malloc(sizeof(int) * 3 * T);
    c->bc = (int*)malloc(sizeof(int) * 3 * T);
    c->shared = (int*)malloc(sizeof(int) * 3 * T);
    memcpy(c->nbr, nbr, sizeof(int) * 3 * T);
    memcpy(c->bc, bc, sizeof(int) * 3 * T);
    c->xy = dalloc(6 * (size_t)T);
    memcpy(c->xy, xy, sizeof(double) * 6 * T);
    c->area = dalloc(T);
    c->perim = dalloc(T);
    c->normal = dalloc(6 * (size_t)T);
    c->len = dalloc(3 * (size_t)T);
    c->bary = dalloc(2 * (size_t)T);
    c->coeff = dalloc(36 * (size_t)T);
    c->mass = dalloc(6 * (size_t)T);
    c->vphi = dalloc((size_t)T * nq * nb);
    c->vdx = dalloc((size_t)T * nq * nb);
    c->vdy = dalloc((size_t)T * nq * nb);
    c->vw = dalloc((size_t)T * nq);
    c->ephi = dalloc((size_t)T * 3 * ng * nb);
    c->ew = dalloc((size_t)T * 3 * ng);
    c->lim_ab = dalloc(6 * (size_t)T);
    c->lim_j = (int*)calloc(3 * (size_t)T, sizeof(int));
    c->lim_dir = dalloc(6 * (size_t)T);
    c->lim_h2 = dalloc(3 * (size_t)T);
    c->lim_mphi = dalloc(6 * (size_t)T);
    c->U = dalloc(4 * (size_t)nb * T);
    c->U0 = dalloc(4 * (size_t)nb * T);
    c->R = dalloc(4 * (size_t)nb * T);

    double vl[MAXNQ][3], vwn[MAXNQ], es[MAXNG], ewn[MAXNG];
    volume_rule(nq, vl, vwn);
    edge_rule(ng, es, ewn);
    double ml[7][3], mw[7];
    volume_rule(7, ml, mw); /* exact for P2 x P2: used for the mass */

    for (int e = 0; e < T; ++e) {
        const double* v = xy + 6 * e;
        double x[3] = {v[0], v[2], v[4]}, y[3] = {v[1], v[3], v[5]};
        /* area, edge lengths, perimeter, barycentre, normals:
         * src/triangleinfo.cpp:171-189 */
        double A = 0.5 * fabs((x[2] - x[0]) * (y[1] - y[0]) - (y[2] - y[0]) * (x[1] - x[0]));
        double l0 = sqrt((x[1] - x[2]) * (x[1] - x[2]) + (y[1] - y[2]) * (y[1] - y[2]));
        double l1 = sqrt((x[0] - x[2]) * (x[0] - x[2]) + (y[0] - y[2]) * (y[0] - y[2]));
        double l2 = sqrt((x[0] - x[1]) * (x[0] - x[1]) + (y[0] - y[1]) * (y[0] - y[1]));
        c->area[e] = A;
        c->len[3 * e] = l0;
        c->len[3 * e + 1] = l1;
        c->len[3 * e + 2] = l2;
        c->perim[e] = l0 + l1 + l2;
        double xc = (x[0] + x[1] + x[2]) / 3.0, yc = (y[0] + y[1] + y[2]) / 3.0;
        c->bary[2 * e] = xc;
        c->bary[2 * e + 1] = yc;
        double* n = c->normal + 6 * e;
        n[0] = (y[2] - y[1]) / l0;
        n[1] = (x[1] - x[2]) / l0;
        n[2] = (y[0] - y[2]) / l1;
        n[3] = (x[2] - x[0]) / l1;
        n[4] = (y[1] - y[0]) / l2;
        n[5] = (x[0] - x[1]) / l2;

        double cf[6][6];
        reference_basis(x, y, A, xc, yc, cf);
        memcpy(c->coeff + 36 * e, cf, sizeof(cf));

        for (int i = 0; i < 6; ++i) { /* mass, src/triangleinfo.cpp:605-624 */
            double m = 0;
            for (int q = 0; q < 7; ++q) {
                double px = ml[q][0] * x[0] + ml[q][1] * x[1] + ml[q][2] * x[2];
                double py = ml[q][0] * y[0] + ml[q][1] * y[1] + ml[q][2] * y[2];
                double f = basis_val(cf[i], px - xc, py - yc);
                m += A * mw[q] * f * f;
            }
            c->mass[6 * e + i] = m;
        }
        for (int q = 0; q < nq; ++q) {
            double px = vl[q][0] * x[0] + vl[q][1] * x[1] + vl[q][2] * x[2];
            double py = vl[q][0] * y[0] + vl[q][1] * y[1] + vl[q][2] * y[2];
            c->vw[(size_t)e * nq + q] = A * vwn[q];
            for (int i = 0; i < nb; ++i) {
                size_t o = ((size_t)e * nq + q) * nb + i;
                c->vphi[o] = basis_val(cf[i], px - xc, py - yc);
                c->vdx[o] = basis_ddx(cf[i], px - xc, py - yc);
                c->vdy[o] = basis_ddy(cf[i], px - xc, py - yc);
            }
        }
        const double lens[3] = {l0, l1, l2};
        for (int k = 0; k < 3; ++k) {
            int a = (k + 1) % 3, b = (k + 2) % 3; /* edge k runs v_a -> v_b */
            for (int g = 0; g < ng; ++g) {
                double px = (1 - es[g]) * x[a] + es[g] * x[b];
                double py = (1 - es[g]) * y[a] + es[g] * y[b];
                c->ew[((size_t)e * 3 + k) * ng + g] = ewn[g] * lens[k];
                for (int i = 0; i < nb; ++i)
                    c->ephi[(((size_t)e * 3 + k) * ng + g) * nb + i] =
                        basis_val(cf[i], px - xc, py - yc);
            }
        }
    }
    /* shared-edge index in the neighbour (src/unstructuredgrid.cpp:934-976) */
    for (int e = 0; e < T; ++e)
        for (int k = 0; k < 3; ++k) {
            int ne = c->nbr[3 * e + k];
            c->shared[3 * e + k] = -1;
            if (ne < 0) continue;
            for (int j = 0; j < 3; ++j)
                if (c->nbr[3 * ne + j] == e) {
                    c->shared[3 * e + k] = j;
                    break;
                }
            if (c->shared[3 * e + k] < 0) {
                oracle_destroy(c);
                return NULL;
            }
        }
    /* limiter geometry (Cockburn & Shu 1998, J. Comput. Phys. 141:199-224, sec. 2.4) */
    for (int e = 0; e < T; ++e) {
        const double* v = xy + 6 * e;
        double b0x = c->bary[2 * e], b0y = c->bary[2 * e + 1];
        double bx[3], by[3], mx[3], my[3];
        for (int k = 0; k < 3; ++k) {
            int a = (k + 1) % 3, b = (k + 2) % 3;
            mx[k] = 0.5 * (v[2 * a] + v[2 * b]);
            my[k] = 0.5 * (v[2 * a + 1] + v[2 * b + 1]);
            int ne = c->nbr[3 * e + k];
            if (ne >= 0) {
                /* neighbour barycentre placed next to this edge (periodic-safe) */
                int se = c->shared[3 * e + k];
                const double* w = xy + 6 * ne;
                int na = (se + 1) % 3, nbv = (se + 2) % 3;
                double nmx = 0.5 * (w[2 * na] + w[2 * nbv]), nmy = 0.5 * (w[2 * na + 1] + w[2 * nbv + 1]);
                bx[k] = mx[k] + (c->bary[2 * ne] - nmx);
                by[k] = my[k] + (c->bary[2 * ne + 1] - nmy);
            } else {
                const double* n = c->normal + 6 * e + 2 * k;
                double d = (mx[k] - b0x) * n[0] + (my[k] - b0y) * n[1];
                bx[k] = b0x + 2 * d * n[0];
                by[k] = b0y + 2 * d * n[1];
            }
        }
        for (int k = 0; k < 3; ++k) {
            double rx = mx[k] - b0x, ry = my[k] - b0y;
            double best = -1e300, ba = 0, bb = 0;
            int bj = (k + 1) % 3;
            for (int t = 1; t <= 2; ++t) {
                int j = (k + t) % 3;
                double ax = bx[k] - b0x, ay = by[k] - b0y, cx = bx[j] - b0x, cy = by[j] - b0y;
                double det = ax * cy - ay * cx;
                if (fabs(det) < 1e-300) continue;
                double al = (rx * cy - ry * cx) / det, be = (ax * ry - ay * rx) / det;
                double sc = al < be ? al : be;
                if (sc > best + 1e-14) {
                    best = sc;
                    ba = al;
                    bb = be;
                    bj = j;
                }
            }
            c->lim_ab[6 * e + 2 * k] = ba;
            c->lim_ab[6 * e + 2 * k + 1] = bb;
            c->lim_j[3 * e + k] = bj;
            double r = sqrt(rx * rx + ry * ry);
            c->lim_dir[6 * e + 2 * k] = rx / r;
            c->lim_dir[6 * e + 2 * k + 1] = ry / r;
            c->lim_h2[3 * e + k] = 4 * r * r;
            const double* cf = c->coeff + 36 * e;
            c->lim_mphi[6 * e + 2 * k] = basis_val(cf + 6, rx, ry);
            c->lim_mphi[6 * e + 2 * k + 1] = basis_val(cf + 12, rx, ry);
        }
    }
    return c;
}

void oracle_destroy(oracle_case* c) {
    if (!c) return;
    free(c->nbr), free(c->bc), free(c->shared), free(c->xy), free(c->area), free(c->perim);
    free(c->normal), free(c->len), free(c->bary), free(c->coeff), free(c->mass);
    free(c->vphi), free(c->vdx), free(c->vdy), free(c->vw), free(c->ephi), free(c->ew);
    free(c->lim_ab), free(c->lim_j), free(c->lim_dir), free(c->lim_h2), free(c->lim_mphi);
    free(c->U), free(c->U0), free(c->R);
    free(c);
}

int oracle_nbasis(const oracle_case* c) { return c->nb; }

void oracle_get_basis(const oracle_case* c, double* coeff, double* mass, double* area,
                      double* perimeter, double* normal) {
    const size_t T = c->T;
    if (coeff) memcpy(coeff, c->coeff, sizeof(double) * 36 * T);
    if (mass) memcpy(mass, c->mass, sizeof(double) * 6 * T);
    if (area) memcpy(area, c->area, sizeof(double) * T);
    if (perimeter) memcpy(perimeter, c->perim, sizeof(double) * T);
    if (normal) memcpy(normal, c->normal, sizeof(double) * 6 * T);
}

void oracle_set_state(oracle_case* c, const double* U) {
    memcpy(c->U, U, sizeof(double) * 4 * c->nb * (size_t)c->T);
}
void oracle_get_state(const oracle_case* c, double* U) {
    memcpy(U, c->U, sizeof(double) * 4 * c->nb * (size_t)c->T);
}
void oracle_save_old(oracle_case* c) {
    memcpy(c->U0, c->U, sizeof(double) * 4 * c->nb * (size_t)c->T);
}

/* ------------------------------------------------------------- physics -- */

static inline double pressure(const double u[4], double gamma) {
    double uu = u[1] / u[0], vv = u[2] / u[0];
    return (gamma - 1) * (u[3] - 0.5 * u[0] * (uu * uu + vv * vv));
}

/* Euler fluxes F and G (src/kernelfunctions.cu:310-341, 413-428). */
static inline void euler_fg(const double u[4], double gamma, double F[4], double G[4]) {
    double rho = u[0], uu = u[1] / rho, vv = u[2] / rho, E = u[3];
    double p = (gamma - 1) * (E - 0.5 * rho * (uu * uu + vv * vv));
    F[0] = rho * uu;
    F[1] = rho * uu * uu + p;
    F[2] = rho * uu * vv;
    F[3] = uu * (E + p);
    G[0] = rho * vv;
    G[1] = rho * vv * uu;
    G[2] = rho * vv * vv + p;
    G[3] = vv * (E + p);
}

/* Ghost state across a boundary edge (src/kernelfunctions.cu:184-268):
 * far field = given state, outflow = copy, wall = velocity mirrored about n. */
static inline void ghost_state(int tag, const double u[4], const double far[4], double nx,
                               double ny, double g[4]) {
    if (tag == 1) {
        g[0] = far[0], g[1] = far[1], g[2] = far[2], g[3] = far[3];
    } else if (tag == 2) {
        g[0] = u[0], g[1] = u[1], g[2] = u[2], g[3] = u[3];
    } else {
        g[0] = u[0];
        g[3] = u[3];
        g[1] = u[1] * (ny * ny - nx * nx) - 2.0 * nx * ny * u[2];
        g[2] = u[2] * (nx * nx - ny * ny) - 2.0 * nx * ny * u[1];
    }
}

/* HLLC flux through unit normal n (Toro, Riemann Solvers and Numerical
 * Methods for Fluid Dynamics, 3rd ed., sec. 10.4): Davis wave-speed bounds
 * S_L = min(q_L - c_L, q_R - c_R), S_R = max(q_L + c_L, q_R + c_R) (eq. 10.48),
 * contact speed S_M (eq. 10.37) and the star flux in its pressure form
 * F*_K = (S_M (S_K U_K - F_K) + S_K p* (0, n_x, n_y, S_M)) / (S_K - S_M)
 * with p* = p_K + rho_K (S_K - q_K)(S_M - q_K) (eqs. 10.36, 10.41-10.43,
 * as written by Toro in sec. 10.6). */
static void hllc_flux(const double uL[4], const double uR[4], double nx, double ny, double gamma,
                      double f[4]) {
    double rL = uL[0], rR = uR[0], iL = 1.0 / rL, iR = 1.0 / rR;
    double vxL = uL[1] * iL, vyL = uL[2] * iL, vxR = uR[1] * iR, vyR = uR[2] * iR;
    double pL = (gamma - 1) * (uL[3] - 0.5 * (uL[1] * vxL + uL[2] * vyL));
    double pR = (gamma - 1) * (uR[3] - 0.5 * (uR[1] * vxR + uR[2] * vyR));
    double qL = vxL * nx + vyL * ny, qR = vxR * nx + vyR * ny;
    double cL = sqrt(gamma * pL * iL), cR = sqrt(gamma * pR * iR);
    double SL = fmin(qL - cL, qR - cR), SR = fmax(qL + cL, qR + cR);
    double FL[4] = {rL * qL, uL[1] * qL + pL * nx, uL[2] * qL + pL * ny, (uL[3] + pL) * qL};
    double FR[4] = {rR * qR, uR[1] * qR + pR * nx, uR[2] * qR + pR * ny, (uR[3] + pR) * qR};
    if (SL >= 0) {
        memcpy(f, FL, sizeof(FL));
        return;
    }
    if (SR <= 0) {
        memcpy(f, FR, sizeof(FR));
        return;
    }
    double dL = rL * (SL - qL), dR = rR * (SR - qR);
    double SM = (pR - pL + dL * qL - dR * qR) / (dL - dR);
    const int left = SM >= 0;
    const double* u = left ? uL : uR;
    const double* F = left ? FL : FR;
    double d = left ? dL : dR, p = left ? pL : pR, q = left ? qL : qR, S = left ? SL : SR;
    double ps = p + d * (SM - q);
    double k = 1.0 / (S - SM);
    f[0] = SM * (S * u[0] - F[0]) * k;
    f[1] = (SM * (S * u[1] - F[1]) + S * ps * nx) * k;
    f[2] = (SM * (S * u[2] - F[2]) + S * ps * ny) * k;
    f[3] = (SM * (S * u[3] - F[3]) + S * ps * SM) * k;
}

/* R(U) of one element (reference basis, not mass-divided): the chain
 * ConVars -> BC -> VolumeRHS -> LFCoeff -> EdgeFG -> Flux -> EdgeRHS of
 * src/kernelfunctions.cu:84-637 for one triangle. */
static void element_residual(const oracle_case* c, int e, double R[4][MAXNB]) {
    const int T = c->T, nb = c->nb, nq = c->nq, ng = c->ng;
    const double gamma = c->p.gamma;
    const double* U = c->U;
#define UCOEF(v, i, t) U[((size_t)(v) * nb + (i)) * T + (t)]
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < nb; ++i) R[v][i] = 0;
    /* volume integral */
    for (int q = 0; q < nq; ++q) {
        const size_t o = ((size_t)e * nq + q) * nb;
        double u[4] = {0, 0, 0, 0};
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < nb; ++i) u[v] += c->vphi[o + i] * UCOEF(v, i, e);
        double F[4], G[4];
        euler_fg(u, gamma, F, G);
        double w = c->vw[(size_t)e * nq + q];
        for (int i = 0; i < nb; ++i) {
            double dx = c->vdx[o + i], dy = c->vdy[o + i];
            for (int v = 0; v < 4; ++v) R[v][i] += w * F[v] * dx + w * G[v] * dy;
        }
    }
    /* edge integrals */
    for (int k = 0; k < 3; ++k) {
        const int ne = c->nbr[3 * e + k];
        const double nx = c->normal[6 * e + 2 * k], ny = c->normal[6 * e + 2 * k + 1];
        double mL[4], mR[4];
        for (int v = 0; v < 4; ++v) mL[v] = UCOEF(v, 0, e);
        if (ne >= 0) {
            for (int v = 0; v < 4; ++v) mR[v] = UCOEF(v, 0, ne);
        } else {
            ghost_state(c->bc[3 * e + k], mL, c->p.farfield, nx, ny, mR);
        }
        /* LLF coefficient from the mean of the two cell averages
         * (src/kernelfunctions.cu:370-387) */
        double alpha;
        {
            double rho = 0.5 * (mL[0] + mR[0]);
            double uu = 0.5 * (mL[1] + mR[1]) / rho;
            double vv = 0.5 * (mL[2] + mR[2]) / rho;
            double E = 0.5 * (mL[3] + mR[3]);
            double p = (gamma - 1) * (E - 0.5 * rho * (uu * uu + vv * vv));
            alpha = fabs(uu * nx + vv * ny) + sqrt(gamma * p / rho);
        }
        for (int g = 0; g < ng; ++g) {
            const size_t oL = (((size_t)e * 3 + k) * ng + g) * nb;
            double uL[4] = {0, 0, 0, 0}, uR[4] = {0, 0, 0, 0};
            for (int v = 0; v < 4; ++v)
                for (int i = 0; i < nb; ++i) uL[v] += c->ephi[oL + i] * UCOEF(v, i, e);
            if (ne >= 0) {
                /* neighbour point ng-1-g on its shared edge (src/kernelfunctions.cu:545-549) */
                const int se = c->shared[3 * e + k];
                const size_t oR = (((size_t)ne * 3 + se) * ng + (ng - 1 - g)) * nb;
                for (int v = 0; v < 4; ++v)
                    for (int i = 0; i < nb; ++i) uR[v] += c->ephi[oR + i] * UCOEF(v, i, ne);
            } else {
                ghost_state(c->bc[3 * e + k], uL, c->p.farfield, nx, ny, uR);
            }
            double fh[4];
            if (c->p.flux == ORACLE_HLLC) {
                hllc_flux(uL, uR, nx, ny, gamma, fh);
            } else {
                double FL[4], GL[4], FR[4], GR[4];
                euler_fg(uL, gamma, FL, GL);
                euler_fg(uR, gamma, FR, GR);
                for (int v = 0; v < 4; ++v)
                    fh[v] = 0.5 * ((FL[v] + FR[v]) * nx + (GL[v] + GR[v]) * ny -
                                   alpha * (uR[v] - uL[v]));
            }
            const double w = c->ew[((size_t)e * 3 + k) * ng + g];
            for (int i = 0; i < nb; ++i) {
                double phi = c->ephi[oL + i];
                for (int v = 0; v < 4; ++v) R[v][i] -= w * fh[v] * phi;
            }
        }
    }
#undef UCOEF
}

void oracle_residual(oracle_case* c, double* Rout) {
    const int T = c->T, nb = c->nb;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (int e = 0; e < T; ++e) {
        double R[4][MAXNB];
        element_residual(c, e, R);
        for (int v = 0; v < 4; ++v)
            for (int i = 0; i < nb; ++i) c->R[((size_t)v * nb + i) * T + e] = R[v][i];
    }
    if (Rout) memcpy(Rout, c->R, sizeof(double) * 4 * nb * (size_t)T);
}

/* dt = cfl / max_e (|u| + c) * perimeter / area over cell means
 * (src/kernelfunctions.cu:17-31, 79). */
double oracle_time_step(const oracle_case* c) {
    const int T = c->T, nb = c->nb;
    const double gamma = c->p.gamma;
    double mx = 0;
    for (int e = 0; e < T; ++e) {
        double rho = c->U[e], u = c->U[(size_t)nb * T + e] / rho, v = c->U[2 * (size_t)nb * T + e] / rho;
        double E = c->U[3 * (size_t)nb * T + e];
        double p = (gamma - 1) * (E - 0.5 * rho * (u * u + v * v));
        double a = sqrt(gamma * p / rho);
        double dx = (sqrt(u * u + v * v) + a) * c->perim[e] / c->area[e];
        if (dx > mx) mx = dx;
    }
    return c->p.cfl / mx;
}

/* ------------------------------------------------------------- limiter -- */

static inline double minmod2(double a, double b) {
    if (a > 0 && b > 0) return a < b ? a : b;
    if (a < 0 && b < 0) return a > b ? a : b;
    return 0;
}

/* Eigenvectors of the x-split Euler Jacobian rotated to direction n, at the
 * state u: right vectors as columns of Rm, left vectors as rows of Lm. */
static void char_basis(const double u[4], double nx, double ny, double gamma, double Rm[4][4],
                       double Lm[4][4]) {
    double rho = u[0], vx = u[1] / rho, vy = u[2] / rho;
    double p = (gamma - 1) * (u[3] - 0.5 * rho * (vx * vx + vy * vy));
    double c = sqrt(gamma * p / rho), H = (u[3] + p) / rho;
    double q = vx * nx + vy * ny, qt = -vx * ny + vy * nx, k2 = 0.5 * (vx * vx + vy * vy);
    double b1 = (gamma - 1) / (c * c), b2 = b1 * k2;
    const double r[4][4] = {{1, vx - c * nx, vy - c * ny, H - q * c},
                            {1, vx, vy, k2},
                            {0, -ny, nx, qt},
                            {1, vx + c * nx, vy + c * ny, H + q * c}};
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Rm[j][i] = r[i][j];
    const double l[4][4] = {
        {0.5 * (b2 + q / c), 0.5 * (-b1 * vx - nx / c), 0.5 * (-b1 * vy - ny / c), 0.5 * b1},
        {1 - b2, b1 * vx, b1 * vy, -b1},
        {-qt, -ny, nx, 0},
        {0.5 * (b2 - q / c), 0.5 * (-b1 * vx + nx / c), 0.5 * (-b1 * vy + ny / c), 0.5 * b1}};
    memcpy(Lm, l, sizeof(l));
}

/* TVB-minmod limiter on characteristic variables for the P1 part
 * (Cockburn & Shu 1998, J. Comput. Phys. 141:199-224, sec. 2.4 and 3.3):
 * per edge midpoint m_i, compare u_h(m_i) - ubar with nu*(alpha (u_i - ubar)
 * + beta (u_j - ubar)), nu = 1.5, in the characteristic fields of direction
 * m_i - b at ubar; a cell is limited when any minmod does not return its
 * first argument; its midpoint increments are then made to sum to zero by
 * the positive/negative scaling of the paper and its quadratic modes are
 * dropped. TVB threshold: |a| <= M (2 |m_i - b|)^2 keeps a. */
int oracle_limit(oracle_case* c) {
    const int T = c->T, nb = c->nb;
    const double gamma = c->p.gamma, M = c->p.tvb_m, nu = 1.5;
    double* U = c->U;
    double* Unew = dalloc(4 * (size_t)nb * T);
    memcpy(Unew, U, sizeof(double) * 4 * nb * (size_t)T);
    int nlim = 0;
#define UC(v, i, t) U[((size_t)(v) * nb + (i)) * T + (t)]
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1) reduction(+ : nlim)
    for (int e = 0; e < T; ++e) {
        double mean[4], nbm[3][4], tilde[3][4];
        for (int v = 0; v < 4; ++v) mean[v] = UC(v, 0, e);
        for (int k = 0; k < 3; ++k) {
            int ne = c->nbr[3 * e + k];
            const double* n = c->normal + 6 * e + 2 * k;
            if (ne >= 0)
                for (int v = 0; v < 4; ++v) nbm[k][v] = UC(v, 0, ne);
            else
                ghost_state(c->bc[3 * e + k], mean, c->p.farfield, n[0], n[1], nbm[k]);
            double p1 = c->lim_mphi[6 * e + 2 * k], p2 = c->lim_mphi[6 * e + 2 * k + 1];
            for (int v = 0; v < 4; ++v) tilde[k][v] = p1 * UC(v, 1, e) + p2 * UC(v, 2, e);
        }
        int limited = 0;
        double delta[3][4];
        for (int k = 0; k < 3; ++k) {
            int j = c->lim_j[3 * e + k];
            double al = c->lim_ab[6 * e + 2 * k], be = c->lim_ab[6 * e + 2 * k + 1];
            double dbar[4];
            for (int v = 0; v < 4; ++v)
                dbar[v] = al * (nbm[k][v] - mean[v]) + be * (nbm[j][v] - mean[v]);
            double Rm[4][4], Lm[4][4];
            char_basis(mean, c->lim_dir[6 * e + 2 * k], c->lim_dir[6 * e + 2 * k + 1], gamma, Rm, Lm);
            double wt[4], wd[4], wl[4];
            for (int a = 0; a < 4; ++a) {
                wt[a] = Lm[a][0] * tilde[k][0] + Lm[a][1] * tilde[k][1] + Lm[a][2] * tilde[k][2] +
                        Lm[a][3] * tilde[k][3];
                wd[a] = Lm[a][0] * dbar[0] + Lm[a][1] * dbar[1] + Lm[a][2] * dbar[2] +
                        Lm[a][3] * dbar[3];
            }
            const double thr = M * c->lim_h2[3 * e + k];
            for (int a = 0; a < 4; ++a) {
                if (fabs(wt[a]) <= thr) {
                    wl[a] = wt[a];
                } else {
                    wl[a] = minmod2(wt[a], nu * wd[a]);
                    if (wl[a] != wt[a]) limited = 1;
                }
            }
            for (int v = 0; v < 4; ++v)
                delta[k][v] = Rm[v][0] * wl[0] + Rm[v][1] * wl[1] + Rm[v][2] * wl[2] +
                              Rm[v][3] * wl[3];
        }
        if (!limited) continue;
        ++nlim;
        for (int v = 0; v < 4; ++v) {
            double s = delta[0][v] + delta[1][v] + delta[2][v];
            if (s != 0) {
                double pos = 0, neg = 0;
                for (int k = 0; k < 3; ++k) {
                    pos += fmax(0.0, delta[k][v]);
                    neg += fmax(0.0, -delta[k][v]);
                }
                double tp = pos > 0 ? fmin(1.0, neg / pos) : 1.0;
                double tn = neg > 0 ? fmin(1.0, pos / neg) : 1.0;
                for (int k = 0; k < 3; ++k)
                    delta[k][v] = tp * fmax(0.0, delta[k][v]) - tn * fmax(0.0, -delta[k][v]);
            }
        }
        /* P1 coefficients with the limited midpoint increments: least squares
         * of the (consistent) 3 x 2 system P c = delta */
        double a11 = 0, a12 = 0, a22 = 0;
        for (int k = 0; k < 3; ++k) {
            double p1 = c->lim_mphi[6 * e + 2 * k], p2 = c->lim_mphi[6 * e + 2 * k + 1];
            a11 += p1 * p1;
            a12 += p1 * p2;
            a22 += p2 * p2;
        }
        double det = a11 * a22 - a12 * a12;
        for (int v = 0; v < 4; ++v) {
            double r1 = 0, r2 = 0;
            for (int k = 0; k < 3; ++k) {
                r1 += c->lim_mphi[6 * e + 2 * k] * delta[k][v];
                r2 += c->lim_mphi[6 * e + 2 * k + 1] * delta[k][v];
            }
            Unew[((size_t)v * nb + 1) * T + e] = (a22 * r1 - a12 * r2) / det;
            Unew[((size_t)v * nb + 2) * T + e] = (a11 * r2 - a12 * r1) / det;
            for (int i = 3; i < nb; ++i) Unew[((size_t)v * nb + i) * T + e] = 0;
        }
    }
#undef UC
    memcpy(U, Unew, sizeof(double) * 4 * nb * (size_t)T);
    free(Unew);
    return nlim;
}

/* ---------------------------------------------------------------- steps -- */

/* SSP-RK stage s: U <- a U0 + b U + b dt M^-1 R(U) (src/kernelfunctions.cu:640-748;
 * SSP-RK2 of Shu & Osher 1988 for rk = 2). */
void oracle_stage(oracle_case* c, int s, double dt) {
    const int T = c->T, nb = c->nb;
    double a, b;
    if (s == 0) {
        a = 0, b = 1;
    } else if (c->p.rk == 2) {
        a = 0.5, b = 0.5;
    } else if (s == 1) {
        a = 0.75, b = 0.25;
    } else {
        a = 1.0 / 3.0, b = 2.0 / 3.0;
    }
    oracle_residual(c, NULL);
    for (int v = 0; v < 4; ++v)
        for (int i = 0; i < nb; ++i)
            for (int e = 0; e < T; ++e) {
                size_t o = ((size_t)v * nb + i) * T + e;
                double m = c->mass[6 * e + i];
                if (s == 0)
                    c->U[o] += dt * (c->R[o]) / m;
                else
                    c->U[o] = a * c->U0[o] + b * c->U[o] + b * dt * (c->R[o]) / m;
            }
    if (c->p.limiter == ORACLE_LIMITER_TVB) oracle_limit(c);
}

double oracle_step(oracle_case* c, double dt, double* monitor) {
    if (dt <= 0) dt = oracle_time_step(c);
    oracle_save_old(c);
    for (int s = 0; s < c->p.rk; ++s) oracle_stage(c, s, dt);
    if (monitor) { /* src/kernelfunctions.cu:751-780 */
        const int T = c->T, nb = c->nb;
        double m0 = 0, m1 = 0;
        for (int e = 0; e < T; ++e) {
            double d0 = fabs(c->U[e] - c->U0[e]);
            double d1 = fabs(c->U[3 * (size_t)nb * T + e] - c->U0[3 * (size_t)nb * T + e]);
            if (d0 > m0) m0 = d0;
            if (d1 > m1) m1 = d1;
        }
        monitor[0] = m0;
        monitor[1] = m1;
    }
    return dt;
}

void oracle_eval(const oracle_case* c, int npts, const double* l1, const double* l2, double* out) {
    const int T = c->T, nb = c->nb;
    for (int e = 0; e < T; ++e) {
        const double* v = c->xy + 6 * e;
        const double* cf = c->coeff + 36 * e;
        double xc = c->bary[2 * e], yc = c->bary[2 * e + 1];
        for (int q = 0; q < npts; ++q) {
            double px = v[0] + l1[q] * (v[2] - v[0]) + l2[q] * (v[4] - v[0]);
            double py = v[1] + l1[q] * (v[3] - v[1]) + l2[q] * (v[5] - v[1]);
            for (int w = 0; w < 4; ++w) {
                double s = 0;
                for (int i = 0; i < nb; ++i)
                    s += basis_val(cf + 6 * i, px - xc, py - yc) * c->U[((size_t)w * nb + i) * T + e];
                out[((size_t)w * npts + q) * T + e] = s;
            }
        }
    }
}
