/*
 * rkdg_oracle.h -- plain-C CPU restatement of the reference RKDG algorithm.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests compare the
 * CUDA path against; it is never linked or loaded by the product library.
 *
 * It restates, per element and in FP64, what the reference computes with
 * its physical-space per-element basis (multi_gpuRkdg/):
 *   geometry, quadrature and Gram-Schmidt basis   src/triangleinfo.cpp:153-624
 *   traces, ghost states, volume/edge integrals     src/kernelfunctions.cu:84-637
 *   SSP-RK3 stages                                  src/kernelfunctions.cu:640-748
 *   CFL time step / residual monitor                src/kernelfunctions.cu:3-81, 751-867
 *   step order                                      src/rkdgadvance.cpp:97-217
 * and extends it with what the reference lacks: P1, the 3-/6-point volume
 * and 2-point edge rules, the HLLC flux, SSP-RK2 and a TVB-minmod limiter
 * on characteristic variables (methods named at each function).
 *
 * Layout: state and residual are [var][basis][tri] (var = rho, rhou, rhov,
 * rhoE), in the reference basis; residuals are NOT divided by the mass
 * (the reference's rhs_edge_*).
 */
#ifndef RKDG_ORACLE_H
#define RKDG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_LLF = 0, ORACLE_HLLC = 1 };
enum { ORACLE_LIMITER_NONE = 0, ORACLE_LIMITER_TVB = 1 };

typedef struct {
    int order;          /* 1 (P1, 3 basis functions) or 2 (P2, 6)            */
    int nq;             /* volume rule: 3 (degree 2), 6 (degree 4), 7 (deg 5) */
    int ng;             /* Gauss-Legendre points per edge: 2 or 3             */
    int flux;           /* ORACLE_LLF or ORACLE_HLLC                          */
    int limiter;        /* ORACLE_LIMITER_NONE or ORACLE_LIMITER_TVB          */
    int rk;             /* 2 (SSP-RK2) or 3 (SSP-RK3)                         */
    double tvb_m;       /* TVB constant M                                     */
    double gamma;
    double cfl;
    double farfield[4]; /* conservative far-field / inflow state              */
} oracle_params;

typedef struct oracle_case oracle_case;

/* xy: per-triangle vertex coordinates [T][3][2] (counter-clockwise);
 * nbr: [T][3] neighbour across edge k (opposite vertex k) or -1;
 * bc:  [T][3] boundary tag of edge k (1 far field, 2 outflow, 3 wall).
 * Returns NULL on invalid input. */
oracle_case* oracle_create(int ntri, const double* xy, const int* nbr, const int* bc,
                           const oracle_params* p);
void oracle_destroy(oracle_case* c);
int oracle_nbasis(const oracle_case* c);
void oracle_set_threads(int n);

/* Per-triangle reference-basis data: coeff [T][6][6] (coefficients of basis
 * i on 1, dx, dy, dx^2, dx*dy, dy^2 about the barycentre), mass [T][6],
 * area [T], perimeter [T], normal [T][3][2]. Any pointer may be NULL. */
void oracle_get_basis(const oracle_case* c, double* coeff, double* mass, double* area,
                      double* perimeter, double* normal);

void oracle_set_state(oracle_case* c, const double* U);
void oracle_get_state(const oracle_case* c, double* U);
void oracle_save_old(oracle_case* c);

/* R(U) of the current state, [4][Nb][T], not mass-divided. */
void oracle_residual(oracle_case* c, double* R);
/* CFL time step of the current state (src/kernelfunctions.cu:3-81). */
double oracle_time_step(const oracle_case* c);
/* Stage s (0-based) of the configured SSP-RK scheme against the state saved
 * by oracle_save_old, then the limiter if enabled. */
void oracle_stage(oracle_case* c, int s, double dt);
/* TVB limiter applied to the current state. Returns the number of limited cells. */
int oracle_limit(oracle_case* c);
/* One full step: dt (CFL time step when dt <= 0), save old, all stages,
 * residual monitor max|d rho_mean|, max|d rhoE_mean| into monitor[2]. */
double oracle_step(oracle_case* c, double dt, double* monitor);

/* Evaluates the solution at barycentric points (l1, l2) of each triangle
 * (x = v0 + l1 (v1 - v0) + l2 (v2 - v0)); out [4][npts][T]. */
void oracle_eval(const oracle_case* c, int npts, const double* l1, const double* l2, double* out);

#ifdef __cplusplus
}
#endif
#endif
