// sm_100a kernels of the RKDG residual and time-step path.
//
// One fused kernel per Runge-Kutta stage replaces the reference's chain of
// nine launches per stage (src/kernelfunctions.cu:84-748): the tile-staged
// stage kernel (stage_tiled.cuh) evaluates each element's state at the
// volume points, projects the contravariant Euler fluxes onto the basis
// gradients, forms the edge traces and the Riemann flux at the Gauss points
// of every edge once per tile, and applies the SSP-RK stage update in its
// epilogue.  Nothing but the state is written to HBM: traces, fluxes and
// residuals live in registers and shared memory.  This file also holds the
// physics helpers, the TVB limiter, the CFL/step kernels and the boundary
// conversions.
//
// HBM layout (element-interleaved packs for 128-bit accesses):
//   state  : row r = 4*i + v (basis i, variable v), packs of W = 16/sizeof(Real)
//            rows; pack p of element e at ((p*ld + e) * W)  -> one 16-byte
//            load per pack, a warp reads 512 contiguous bytes; RKDG_FP32C
//            adds one pack row holding the low parts of the cell means;
//   jinv   : FP64 rows of J^-1, [2][ld] double2 = (r0x, r0y), (r1x, r1y);
//   conn   : [ld] int4 = (neighbour 0, 1, 2, packed shared-edge/boundary tags).
// The basis is orthonormal under the area average on the reference
// triangle, so M = area * I and every geometric factor of the stage comes
// from J^-1: the scaled normals N_k/area are 2(r0+r1), -2 r0, -2 r1.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <type_traits>

#include "rkdg_internal.hpp"

namespace rkdg {

// -------------------------------------------------------------- tables --
template <typename Real>
struct Tab {
    Real vphi[kMaxNQ][kMaxNB];
    Real vdxi[kMaxNQ][kMaxNB];  // weight * d psi / d xi
    Real veta[kMaxNQ][kMaxNB];  // weight * d psi / d eta
    Real ephi[3][kMaxNG][kMaxNB];
    Real ephiw[3][kMaxNG][kMaxNB];  // 2 w_g psi_i at point g of edge k (surface projection)
    Real ew[kMaxNG];
    Real mphi[3][2];
    Real minv[2][3];
};

// rule configurations: index = 2 * (nq == 7 ? 0 : nq == 6 ? 1 : 2) + (ng == 3 ? 0 : 1)
constexpr int kNumCfg = 6;
__constant__ Tab<double> c_tab_d[kNumCfg];
__constant__ Tab<float> c_tab_f[kNumCfg];

// FP32 tables with every value in both lanes of a pair, for the packed
// two-lane FP32 arithmetic (f32x2) of the tile kernel; nephiw = -(2 w_g psi_i).
struct Tab2 {
    float2 vphi[kMaxNQ][kMaxNB];
    float2 vdxi[kMaxNQ][kMaxNB];
    float2 veta[kMaxNQ][kMaxNB];
    float2 ephi[3][kMaxNG][kMaxNB];
    float2 nephiw[3][kMaxNG][kMaxNB];
};
__constant__ Tab2 c_tab_f2[kNumCfg];

// Two-lane FP32 arithmetic (PTX fma/mul/add/sub .f32x2, sm_100a): each lane is
// one IEEE single-precision operation (a fused multiply-add rounds once).
// The pairing fixes the order of operations; a scalar build may contract a
// sum of products differently and so differ in the last bit.
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n .reg .b64 a, b, c, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n mov.b64 c, {%6, %7};\n"
        " fma.rn.f32x2 d, a, b, c;\n mov.b64 {%0, %1}, d;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) {
    float2 r;
    asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
        " mul.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b) {
    float2 r;
    asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
        " add.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
    float2 r;
    asm("{\n .reg .b64 a, b, d;\n mov.b64 a, {%2, %3};\n mov.b64 b, {%4, %5};\n"
        " sub.rn.f32x2 d, a, b;\n mov.b64 {%0, %1}, d;\n}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}

__host__ __device__ constexpr int cfg_index(int nq, int ng) {
    return 2 * (nq == 7 ? 0 : (nq == 6 ? 1 : 2)) + (ng == 3 ? 0 : 1);
}

template <typename Real>
__device__ __forceinline__ const Tab<Real>& tab(int c);
template <>
__device__ __forceinline__ const Tab<double>& tab<double>(int c) { return c_tab_d[c]; }
template <>
__device__ __forceinline__ const Tab<float>& tab<float>(int c) { return c_tab_f[c]; }

void upload_tables(int nq, int ng) {
    RuleTables t = make_tables(nq, ng);
    // the tile kernel forms the psi_0 term once (psi_0 is the same constant
    // at every volume and edge point) and skips the eta-derivative of psi_1
    // (a function of xi alone): both hold exactly for the native basis
    for (int q = 0; q < nq; ++q)
        if (t.vphi[q][0] != t.vphi[0][0] || t.veta_w[q][1] != 0.0)
            throw Error{RKDG_ERR_INVALID, "basis tables: psi_0 not constant or psi_1 not a function of xi"};
    for (int k = 0; k < 3; ++k)
        for (int g = 0; g < ng; ++g)
            if (t.ephi[k][g][0] != t.vphi[0][0])
                throw Error{RKDG_ERR_INVALID, "basis tables: psi_0 not constant on the edges"};
    Tab<double> d{};
    Tab<float> f{};
    for (int q = 0; q < kMaxNQ; ++q)
        for (int i = 0; i < kMaxNB; ++i) {
            d.vphi[q][i] = t.vphi[q][i];
            d.vdxi[q][i] = t.vdxi_w[q][i];
            d.veta[q][i] = t.veta_w[q][i];
            f.vphi[q][i] = (float)t.vphi[q][i];
            f.vdxi[q][i] = (float)t.vdxi_w[q][i];
            f.veta[q][i] = (float)t.veta_w[q][i];
        }
    for (int k = 0; k < 3; ++k)
        for (int g = 0; g < kMaxNG; ++g)
            for (int i = 0; i < kMaxNB; ++i) {
                d.ephi[k][g][i] = t.ephi[k][g][i];
                f.ephi[k][g][i] = (float)t.ephi[k][g][i];
                d.ephiw[k][g][i] = 2.0 * t.ew[g] * t.ephi[k][g][i];
                f.ephiw[k][g][i] = (float)(2.0 * t.ew[g] * t.ephi[k][g][i]);
            }
    for (int g = 0; g < kMaxNG; ++g) {
        d.ew[g] = t.ew[g];
        f.ew[g] = (float)t.ew[g];
    }
    for (int k = 0; k < 3; ++k)
        for (int j = 0; j < 2; ++j) {
            d.mphi[k][j] = t.mphi[k][j];
            f.mphi[k][j] = (float)t.mphi[k][j];
            d.minv[j][k] = t.minv[j][k];
            f.minv[j][k] = (float)t.minv[j][k];
        }
    Tab2 f2{};
    auto dup = [](double x) { return make_float2((float)x, (float)x); };
    for (int q = 0; q < kMaxNQ; ++q)
        for (int i = 0; i < kMaxNB; ++i) {
            f2.vphi[q][i] = dup(t.vphi[q][i]);
            f2.vdxi[q][i] = dup(t.vdxi_w[q][i]);
            f2.veta[q][i] = dup(t.veta_w[q][i]);
        }
    for (int k = 0; k < 3; ++k)
        for (int g = 0; g < kMaxNG; ++g)
            for (int i = 0; i < kMaxNB; ++i) {
                f2.ephi[k][g][i] = dup(t.ephi[k][g][i]);
                f2.nephiw[k][g][i] = make_float2(-f.ephiw[k][g][i], -f.ephiw[k][g][i]);
            }
    const int c = cfg_index(nq, ng);
    RKDG_CUDA_TRY(cudaMemcpyToSymbol(c_tab_d, &d, sizeof(d), sizeof(d) * c));
    RKDG_CUDA_TRY(cudaMemcpyToSymbol(c_tab_f, &f, sizeof(f), sizeof(f) * c));
    RKDG_CUDA_TRY(cudaMemcpyToSymbol(c_tab_f2, &f2, sizeof(f2), sizeof(f2) * c));
}

// --------------------------------------------------------- state packs --
template <typename Real, int NB>
__device__ __forceinline__ void load_state(const Real* __restrict__ U, int ld, int e,
                                           Real u[NB][4]) {
    if constexpr (sizeof(Real) == 8) {
        const double2* p = reinterpret_cast<const double2*>(U);
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            double2 a = __ldg(p + (size_t)(2 * i) * ld + e);
            double2 b = __ldg(p + (size_t)(2 * i + 1) * ld + e);
            u[i][0] = a.x;
            u[i][1] = a.y;
            u[i][2] = b.x;
            u[i][3] = b.y;
        }
    } else {
        const float4* p = reinterpret_cast<const float4*>(U);
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            float4 a = __ldg(p + (size_t)i * ld + e);
            u[i][0] = a.x;
            u[i][1] = a.y;
            u[i][2] = a.z;
            u[i][3] = a.w;
        }
    }
}

template <typename Real, int NB>
__device__ __forceinline__ void load_mean(const Real* __restrict__ U, int ld, int e, Real m[4]) {
    Real u[1][4];
    load_state<Real, 1>(U, ld, e, u);
    m[0] = u[0][0], m[1] = u[0][1], m[2] = u[0][2], m[3] = u[0][3];
}

// FP32 states store every cell mean as its deviation from the solve's
// reference (far-field) state, so that rounding scales with the flow's
// deviation instead of with the state (the SSP-RK combination coefficients
// sum to one, so stage updates apply to deviations unchanged); FP64 states
// store the mean itself.  ref_of returns the offset to add to a stored mean.
template <typename Real>
__device__ __forceinline__ Real ref_of(const double* ref, int v) {
    if constexpr (sizeof(Real) == 4) return (Real)ref[v];
    else return Real(0);
}
template <typename Real>
__host__ __device__ constexpr bool stores_deviation() { return sizeof(Real) == 4; }

struct Ref4 {
    double v[4];
};

template <typename Real, int NB>
__device__ __forceinline__ void store_state(Real* __restrict__ U, int ld, int e,
                                            const Real u[NB][4]) {
    if constexpr (sizeof(Real) == 8) {
        double2* p = reinterpret_cast<double2*>(U);
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            p[(size_t)(2 * i) * ld + e] = make_double2(u[i][0], u[i][1]);
            p[(size_t)(2 * i + 1) * ld + e] = make_double2(u[i][2], u[i][3]);
        }
    } else {
        float4* p = reinterpret_cast<float4*>(U);
#pragma unroll
        for (int i = 0; i < NB; ++i) p[(size_t)i * ld + e] = make_float4(u[i][0], u[i][1], u[i][2], u[i][3]);
    }
}

// rows I0..NB-1 of a state (the FP32 form's one 16-byte pack per basis function)
template <typename Real, int I0, int NB>
__device__ __forceinline__ void store_rows(Real* __restrict__ U, int ld, int e, const Real u[NB][4]) {
    static_assert(sizeof(Real) == 4, "one pack per row: FP32 states");
    float4* p = reinterpret_cast<float4*>(U);
#pragma unroll
    for (int i = I0; i < NB; ++i) p[(size_t)i * ld + e] = make_float4(u[i][0], u[i][1], u[i][2], u[i][3]);
}

// ------------------------------------------------------------- physics --
// Ghost state of a boundary edge (the reference's boundaryCondition kernel,
// src/kernelfunctions.cu:184-268, applied inline): 1 far field, 2 outflow
// copy, 3 slip wall mirroring the momentum about the unit normal.
template <typename Real>
__device__ __forceinline__ void ghost(int tag, const Real u[4], const Real far[4], Real nx, Real ny,
                                      Real g[4]) {
    if (tag == RKDG_BC_FARFIELD) {
        g[0] = far[0], g[1] = far[1], g[2] = far[2], g[3] = far[3];
    } else if (tag == RKDG_BC_OUTFLOW) {
        g[0] = u[0], g[1] = u[1], g[2] = u[2], g[3] = u[3];
    } else {
        g[0] = u[0];
        g[3] = u[3];
        g[1] = u[1] * (ny * ny - nx * nx) - Real(2) * nx * ny * u[2];
        g[2] = u[2] * (nx * nx - ny * ny) - Real(2) * nx * ny * u[1];
    }
}

// Reciprocal, quotient and square root: IEEE in FP64 (the parity path);
// in FP32 the PTX approximations (rcp.approx, rsqrt.approx: about 1 ulp),
// which the FP32 precision form's tolerance absorbs, with subnormal inputs
// and results flushed to zero (.ftz: one instruction each, no subnormal
// range handling; the arguments are densities, pressures, edge lengths and
// wave-speed differences, all far above the subnormal range).
__device__ __forceinline__ float rcp_ftz(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_ftz(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ double rcp_(double x) { return 1.0 / x; }
__device__ __forceinline__ float rcp_(float x) { return rcp_ftz(x); }
__device__ __forceinline__ double div_(double a, double b) { return a / b; }
__device__ __forceinline__ float div_(float a, float b) { return a * rcp_ftz(b); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_(float x) { return x * rsqrt_ftz(x); }

// Normal Euler flux through the scaled normal (Nx, Ny): F Nx + G Ny.
template <typename Real>
__device__ __forceinline__ void normal_flux(const Real u[4], Real Nx, Real Ny, Real gm1, Real f[4],
                                            Real& p) {
    Real ri = rcp_(u[0]);
    Real vx = u[1] * ri, vy = u[2] * ri;
    p = gm1 * (u[3] - Real(0.5) * (u[1] * vx + u[2] * vy));
    Real qn = vx * Nx + vy * Ny;
    f[0] = u[0] * qn;
    f[1] = u[1] * qn + p * Nx;
    f[2] = u[2] * qn + p * Ny;
    f[3] = (u[3] + p) * qn;
}

// HLLC through the unit normal (nx, ny) (Toro, Riemann Solvers and Numerical
// Methods for Fluid Dynamics, 3rd ed., sec. 10.4): Davis wave-speed bounds
// (eq. 10.48), contact speed S_M (eq. 10.37), star flux in its pressure form
// F*_K = (S_M (S_K U_K - F_K) + S_K p* (0, nx, ny, S_M)) / (S_K - S_M),
// p* = p_K + rho_K (S_K - q_K)(S_M - q_K).  Branch-free: both physical
// fluxes and the star flux are formed and the result selected (F_L when
// S_L >= 0, F_R when S_R <= 0), so a warp whose points fall in different
// wave regions runs one path; a star value formed where it is not selected
// (even inf or NaN) is discarded.
template <typename Real>
__device__ __forceinline__ void hllc(const Real uL[4], const Real uR[4], Real nx, Real ny,
                                     Real gamma, Real f[4]) {
    const Real gm1 = gamma - Real(1);
    Real rL = uL[0], rR = uR[0];
    Real iL = rcp_(rL), iR = rcp_(rR);
    Real vxL = uL[1] * iL, vyL = uL[2] * iL, vxR = uR[1] * iR, vyR = uR[2] * iR;
    Real pL = gm1 * (uL[3] - Real(0.5) * (uL[1] * vxL + uL[2] * vyL));
    Real pR = gm1 * (uR[3] - Real(0.5) * (uR[1] * vxR + uR[2] * vyR));
    Real qL = vxL * nx + vyL * ny, qR = vxR * nx + vyR * ny;
    Real cL = sqrt_(gamma * pL * iL), cR = sqrt_(gamma * pR * iR);
    Real SL = fmin(qL - cL, qR - cR), SR = fmax(qL + cL, qR + cR);
    const Real FL[4] = {rL * qL, uL[1] * qL + pL * nx, uL[2] * qL + pL * ny, (uL[3] + pL) * qL};
    const Real FR[4] = {rR * qR, uR[1] * qR + pR * nx, uR[2] * qR + pR * ny, (uR[3] + pR) * qR};
    Real dL = rL * (SL - qL), dR = rR * (SR - qR);
    Real SM = div_(pR - pL + dL * qL - dR * qR, dL - dR);
    const bool left = SM >= Real(0);
    Real d = left ? dL : dR, p = left ? pL : pR, q = left ? qL : qR, S = left ? SL : SR;
    Real ps = p + d * (SM - q);
    Real k = rcp_(S - SM);
    const bool sl = SL >= Real(0), sr = SR <= Real(0);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const Real uK = left ? uL[v] : uR[v], FK = left ? FL[v] : FR[v];
        const Real pn = v == 0 ? Real(0) : (v == 1 ? nx : (v == 2 ? ny : SM));
        const Real fs = (SM * (S * uK - FK) + S * ps * pn) * k;
        f[v] = sl ? FL[v] : (sr ? FR[v] : fs);
    }
}

// ------------------------------------------- deviation form (FP32 path) --
// FP32 states hold each cell mean as its deviation d = U - U_r from the
// solve's reference state U_r (the far field).  The flux terms of a stage
// are formed from d directly: the reference flux F(U_r) integrates to zero
// over every element (its volume and surface integrals cancel exactly for a
// constant flux), so only F(U_r + d) - F(U_r) enters the residual, and its
// rounding scales with the deviation instead of the state.  Primitive
// deviations: du = (dm - u_r drho) / rho, dp = (gamma - 1)(dE - 1/2 (m_r.du
// + dm.u)), with rho = rho_r + drho and u = u_r + du.
template <typename Real>
struct RefState {
    Real rho, mx, my, E, u, v, p, Ep;  // Ep = E + p
};
template <typename Real>
__device__ __forceinline__ RefState<Real> ref_state(const double f[4], double gamma) {
    const double u = f[1] / f[0], v = f[2] / f[0];
    const double p = (gamma - 1.0) * (f[3] - 0.5 * (f[1] * u + f[2] * v));
    return RefState<Real>{(Real)f[0], (Real)f[1], (Real)f[2], (Real)f[3], (Real)u, (Real)v, (Real)p,
                          (Real)(f[3] + p)};
}
template <typename Real>
struct DevPrims {
    Real rho, ir, du, dv, u, v, dp;
};
template <typename Real>
__device__ __forceinline__ DevPrims<Real> dev_prims(const Real d[4], const RefState<Real>& r, Real gm1) {
    DevPrims<Real> w;
    w.rho = r.rho + d[0];
    w.ir = rcp_(w.rho);
    w.du = (d[1] - r.u * d[0]) * w.ir;
    w.dv = (d[2] - r.v * d[0]) * w.ir;
    w.u = r.u + w.du;
    w.v = r.v + w.dv;
    w.dp = gm1 * (d[3] - Real(0.5) * (r.mx * w.du + r.my * w.dv + d[1] * w.u + d[2] * w.v));
    return w;
}
// F(U_r + d).N - F(U_r).N for a (scaled or unit) normal N.
template <typename Real>
__device__ __forceinline__ void dev_flux(const Real d[4], const DevPrims<Real>& w, const RefState<Real>& r,
                                         Real Nx, Real Ny, Real f[4]) {
    const Real q = w.u * Nx + w.v * Ny, dq = w.du * Nx + w.dv * Ny;
    f[0] = d[1] * Nx + d[2] * Ny;
    f[1] = r.mx * dq + d[1] * q + w.dp * Nx;
    f[2] = r.my * dq + d[2] * q + w.dp * Ny;
    f[3] = r.Ep * dq + (d[3] + w.dp) * q;
}
// Ghost deviation across a boundary edge (the far field is the reference
// state, so its deviation is zero; walls mirror the momentum).
template <typename Real>
__device__ __forceinline__ void ghost_dev(int tag, const Real d[4], const RefState<Real>& r, Real nx, Real ny,
                                          Real g[4]) {
    if (tag == RKDG_BC_FARFIELD) {
        g[0] = g[1] = g[2] = g[3] = Real(0);
    } else if (tag == RKDG_BC_OUTFLOW) {
        g[0] = d[0], g[1] = d[1], g[2] = d[2], g[3] = d[3];
    } else {
        const Real mn = (r.mx + d[1]) * nx + (r.my + d[2]) * ny;
        g[0] = d[0];
        g[1] = d[1] - Real(2) * mn * nx;
        g[2] = d[2] - Real(2) * mn * ny;
        g[3] = d[3];
    }
}
// HLLC (as hllc() above) in deviation form: returns F^ - F(U_r).n.  With
// d_K = rho_K (S_K - q_K), the contact offsets D_K = S_M - q_K come from
// pressure and velocity differences only,
//   D_L = (p_R - p_L + d_R (q_L - q_R)) / (d_L - d_R),
//   D_R = (p_R - p_L + d_L (q_L - q_R)) / (d_L - d_R),
// and the star flux is F*_K = F_K + S_K (U*_K - U_K) with
//   U*_K - U_K = D_K / (S_K - S_M) (U_K + (0, d_K n, d_K S_M + p_K)).
template <typename Real>
__device__ __forceinline__ void hllc_dev(const Real dL[4], const Real dR[4], Real nx, Real ny, Real gamma,
                                         const RefState<Real>& r, Real f[4]) {
    const Real gm1 = gamma - Real(1);
    const DevPrims<Real> L = dev_prims(dL, r, gm1), R = dev_prims(dR, r, gm1);
    const Real pL = r.p + L.dp, pR = r.p + R.dp;
    const Real qL = L.u * nx + L.v * ny, qR = R.u * nx + R.v * ny;
    const Real dqLR = (L.du - R.du) * nx + (L.dv - R.dv) * ny;  // q_L - q_R
    const Real cL = sqrt_(gamma * pL * L.ir), cR = sqrt_(gamma * pR * R.ir);
    const Real SL = fmin(qL - cL, qR - cR), SR = fmax(qL + cL, qR + cR);
    Real FL[4], FR[4];
    dev_flux(dL, L, r, nx, ny, FL);
    dev_flux(dR, R, r, nx, ny, FR);
    const Real kL = L.rho * (SL - qL), kR = R.rho * (SR - qR);
    const Real idk = rcp_(kL - kR);
    const Real dpRL = R.dp - L.dp;
    const Real DL = (dpRL + kR * dqLR) * idk, DR = (dpRL + kL * dqLR) * idk;
    const Real SM = qL + DL;
    // one selection instead of hllc()'s three-way one: the result is
    // F_K + c (U_K + ex) with K = L when S_L >= 0, R when S_R <= 0 (both
    // with c = 0) and else the side of S_M, which equals F_L, F_R or F*_K
    // exactly as selected there (S_M stays finite while either side has a
    // positive sound speed)
    const bool sl = SL >= Real(0), sr = SR <= Real(0);
    const bool left = sl || (!sr && SM >= Real(0));
    const Real S = left ? SL : SR, D = left ? DL : DR, k = left ? kL : kR, p = left ? pL : pR;
    const Real c = (sl || sr) ? Real(0) : S * D * rcp_(S - SM);
    const Real UK[4] = {r.rho + (left ? dL[0] : dR[0]), r.mx + (left ? dL[1] : dR[1]),
                        r.my + (left ? dL[2] : dR[2]), r.E + (left ? dL[3] : dR[3])};
    const Real ex[4] = {Real(0), k * nx, k * ny, k * SM + p};
    if constexpr (sizeof(Real) == 4) {  // by component pairs, as the scalar form
        const float2 cc = make_float2(c, c);
        const float2 e01 = f2add(make_float2(UK[0], UK[1]), make_float2(ex[0], ex[1]));
        const float2 e23 = f2add(make_float2(UK[2], UK[3]), make_float2(ex[2], ex[3]));
        const float2 r01 = f2fma(cc, e01, make_float2(left ? FL[0] : FR[0], left ? FL[1] : FR[1]));
        const float2 r23 = f2fma(cc, e23, make_float2(left ? FL[2] : FR[2], left ? FL[3] : FR[3]));
        f[0] = r01.x, f[1] = r01.y, f[2] = r23.x, f[3] = r23.y;
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) f[v] = (left ? FL[v] : FR[v]) + c * (UK[v] + ex[v]);
    }
}

// ---------------------------------------------------------- reductions --
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide max of up to three non-negative doubles, then one atomicMax
// each on their bit patterns (ordered like the values for x >= 0; a NaN
// compares above +inf and so propagates).
__device__ __forceinline__ void block_max3_atomic(double a, double b, double c,
                                                  unsigned long long* da,
                                                  unsigned long long* db,
                                                  unsigned long long* dc) {
    __shared__ double sm[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_max(a);
    b = warp_max(b);
    c = warp_max(c);
    if (lane == 0) {
        sm[0][wid] = a;
        sm[1][wid] = b;
        sm[2][wid] = c;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        a = lane < nw ? sm[0][lane] : 0.0;
        b = lane < nw ? sm[1][lane] : 0.0;
        c = lane < nw ? sm[2][lane] : 0.0;
        a = warp_max(a);
        b = warp_max(b);
        c = warp_max(c);
        if (lane == 0) {
            if (da) atomicMax(da, (unsigned long long)__double_as_longlong(a));
            if (db) atomicMax(db, (unsigned long long)__double_as_longlong(b));
            if (dc) atomicMax(dc, (unsigned long long)__double_as_longlong(c));
        }
    }
}

// sqrt that returns 0 at 0 (the FP32 form uses the reciprocal square root).
__device__ __forceinline__ double sqrt0_(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt0_(float x) { return x > 0.0f ? x * rsqrt_ftz(x) : 0.0f; }

// Edge lengths |N_k| and 1 / area of an element from its FP64 J^-1 rows:
// N_k = 2 area (r0 + r1, -r0, -r1) formed in the working precision from
// the rounded rows, its length there; 1 / area = 2 det J^-1.  The tile kernel forms the same
// values in phase A.
template <typename Real>
__device__ __forceinline__ void elem_lengths(double2 r0, double2 r1, Real len[3], Real& inv_area) {
    const double det = r0.x * r1.y - r0.y * r1.x;
    inv_area = (Real)(2.0 * det);
    const Real area2 = rcp_((Real)det);
    const Real ax = (Real)r0.x, ay = (Real)r0.y, bx = (Real)r1.x, by = (Real)r1.y;
    const Real cx[3] = {ax + bx, -ax, -bx}, cy[3] = {ay + by, -ay, -by};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const Real Nx = cx[k] * area2, Ny = cy[k] * area2;
        len[k] = sqrt_(Nx * Nx + Ny * Ny);
    }
}

// (|u| + c) * perimeter / area of a cell mean (src/kernelfunctions.cu:19-25)
// in the working precision; the max over cells and dt = CFL / max are FP64.
// A non-physical mean (rho <= 0, p <= 0, NaN) sets bad and returns NaN.
template <typename Real>
__device__ __forceinline__ double wave_of(const Real m[4], Real gamma, const Real len[3], Real inv_area,
                                          bool& bad) {
    const Real ri = rcp_(m[0]);
    const Real u = m[1] * ri, v = m[2] * ri;
    const Real p = (gamma - Real(1)) * (m[3] - Real(0.5) * (m[1] * u + m[2] * v));
    bad = !(m[0] > Real(0)) || !(p > Real(0));
    const Real c = sqrt0_(gamma * p * ri);
    const Real w = (sqrt0_(u * u + v * v) + c) * ((len[0] + len[1] + len[2]) * inv_area);
    return bad ? __longlong_as_double(0x7ff8000000000000LL) : (double)w;
}

// ------------------------------------------------------------ the stage --
// MODE_STAGE_COMP: the FP32 stage of RKDG_FP32C (cell means updated in FP64
// from their high and low parts); MODE_LIMITED (added to a stage mode): the
// stage is followed by the TVB limiter and writes its per-tile test
// (tvb_keeps) for it.  Kernels without MODE_LIMITED carry none of that code.
enum { MODE_STAGE = 0, MODE_RESIDUAL = 1, MODE_STAGE_COMP = 2, MODE_LIMITED = 4 };

// Exact test that the TVB limiter (limit_element) leaves an element unchanged: every
// row of its left eigenvector matrix has 1-norm at most B (|q|, |q_t| <=
// |vx| + |vy|, |nx| + |ny| <= 1.5; 1.001 covers rounding), so when B times
// the largest |P1 midpoint increment| (tilde) is within the smallest TVB
// threshold, every characteristic increment is kept.  A non-physical mean
// (NaN bound) fails the test.  The stage kernel applies it to each stage's
// output per tile, so the limiter can skip whole tiles.
template <typename Real>
__device__ __forceinline__ bool tvb_keeps(const Real mean[4], Real gamma, Real tmax, Real thr_min) {
    const Real rho = mean[0], ir = Real(1) / rho, vx = mean[1] * ir, vy = mean[2] * ir;
    const Real p = (gamma - Real(1)) * (mean[3] - Real(0.5) * rho * (vx * vx + vy * vy));
    const Real c = sqrt(gamma * p * ir);
    const Real k2 = Real(0.5) * (vx * vx + vy * vy);
    const Real b1 = (gamma - Real(1)) / (c * c), b2 = b1 * k2, ic = Real(1) / c;
    const Real av = fabs(vx) + fabs(vy);
    const Real B0 = Real(0.5) * (b2 + av * ic + b1 * av + Real(1.5) * ic + b1);
    const Real B1 = fabs(Real(1) - b2) + b1 * av + b1;
    const Real B2 = av + Real(1.5);
    const Real B = fmax(fmax(B0, B1), B2) * Real(1.001);
    return B * tmax <= thr_min;
}
// The TVB thresholds M (2 |m_k - b0|)^2 of an element's three edges (m_k
// the edge midpoint, b0 the centroid): m_k - b0 = J d_k with the
// reference-element offsets d_0 = (1/6, 1/6), d_1 = (-1/3, 1/6),
// d_2 = (1/6, -1/3) and the columns of J, x_1 - x_0 = (c0x, c0y) and
// x_2 - x_0 = (c1x, c1y); also the unit directions (m_k - b0)/|m_k - b0|.
template <typename Real>
__device__ __forceinline__ void tvb_geometry(Real c0x, Real c0y, Real c1x, Real c1y, Real tvb_m, Real dirx[3],
                                             Real diry[3], Real thr[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const Real dxi = k == 1 ? Real(-1.0 / 3.0) : Real(1.0 / 6.0), deta = k == 2 ? Real(-1.0 / 3.0) : Real(1.0 / 6.0);
        const Real dx = c0x * dxi + c1x * deta, dy = c0y * dxi + c1y * deta;
        const Real r2 = dx * dx + dy * dy, irl = Real(1) / sqrt(r2);
        dirx[k] = dx * irl;
        diry[k] = dy * irl;
        thr[k] = tvb_m * (Real(4) * r2);
    }
}
#include "stage_tiled.cuh"

// CFL measure of the current state per solve (first step, rkdg_compute_dt):
// one CTA per tile (its threads loop over the tile's elements), a block max
// per tile, one atomicMax into its solve.
constexpr int kAuxBlock = 128;
template <typename Real>
__global__ void __launch_bounds__(kAuxBlock) wave_kernel(const TileArgs ta, int ld,
                                                         const Real* __restrict__ U,
                                                         const double* __restrict__ jinv, double gamma,
                                                         StepCtl* ctl, const double* __restrict__ refs) {
    const int ntiles = ta.ntiles_dev ? *ta.ntiles_dev : ta.ntiles;
    if ((int)blockIdx.x >= ntiles) return;
    const int4 d0 = __ldg(ta.desc + 2 * blockIdx.x);
    StepCtl* c = ctl + d0.z;
    const double* ref = refs + 4 * d0.z;
    double w = 0.0;
    for (int x = threadIdx.x; x < d0.y; x += blockDim.x) {
        const int e = d0.x + x;
        Real m[4];
        load_mean<Real, 1>(U, ld, e, m);
        const double2* j2 = reinterpret_cast<const double2*>(jinv);
        bool bad;
        Real mm[4], len[3], ia;
#pragma unroll
        for (int v = 0; v < 4; ++v) mm[v] = m[v] + ref_of<Real>(ref, v);
        elem_lengths<Real>(j2[e], j2[ld + e], len, ia);
        w = fmax(w, wave_of<Real>(mm, (Real)gamma, len, ia, bad));
        if (bad) atomicOr(&c->error, 1);
    }
    block_max3_atomic(w, 0.0, 0.0, &c->wave_bits, nullptr, nullptr);
}

__global__ void reset_wave_kernel(StepCtl* ctl, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ctl[i].wave_bits = 0ull;
}

// dt of the step: CFL (or fixed), clipped to land on t_final; advances t.
__global__ void step_begin_kernel(StepCtl* ctls, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    StepCtl* ctl = ctls + i;
    if (ctl->done) return;
    double dt = ctl->dt_fixed > 0 ? ctl->dt_fixed : ctl->cfl / __longlong_as_double((long long)ctl->wave_bits);
    bool last = false;
    if (ctl->t_final > 0) {
        double rem = ctl->t_final - ctl->t;
        if (!(rem > 0)) {
            ctl->done = 1;
            return;
        }
        if (dt >= rem) {
            dt = rem;
            last = true;
        }
    }
    if (!(dt > 0) || !isfinite(dt)) {  // non-physical state: stop, report
        ctl->error |= 1;
        ctl->done = 1;
        return;
    }
    ctl->dt = dt;
    ctl->t = last ? ctl->t_final : ctl->t + dt;
    ctl->step += 1;
    ctl->wave_bits = 0ull;
    ctl->mon_bits[0] = 0ull;
    ctl->mon_bits[1] = 0ull;
}

// ------------------------------------------------------------ limiter --
// TVB minmod on characteristic variables for the P1 part (Cockburn & Shu,
// J. Comput. Phys. 141 (1998) 199-224, sec. 2.4/3.3).  In place: only
// modes >= 1 change, and neighbours read only cell means.  Per edge k the
// table holds (alpha, beta) of m_k - b0 = alpha (b_k - b0) + beta (b_j - b0)
// in the working precision (rows k of [3][ld]); the pairing edge j is bit
// 12 + k of the packed connectivity word, and the direction m_k - b0 (edge
// midpoint minus centroid) with its length, the TVB threshold's scale, are
// formed here from J^-1: m_k - b0 = J d_k with the reference-element offsets
// d_0 = (1/6, 1/6), d_1 = (-1/3, 1/6), d_2 = (1/6, -1/3), and J = (J^-1)^-1.
template <typename Real, int NB>
__device__ __forceinline__ void limit_element(int e, int ld, Real* __restrict__ U,
                                              const int4* __restrict__ conn,
                                              const void* __restrict__ limv,
                                              const double* __restrict__ jinv, double gammad,
                                              double f0, double f1, double f2, double f3,
                                              double tvb_m, const Tab<Real>& tb) {
    using Pair = typename std::conditional<sizeof(Real) == 8, double2, float2>::type;
    const Pair* lim = static_cast<const Pair*>(limv);
    const double2* j2 = reinterpret_cast<const double2*>(jinv);
    const double2 r0 = __ldg(j2 + e), r1 = __ldg(j2 + ld + e);
    Real u[3][4];
    load_state<Real, 3>(U, ld, e, u);
    const int4 cn = __ldg(conn + e);
    const Real gamma = (Real)gammad;
    const Real far[4] = {(Real)f0, (Real)f1, (Real)f2, (Real)f3};
    const double fref[4] = {f0, f1, f2, f3};
    Real mean[4], dev0[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        dev0[v] = u[0][v];
        mean[v] = u[0][v] + ref_of<Real>(fref, v);
    }
    Real nbm[3][4], tilde[3][4];
    const unsigned pair_bits = ((unsigned)cn.w >> 12) & 7u;
    // the directions and threshold scales in the working precision: FP64
    // for the parity path, FP32 (from the FP64 J^-1 rows) for the FP32 forms
    const Real idet = Real(1) / (Real)(r0.x * r1.y - r0.y * r1.x);  // det J
    // columns of J: x_1 - x_0 and x_2 - x_0
    Real dirx[3], diry[3], thrk[3];
    tvb_geometry<Real>((Real)r1.y * idet, -(Real)r1.x * idet, -(Real)r0.y * idet, (Real)r0.x * idet, (Real)tvb_m,
                       dirx, diry, thrk);
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int v = 0; v < 4; ++v) tilde[k][v] = tb.mphi[k][0] * u[1][v] + tb.mphi[k][1] * u[2][v];
    // the mean's primitive state and sound speed (the eigenvectors below)
    const Real rho = mean[0], ir = Real(1) / rho, vx = mean[1] * ir, vy = mean[2] * ir;
    const Real p = (gamma - Real(1)) * (mean[3] - Real(0.5) * rho * (vx * vx + vy * vy));
    const Real c = sqrt(gamma * p * ir), H = (mean[3] + p) * ir;
    const Real k2 = Real(0.5) * (vx * vx + vy * vy);
    const Real b1 = (gamma - Real(1)) / (c * c), b2 = b1 * k2, ic = Real(1) / c;
    {
        // exact early exit (tvb_keeps): uniform and near-uniform regions skip
        // the neighbour means and the decompositions
        Real tmax = Real(0);
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int v = 0; v < 4; ++v) tmax = fmax(tmax, fabs(tilde[k][v]));
        if (tvb_keeps<Real>(mean, gamma, tmax, fmin(fmin(thrk[0], thrk[1]), thrk[2]))) return;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        int ne = k == 0 ? cn.x : (k == 1 ? cn.y : cn.z);
        if (ne >= 0) {
            load_mean<Real, 1>(U, ld, ne, nbm[k]);
#pragma unroll
            for (int v = 0; v < 4; ++v) nbm[k][v] += ref_of<Real>(fref, v);
        } else {
            // ghost mean across a boundary edge, mirrored about the unit
            // normal of edge k (N_k / area = 2(r0+r1), -2 r0, -2 r1)
            int tag = ((unsigned)cn.w >> (6 + 2 * k)) & 3u;
            double Nx = k == 0 ? r0.x + r1.x : (k == 1 ? -r0.x : -r1.x);
            double Ny = k == 0 ? r0.y + r1.y : (k == 1 ? -r0.y : -r1.y);
            double il = 1.0 / sqrt(Nx * Nx + Ny * Ny);
            ghost<Real>(tag, mean, far, (Real)(Nx * il), (Real)(Ny * il), nbm[k]);
        }
    }
    bool limited = false;
    Real delta[3][4];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const Pair ab = __ldg(lim + (size_t)k * ld + e);
        const Real al = (Real)ab.x, be = (Real)ab.y;
        const int j = (pair_bits >> k) & 1u ? (k + 2) % 3 : (k + 1) % 3;
        const Real nx = dirx[k], ny = diry[k];
        const Real thr = thrk[k];
        Real dbar[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Real nj = j == 0 ? nbm[0][v] : (j == 1 ? nbm[1][v] : nbm[2][v]);
            dbar[v] = al * (nbm[k][v] - mean[v]) + be * (nj - mean[v]);
        }
        // eigenvectors of the Euler flux Jacobian in direction n at the mean
        const Real q = vx * nx + vy * ny, qt = -vx * ny + vy * nx;
        Real Lm[4][4] = {{Real(0.5) * (b2 + q * ic), Real(0.5) * (-b1 * vx - nx * ic),
                          Real(0.5) * (-b1 * vy - ny * ic), Real(0.5) * b1},
                         {Real(1) - b2, b1 * vx, b1 * vy, -b1},
                         {-qt, -ny, nx, Real(0)},
                         {Real(0.5) * (b2 - q * ic), Real(0.5) * (-b1 * vx + nx * ic),
                          Real(0.5) * (-b1 * vy + ny * ic), Real(0.5) * b1}};
        Real Rc[4][4] = {{Real(1), vx - c * nx, vy - c * ny, H - q * c},
                         {Real(1), vx, vy, k2},
                         {Real(0), -ny, nx, qt},
                         {Real(1), vx + c * nx, vy + c * ny, H + q * c}};  // rows = right vectors
        Real wl[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            Real wt = Lm[r][0] * tilde[k][0] + Lm[r][1] * tilde[k][1] + Lm[r][2] * tilde[k][2] +
                      Lm[r][3] * tilde[k][3];
            Real wd = Real(1.5) * (Lm[r][0] * dbar[0] + Lm[r][1] * dbar[1] + Lm[r][2] * dbar[2] +
                                   Lm[r][3] * dbar[3]);
            Real out;
            if (fabs(wt) <= thr) {
                out = wt;
            } else {
                out = (wt > Real(0) && wd > Real(0)) ? fmin(wt, wd)
                      : (wt < Real(0) && wd < Real(0)) ? fmax(wt, wd)
                                                       : Real(0);
                if (out != wt) limited = true;
            }
            wl[r] = out;
        }
#pragma unroll
        for (int v = 0; v < 4; ++v)
            delta[k][v] = Rc[0][v] * wl[0] + Rc[1][v] * wl[1] + Rc[2][v] * wl[2] + Rc[3][v] * wl[3];
    }
    if (!limited) return;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        Real s = delta[0][v] + delta[1][v] + delta[2][v];
        if (s != Real(0)) {
            Real pos = Real(0), neg = Real(0);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                pos += fmax(Real(0), delta[k][v]);
                neg += fmax(Real(0), -delta[k][v]);
            }
            Real tp = pos > Real(0) ? fmin(Real(1), neg / pos) : Real(1);
            Real tn = neg > Real(0) ? fmin(Real(1), pos / neg) : Real(1);
#pragma unroll
            for (int k = 0; k < 3; ++k)
                delta[k][v] = tp * fmax(Real(0), delta[k][v]) - tn * fmax(Real(0), -delta[k][v]);
        }
    }
    Real out[NB][4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        out[0][v] = dev0[v];
        out[1][v] = tb.minv[0][0] * delta[0][v] + tb.minv[0][1] * delta[1][v] + tb.minv[0][2] * delta[2][v];
        out[2][v] = tb.minv[1][0] * delta[0][v] + tb.minv[1][1] * delta[1][v] + tb.minv[1][2] * delta[2][v];
#pragma unroll
        for (int i = 3; i < NB; ++i) out[i][v] = Real(0);
    }
    store_state<Real, NB>(U, ld, e, out);
}

// One tile of the limiter (all threads of the CTA): tiles of solves whose
// flag is 0 (when flags is set) or whose control block says done are
// skipped; P1 and P2 tiles limit their P1 part (P2 tiles drop their
// quadratic modes where limited).
template <typename Real>
__device__ __forceinline__ void limit_tile(const TileArgs& ta, int tile, int ld, Real* __restrict__ U,
                                           const int4* __restrict__ conn, const void* __restrict__ lim,
                                           const double* __restrict__ jinv, const int* __restrict__ flags,
                                           const double* __restrict__ refs, double gamma, double tvb_m, int cfg1,
                                           int cfg2, const StepCtl* __restrict__ ctl) {
    const int4 d0 = __ldg(ta.desc + 2 * tile);
    if ((flags && !flags[d0.z]) || (ctl && ctl[d0.z].done)) return;
    const double* f = refs + 4 * d0.z;
    for (int x = threadIdx.x; x < d0.y; x += blockDim.x) {
        const int e = d0.x + x;
        if (d0.w == 2)
            limit_element<Real, 6>(e, ld, U, conn, lim, jinv, gamma, f[0], f[1], f[2], f[3], tvb_m, tab<Real>(cfg2));
        else
            limit_element<Real, 3>(e, ld, U, conn, lim, jinv, gamma, f[0], f[1], f[2], f[3], tvb_m, tab<Real>(cfg1));
    }
}

// The limiter over tiles (one solve, a pack of solves or the serving pool).
// Every path runs this one kernel, so a solve limits to the same bits
// wherever it runs.  Without a tile list every tile is visited; with one
// (the stage kernel's LimitList), only the listed tiles, spread over the
// CTAs of a persistent grid: most of a flow's tiles cannot change (no
// element fails tvb_keeps) and cost nothing.
template <typename Real>
__global__ void __launch_bounds__(kAuxBlock) tiled_limiter_kernel(const TileArgs ta, int ld,
                                                              Real* __restrict__ U,
                                                              const int4* __restrict__ conn,
                                                              const void* __restrict__ lim,
                                                              const double* __restrict__ jinv,
                                                              const int* __restrict__ flags,
                                                              const double* __restrict__ refs,
                                                              double gamma, double tvb_m,
                                                              int cfg1, int cfg2,
                                                              const StepCtl* __restrict__ ctl,
                                                              int* __restrict__ tile_flags,
                                                              int* __restrict__ tile_list, int tile_cap) {
    if (tile_list == nullptr) {
        const int ntiles = ta.ntiles_dev ? *ta.ntiles_dev : ta.ntiles;
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
            limit_tile<Real>(ta, tile, ld, U, conn, lim, jinv, flags, refs, gamma, tvb_m, cfg1, cfg2, ctl);
        return;
    }
    // every CTA reads the count before the last one resets it (the reset
    // follows every CTA's arrival below)
    const int n = min(*(volatile int*)tile_list, tile_cap);
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int tile = tile_list[kListHead + i];
        limit_tile<Real>(ta, tile, ld, U, conn, lim, jinv, flags, refs, gamma, tvb_m, cfg1, cfg2, ctl);
        if (threadIdx.x == 0) tile_flags[tile] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(tile_list + 1, 1) == (int)gridDim.x - 1) {  // the last CTA: empty list for the next stage
            tile_list[0] = 0;
            tile_list[1] = 0;
        }
    }
}

// ------------------------------------------------- halo row exchange --
// Rows 0..nrows-1 (16-byte packs) of the listed elements of a state, to or
// from a contiguous buffer [n][nrows]: the pack and unpack of a partition's
// halo exchange.  An index outside [0, T) is skipped and sets bit 2 of the
// error word.
__global__ void gather_rows_kernel(const int4* __restrict__ U, int ld, int T, const int* __restrict__ idx, int n,
                                   int nrows, int4* __restrict__ out, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * nrows) return;
    const int j = i / nrows, r = i - j * nrows;
    const int e = idx[j];
    if (e < 0 || e >= T) {
        atomicOr(err, 4);
        return;
    }
    out[i] = U[(size_t)r * ld + e];
}

__global__ void scatter_rows_kernel(int4* __restrict__ U, int ld, int T, const int* __restrict__ idx, int n,
                                    int nrows, const int4* __restrict__ in, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * nrows) return;
    const int j = i / nrows, r = i - j * nrows;
    const int e = idx[j];
    if (e < 0 || e >= T) {
        atomicOr(err, 4);
        return;
    }
    U[(size_t)r * ld + e] = in[i];
}

// ---------------------------------------------------- basis conversion --
// Caller layout [4][NB][ldh] FP64 (caller element order) <-> HBM packs
// (internal order), with an optional per-element basis change.
template <typename Real, int NB>
__global__ void import_kernel(int T, int ld, const double* __restrict__ st, int ldh,
                              const double* __restrict__ conv, const int32_t* __restrict__ perm,
                              Real* __restrict__ U, Ref4 ref, int lo_row) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    const int c = perm ? perm[e] : e;
    double a[NB][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int i = 0; i < NB; ++i) a[i][v] = st[((size_t)v * NB + i) * ldh + c];
    Real b[NB][4];
    if (conv) {
        const double* C = conv + (size_t)36 * e;
#pragma unroll
        for (int j = 0; j < NB; ++j)
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                double s = 0;
#pragma unroll
                for (int i = 0; i < NB; ++i) s += a[i][v] * C[6 * i + j];
                b[j][v] = (Real)s;
            }
    } else {
#pragma unroll
        for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) b[i][v] = (Real)a[i][v];
    }
    float lo[4] = {0.f, 0.f, 0.f, 0.f};
    if (stores_deviation<Real>()) {  // mean row = basis 0 (basis-invariant)
        const double* Cm = conv ? conv + (size_t)36 * e : nullptr;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double m = 0;
            if (Cm) {
#pragma unroll
                for (int i = 0; i < NB; ++i) m += a[i][v] * Cm[6 * i];
            } else {
                m = a[0][v];
            }
            b[0][v] = (Real)(m - ref.v[v]);
            lo[v] = (float)((m - ref.v[v]) - (double)b[0][v]);
        }
    }
    store_state<Real, NB>(U, ld, e, b);
    if (sizeof(Real) == 4 && lo_row >= 0)  // FP32C: the low parts of the cell means
        reinterpret_cast<float4*>(U)[(size_t)lo_row * ld + e] = make_float4(lo[0], lo[1], lo[2], lo[3]);
}

template <typename Real, int NB>
__global__ void export_kernel(int T, int ld, const Real* __restrict__ U,
                              const double* __restrict__ conv, const int32_t* __restrict__ perm,
                              double* __restrict__ st, int ldh, int residual_scale,
                              const double* __restrict__ jinv, Ref4 ref, int lo_row) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= T) return;
    const int c = perm ? perm[e] : e;
    Real bl[NB][4];
    load_state<Real, NB>(U, ld, e, bl);
    double b[NB][4];
#pragma unroll
    for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) b[i][v] = (double)bl[i][v];
    if (sizeof(Real) == 4 && lo_row >= 0 && !residual_scale) {  // FP32C: add the low parts
        const float4 l = reinterpret_cast<const float4*>(U)[(size_t)lo_row * ld + e];
        b[0][0] += (double)l.x, b[0][1] += (double)l.y, b[0][2] += (double)l.z, b[0][3] += (double)l.w;
    }
    if (stores_deviation<Real>() && !residual_scale)
#pragma unroll
        for (int v = 0; v < 4; ++v) b[0][v] += ref.v[v];
    double scale = 1.0;
    if (residual_scale) {  // area = 1 / (2 det J^-1)
        const double2* j2 = reinterpret_cast<const double2*>(jinv);
        double2 r0 = j2[e], r1 = j2[ld + e];
        scale = 0.5 / (r0.x * r1.y - r0.y * r1.x);
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double s;
            if (conv) {
                const double* M = conv + (size_t)36 * e + 6 * i;
                s = 0;
#pragma unroll
                for (int j = 0; j < NB; ++j) s += M[j] * b[j][v];
            } else {
                s = b[i][v];
            }
            st[((size_t)v * NB + i) * ldh + c] = scale * s;
        }
}

// --------------------------------------------------- conservation totals --
constexpr int kTotBlock = 256;
int totals_partial_count(int T) { return (T + kTotBlock - 1) / kTotBlock; }

template <typename Real>
__global__ void __launch_bounds__(kTotBlock) totals_partial_kernel(int T, int ld,
                                                                   const Real* __restrict__ U,
                                                                   const double* __restrict__ jinv,
                                                                   double* __restrict__ partial,
                                                                   Ref4 ref, int lo_row) {
    __shared__ double s[4][kTotBlock];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double v4[4] = {0, 0, 0, 0};
    if (e < T) {
        Real m[4];
        load_mean<Real, 1>(U, ld, e, m);
        const double2* j2 = reinterpret_cast<const double2*>(jinv);
        double2 r0 = j2[e], r1 = j2[ld + e];
        double area = 0.5 / (r0.x * r1.y - r0.y * r1.x);
        double lo[4] = {0.0, 0.0, 0.0, 0.0};
        if (sizeof(Real) == 4 && lo_row >= 0) {  // FP32C: the low parts of the means
            const float4 l = reinterpret_cast<const float4*>(U)[(size_t)lo_row * ld + e];
            lo[0] = l.x, lo[1] = l.y, lo[2] = l.z, lo[3] = l.w;
        }
        for (int v = 0; v < 4; ++v)
            v4[v] = area * (((double)m[v] + lo[v]) + (stores_deviation<Real>() ? ref.v[v] : 0.0));
    }
    for (int v = 0; v < 4; ++v) s[v][threadIdx.x] = v4[v];
    __syncthreads();
    for (int o = kTotBlock / 2; o > 0; o >>= 1) {  // fixed-order tree: deterministic
        if (threadIdx.x < o)
            for (int v = 0; v < 4; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 4; ++v) partial[(size_t)4 * blockIdx.x + v] = s[v][0];
}

__global__ void __launch_bounds__(kTotBlock) totals_final_kernel(int n, const double* __restrict__ partial,
                                                                 double* __restrict__ out) {
    __shared__ double s[4][kTotBlock];
    double acc[4] = {0, 0, 0, 0};
    for (int i = threadIdx.x; i < n; i += kTotBlock)
        for (int v = 0; v < 4; ++v) acc[v] += partial[(size_t)4 * i + v];
    for (int v = 0; v < 4; ++v) s[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int o = kTotBlock / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int v = 0; v < 4; ++v) s[v][threadIdx.x] += s[v][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 4; ++v) out[v] = s[v][0];
}

// ----------------------------------------------------------- launchers --
namespace {

// The device's largest opt-in dynamic + static shared memory per CTA, less
// the stage kernel's static shared memory (barrier, maxima, dt, tables).
size_t smem_limit() {
    static int limit = 0;
    if (limit == 0) {
        int dev = 0, v = 0;
        RKDG_CUDA_TRY(cudaGetDevice(&dev));
        RKDG_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        limit = v;
    }
    return (size_t)limit - 1024;
}

}  // namespace

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0, v = 0;
        RKDG_CUDA_TRY(cudaGetDevice(&dev));
        RKDG_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        n = v;
    }
    return n;
}

namespace {

// Shared-memory attributes of one instantiation for a halo size; returns the
// dynamic shared memory per CTA.

template <typename Real, int NQ2, int FLUX, int MODE, int ORD, int BT, int LAT = 0>
size_t prepare_tiled(int max_halo) {
    const size_t smem = TiledSmem<Real, ORD, FLUX, BT>::bytes(max_halo);
    if (smem > smem_limit())
        throw Error{RKDG_ERR_INVALID, "tiles of " + std::to_string(BT) + " elements with halo lists of " +
                                          std::to_string(max_halo) + " entries need " + std::to_string(smem) +
                                          " bytes of shared memory per CTA, above the device's limit: use "
                                          "128-element tiles or the locality order"};
    // dynamic + static shared memory above 48 KB needs the opt-in.  Per
    // instantiation; raised when a context with a larger halo appears.
    static size_t configured = 0;
    if (configured == 0)  // give shared memory the whole carveout
        RKDG_CUDA_TRY(cudaFuncSetAttribute(tiled_stage_kernel<Real, NQ2, FLUX, MODE, ORD, BT, LAT>,
                                           cudaFuncAttributePreferredSharedMemoryCarveout,
                                           (int)cudaSharedmemCarveoutMaxShared));
    if (smem > configured) {
        RKDG_CUDA_TRY(cudaFuncSetAttribute(tiled_stage_kernel<Real, NQ2, FLUX, MODE, ORD, BT, LAT>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        configured = smem;
    }
    return smem;
}

template <typename Real, int NQ2, int FLUX, int MODE, int ORD, int BT>
int occupancy_tiled(int max_halo) {
    const size_t smem = prepare_tiled<Real, NQ2, FLUX, MODE, ORD, BT>(max_halo);
    int n = 0;
    RKDG_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &n, tiled_stage_kernel<Real, NQ2, FLUX, MODE, ORD, BT>, BT, smem));
    return n;
}

template <typename Real, int NQ2, int FLUX, int MODE, int ORD, int BT, int LAT = 0>
void launch_tiled(const StageArgs& a, const TileArgs& t, int ctas, cudaStream_t s) {
    const size_t smem = prepare_tiled<Real, NQ2, FLUX, MODE, ORD, BT, LAT>(t.max_halo);
    const int grid = (ctas > 0 && ctas < t.ntiles) ? ctas : t.ntiles;
    if (grid > 0) tiled_stage_kernel<Real, NQ2, FLUX, MODE, ORD, BT, LAT><<<grid, BT, smem, s>>>(a, t);
}

// Tile sizes the stage kernel is built for: 128 everywhere, 256 for the
// stage (not the residual) kernels the batch autotuner may pick.  FP64
// launches of one CTA per tile whose tiles all fit on the device at once
// run the latency form (fewer warps per SM, no register spills: 3,200- and
// 28,800-triangle P2 meshes step 3-4 % faster than in the throughput form).
template <typename Real, int NQ2, int FLUX, int MODE, int ORD>
void launch_tiled_bt(const StageArgs& a, const TileArgs& t, int ctas, cudaStream_t s) {
    if (t.tile == 128) {
        if constexpr (sizeof(Real) == 8) {
            const int fit = sm_count() * TiledOccupancy<Real, ORD, 128, 1>::value;
            if ((ctas <= 0 || ctas >= t.ntiles) && t.ntiles_dev == nullptr && t.ntiles <= fit)
                return launch_tiled<Real, NQ2, FLUX, MODE, ORD, 128, 1>(a, t, ctas, s);
        }
        return launch_tiled<Real, NQ2, FLUX, MODE, ORD, 128>(a, t, ctas, s);
    }
    if constexpr (MODE != MODE_RESIDUAL && !(MODE & MODE_LIMITED))
        if (t.tile == 256) return launch_tiled<Real, NQ2, FLUX, MODE, ORD, 256>(a, t, ctas, s);
    throw Error{RKDG_ERR_INVALID, "no stage kernel for a tile of " + std::to_string(t.tile) + " elements"};
}

template <typename Real, int FLUX, int MODE>
void dispatch_tiled(const StageArgs& a, const TileArgs& t, int order, int nq, int ctas,
                    cudaStream_t s) {
    if (order == 1) return launch_tiled_bt<Real, 6, FLUX, MODE, 1>(a, t, ctas, s);
    if (order == 2 && nq == 7) return launch_tiled_bt<Real, 7, FLUX, MODE, 2>(a, t, ctas, s);
    if (order == 2 && nq == 6) return launch_tiled_bt<Real, 6, FLUX, MODE, 2>(a, t, ctas, s);
    if (order == 3 && nq == 6) return launch_tiled_bt<Real, 6, FLUX, MODE, 3>(a, t, ctas, s);
    throw Error{RKDG_ERR_INVALID, "unsupported order/rule combination for the tiled kernel"};
}

template <int MODE>
void dispatch(const StageArgs& a, const TileArgs& t, int order, int nq, int flux, int prec, int ctas,
              cudaStream_t s) {
    const bool hllc = flux == RKDG_FLUX_HLLC;
    if (prec == RKDG_FP32) {
        if (hllc) dispatch_tiled<float, RKDG_FLUX_HLLC, MODE>(a, t, order, nq, ctas, s);
        else dispatch_tiled<float, RKDG_FLUX_LLF, MODE>(a, t, order, nq, ctas, s);
    } else if constexpr (!(MODE & MODE_STAGE_COMP)) {
        if (hllc) dispatch_tiled<double, RKDG_FLUX_HLLC, MODE>(a, t, order, nq, ctas, s);
        else dispatch_tiled<double, RKDG_FLUX_LLF, MODE>(a, t, order, nq, ctas, s);
    } else {
        throw Error{RKDG_ERR_INVALID, "a low-part row needs the FP32 stage"};
    }
    RKDG_CUDA_TRY(cudaGetLastError());
}

}  // namespace

void launch_stage(const StageArgs& a, const TileArgs& t, int order, int nq, int flux, int prec, int ctas,
                  cudaStream_t stream) {
    if (a.tile_flags != nullptr) {
        if (a.lo_row >= 0) dispatch<MODE_STAGE_COMP | MODE_LIMITED>(a, t, order, nq, flux, prec, ctas, stream);
        else dispatch<MODE_STAGE | MODE_LIMITED>(a, t, order, nq, flux, prec, ctas, stream);
    } else {
        if (a.lo_row >= 0) dispatch<MODE_STAGE_COMP>(a, t, order, nq, flux, prec, ctas, stream);
        else dispatch<MODE_STAGE>(a, t, order, nq, flux, prec, ctas, stream);
    }
}

void launch_residual(const StageArgs& a, const TileArgs& t, int order, int nq, int flux, int prec, int ctas,
                     cudaStream_t stream) {
    dispatch<MODE_RESIDUAL>(a, t, order, nq, flux, prec, ctas, stream);
}

void wait_selftest(double limit_s, int* timed_out, double* waited_s) {
    unsigned long long* d = nullptr;
    RKDG_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(unsigned long long)));
    unsigned long long h[2] = {0, 0};
    wait_selftest_kernel<<<1, 32>>>((uint64_t)(limit_s * 1e9), d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) throw Error{RKDG_ERR_CUDA, std::string("wait self-test: ") + cudaGetErrorString(e)};
    *timed_out = (int)h[0];
    *waited_s = (double)h[1] * 1e-9;
}

void launch_wave(const TileArgs& t, int ld, const void* U, int prec, const double* jinv,
                 double gamma, StepCtl* ctl, int nsolves, const double* refs, cudaStream_t stream) {
    if (nsolves > 0) reset_wave_kernel<<<(nsolves + 127) / 128, 128, 0, stream>>>(ctl, nsolves);
    if (t.ntiles > 0) {
        if (prec == RKDG_FP32)
            wave_kernel<float><<<t.ntiles, kAuxBlock, 0, stream>>>(t, ld, static_cast<const float*>(U), jinv, gamma, ctl, refs);
        else
            wave_kernel<double><<<t.ntiles, kAuxBlock, 0, stream>>>(t, ld, static_cast<const double*>(U), jinv, gamma, ctl, refs);
    }
    RKDG_CUDA_TRY(cudaGetLastError());
}

void launch_step_begin(StepCtl* ctl, int nsolves, cudaStream_t stream) {
    step_begin_kernel<<<(nsolves + 127) / 128, 128, 0, stream>>>(ctl, nsolves);
    RKDG_CUDA_TRY(cudaGetLastError());
}

namespace {
template <typename Real, int FLUX>
int occupancy_for(int order, int nq, int tile, int max_halo) {
    auto pick = [&](auto bt) -> int {
        constexpr int BT = decltype(bt)::value;
        if (order == 1) return occupancy_tiled<Real, 6, FLUX, MODE_STAGE, 1, BT>(max_halo);
        if (order == 3) return occupancy_tiled<Real, 6, FLUX, MODE_STAGE, 3, BT>(max_halo);
        if (nq == 7) return occupancy_tiled<Real, 7, FLUX, MODE_STAGE, 2, BT>(max_halo);
        return occupancy_tiled<Real, 6, FLUX, MODE_STAGE, 2, BT>(max_halo);
    };
    if (tile == 256) return pick(std::integral_constant<int, 256>{});
    return pick(std::integral_constant<int, 128>{});
}
}  // namespace

size_t tiled_smem_bytes(int prec, int order, int flux, int max_halo, int tile) {
    auto f = [&](auto r, auto bt) -> size_t {
        using Real = decltype(r);
        constexpr int BT = decltype(bt)::value;
        const bool h = flux == RKDG_FLUX_HLLC;
        if (order == 1)
            return h ? TiledSmem<Real, 1, RKDG_FLUX_HLLC, BT>::bytes(max_halo) : TiledSmem<Real, 1, RKDG_FLUX_LLF, BT>::bytes(max_halo);
        if (order == 2)
            return h ? TiledSmem<Real, 2, RKDG_FLUX_HLLC, BT>::bytes(max_halo) : TiledSmem<Real, 2, RKDG_FLUX_LLF, BT>::bytes(max_halo);
        return h ? TiledSmem<Real, 3, RKDG_FLUX_HLLC, BT>::bytes(max_halo) : TiledSmem<Real, 3, RKDG_FLUX_LLF, BT>::bytes(max_halo);
    };
    if (prec == RKDG_FP32)
        return tile == 256 ? f(0.0f, std::integral_constant<int, 256>{}) : f(0.0f, std::integral_constant<int, 128>{});
    return tile == 256 ? f(0.0, std::integral_constant<int, 256>{}) : f(0.0, std::integral_constant<int, 128>{});
}

bool tiled_fits(int prec, int order, int flux, int max_halo, int tile) {
    return tiled_smem_bytes(prec, order, flux, max_halo, tile) <= smem_limit();
}

int tiled_max_ctas_per_sm(int prec, int order, int nq, int flux, int max_halo, int tile) {
    const bool h = flux == RKDG_FLUX_HLLC;
    if (prec == RKDG_FP32)
        return h ? occupancy_for<float, RKDG_FLUX_HLLC>(order, nq, tile, max_halo)
                 : occupancy_for<float, RKDG_FLUX_LLF>(order, nq, tile, max_halo);
    return h ? occupancy_for<double, RKDG_FLUX_HLLC>(order, nq, tile, max_halo)
             : occupancy_for<double, RKDG_FLUX_LLF>(order, nq, tile, max_halo);
}

void launch_tiled_limiter(const TileArgs& t, int ctas, int ld, void* U, const int4* conn,
                          const void* lim, const double* jinv, const int* flags,
                          const double* refs, int prec, int nq2, double gamma, double tvb_m,
                          const StepCtl* ctl, int* tile_flags, int* tile_list, int tile_cap,
                          cudaStream_t stream) {
    const int cfg1 = cfg_index(3, 2), cfg2 = cfg_index(nq2, 3);
    if (tile_list != nullptr && tile_flags == nullptr)
        throw Error{RKDG_ERR_INVALID, "a limiter tile list needs its tile flags"};
    // one CTA per tile, or a persistent grid (the caller's, else four CTAs
    // per SM) over a tile list
    int grid = ctas > 0 ? ctas : std::max(1, t.ntiles);
    if (tile_list != nullptr && ctas <= 0) grid = std::max(1, std::min(t.ntiles, 4 * sm_count()));
    if (prec == RKDG_FP32)
        tiled_limiter_kernel<float><<<grid, kAuxBlock, 0, stream>>>(t, ld, static_cast<float*>(U), conn, lim, jinv, flags, refs, gamma, tvb_m, cfg1, cfg2, ctl, tile_flags, tile_list, tile_cap);
    else
        tiled_limiter_kernel<double><<<grid, kAuxBlock, 0, stream>>>(t, ld, static_cast<double*>(U), conn, lim, jinv, flags, refs, gamma, tvb_m, cfg1, cfg2, ctl, tile_flags, tile_list, tile_cap);
    RKDG_CUDA_TRY(cudaGetLastError());
}

void launch_rows(bool gather, void* U, int ld, int T, const int* idx, int n, int nrows, void* buf, int* err,
                 cudaStream_t stream) {
    const int total = n * nrows;
    if (total <= 0) return;
    const int grid = (total + 255) / 256;
    if (gather)
        gather_rows_kernel<<<grid, 256, 0, stream>>>(static_cast<const int4*>(U), ld, T, idx, n, nrows,
                                                      static_cast<int4*>(buf), err);
    else
        scatter_rows_kernel<<<grid, 256, 0, stream>>>(static_cast<int4*>(U), ld, T, idx, n, nrows,
                                                       static_cast<const int4*>(buf), err);
    RKDG_CUDA_TRY(cudaGetLastError());
}

void launch_import(int T, int ld, const double* staging, int ldh, const double* conv,
                   const int32_t* perm, void* U, int order, int prec, const double* ref, int lo_row,
                   cudaStream_t stream) {
    Ref4 r{{ref[0], ref[1], ref[2], ref[3]}};
    const int grid = (T + 127) / 128;
    if (prec == RKDG_FP32) {
        if (order == 1) import_kernel<float, 3><<<grid, 128, 0, stream>>>(T, ld, staging, ldh, conv, perm, static_cast<float*>(U), r, lo_row);
        else import_kernel<float, 6><<<grid, 128, 0, stream>>>(T, ld, staging, ldh, conv, perm, static_cast<float*>(U), r, lo_row);
    } else {
        if (order == 1) import_kernel<double, 3><<<grid, 128, 0, stream>>>(T, ld, staging, ldh, conv, perm, static_cast<double*>(U), r, -1);
        else import_kernel<double, 6><<<grid, 128, 0, stream>>>(T, ld, staging, ldh, conv, perm, static_cast<double*>(U), r, -1);
    }
    RKDG_CUDA_TRY(cudaGetLastError());
}

void launch_export(int T, int ld, const void* U, const double* conv, const int32_t* perm,
                   double* staging, int ldh, int order, int prec, int residual_scale,
                   const double* jinv, const double* ref, int lo_row, cudaStream_t stream) {
    Ref4 r{{ref[0], ref[1], ref[2], ref[3]}};
    const int grid = (T + 127) / 128;
    if (prec == RKDG_FP32) {
        if (order == 1) export_kernel<float, 3><<<grid, 128, 0, stream>>>(T, ld, static_cast<const float*>(U), conv, perm, staging, ldh, residual_scale, jinv, r, lo_row);
        else export_kernel<float, 6><<<grid, 128, 0, stream>>>(T, ld, static_cast<const float*>(U), conv, perm, staging, ldh, residual_scale, jinv, r, lo_row);
    } else {
        if (order == 1) export_kernel<double, 3><<<grid, 128, 0, stream>>>(T, ld, static_cast<const double*>(U), conv, perm, staging, ldh, residual_scale, jinv, r, -1);
        else export_kernel<double, 6><<<grid, 128, 0, stream>>>(T, ld, static_cast<const double*>(U), conv, perm, staging, ldh, residual_scale, jinv, r, -1);
    }
    RKDG_CUDA_TRY(cudaGetLastError());
}

void launch_totals(int T, int ld, const void* U, int order, int prec, const double* jinv,
                   double* partial, double* out4, const double* ref, int lo_row, cudaStream_t stream) {
    Ref4 r{{ref[0], ref[1], ref[2], ref[3]}};
    (void)order;
    const int n = totals_partial_count(T);
    if (prec == RKDG_FP32)
        totals_partial_kernel<float><<<n, kTotBlock, 0, stream>>>(T, ld, static_cast<const float*>(U), jinv, partial, r, lo_row);
    else
        totals_partial_kernel<double><<<n, kTotBlock, 0, stream>>>(T, ld, static_cast<const double*>(U), jinv, partial, r, -1);
    totals_final_kernel<<<1, kTotBlock, 0, stream>>>(n, partial, out4);
    RKDG_CUDA_TRY(cudaGetLastError());
}

}  // namespace rkdg
