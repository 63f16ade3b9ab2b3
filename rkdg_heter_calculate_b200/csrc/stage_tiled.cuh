// Tile-staged fused stage kernel (included by kernels.cu).
//
// A tile is up to kTile consecutive (locality-ordered) elements of one
// solve; its descriptor names the element range, the solve, the polynomial
// order, and its halo and flux-task ranges.  One CTA processes a tile:
//   phase A  each thread: its element's state, volume integral (registers),
//            traces at the 3*NG edge points and cell mean -> shared memory;
//            the CTA together: traces of the out-of-tile (halo) neighbours
//            on the shared edges -> shared memory.
//   phase B  the tile's flux tasks (each interior in-tile edge once, from
//            its lower-index side; every halo and boundary edge from the
//            in-tile side), spread evenly over the threads; the physical
//            flux (normal scaled by the edge length) overwrites the
//            computing side's trace slot.
//   phase C  each thread adds its three edges' fluxes (its own slot, or the
//            negated flux of the in-tile neighbour that computed it) to the
//            residual and applies the stage update.
// The kernel loops over tiles (tile = blockIdx.x + k * gridDim.x), so one
// launch serves a single solve (one CTA per tile) or a persistent pass over
// the packed tiles of many solves of uneven size and mixed order, each with
// its own dt, CFL measure and monitor.  A tile's arithmetic depends only on
// its own solve's data: results are deterministic and identical whether a
// solve runs alone or in a batch.

template <typename Real, int NQ2>
struct TiledSmem {
    // sized for the larger (P2, 3 edge points) layout; P1 tiles use a prefix
    static constexpr size_t bytes(int hm) {
        constexpr int NG = 3;
        return sizeof(double) * 5 * kTile +
               sizeof(Real) * ((size_t)3 * NG * 4 * kTile + 4 * kTile + (size_t)NG * 4 * hm + 4 * hm);
    }
};

// Resident CTAs per SM the register allocation is held to (FP64 P2 would
// otherwise take ~218 registers and leave 8 warps per SM).
template <typename Real, int ORD>
struct TiledOccupancy {
    static constexpr int value = sizeof(Real) == 8 ? (ORD == 1 ? 4 : 3) : (ORD == 1 ? 8 : 5);
};

template <typename Real, int NB, int NQ, int NG, int FLUX, int MODE>
__device__ __forceinline__ void tile_stage(const StageArgs& a, const TileArgs& ta, const int4 d0,
                                           const int4 d1, unsigned char* smem_raw) {
    constexpr int CFG = cfg_index(NQ, NG);
    constexpr int BT = kTile;
    const Tab<Real>& tb = tab<Real>(CFG);
    const int HM = ta.max_halo;
    double* s_jinv = reinterpret_cast<double*>(smem_raw);  // [4][BT]
    double* s_area2 = s_jinv + 4 * BT;                     // [BT] twice the area
    Real* s_tr = reinterpret_cast<Real*>(s_area2 + BT);    // [3][NG][4][BT]
    Real* s_mean = s_tr + 3 * NG * 4 * BT;                 // [4][BT]
    Real* s_htr = s_mean + 4 * BT;                         // [NG][4][HM]
    Real* s_hmean = s_htr + NG * 4 * HM;                   // [4][HM]
    __shared__ Real s_ephi[3][NG][NB];
    for (int x = threadIdx.x; x < 3 * NG * NB; x += BT) {
        int k = x / (NG * NB), g = (x / NB) % NG, i = x % NB;
        s_ephi[k][g][i] = tb.ephi[k][g][i];
    }
    const int sid = d0.z;
    StepCtl* ctl = a.ctl + sid;
    if (MODE == MODE_STAGE && ctl->done) return;  // uniform over the CTA

    const int tid = threadIdx.x;
    const int e0 = d0.x;
    const int e = e0 + tid;
    const bool active = tid < d0.y;
    const int ee = active ? e : e0;
    const Real* __restrict__ U = static_cast<const Real*>(a.U);
    const Real gamma = (Real)a.gamma, gm1 = gamma - Real(1);
    const double* fs = a.far_sid ? a.far_sid + 4 * sid : a.far;
    Real far[4] = {(Real)fs[0], (Real)fs[1], (Real)fs[2], (Real)fs[3]};

    // ------------------------------------------------------------ phase A
    Real R[NB][4];
    const double2* jinv2 = reinterpret_cast<const double2*>(a.jinv);
    const double2 r0 = __ldg(jinv2 + ee), r1 = __ldg(jinv2 + a.ld + ee);
    s_jinv[0 * BT + tid] = r0.x;
    s_jinv[1 * BT + tid] = r0.y;
    s_jinv[2 * BT + tid] = r1.x;
    s_jinv[3 * BT + tid] = r1.y;
    s_area2[tid] = 1.0 / (r0.x * r1.y - r0.y * r1.x);  // 2 * area
    {
        Real u[NB][4];
        load_state<Real, NB>(U, a.ld, ee, u);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            u[0][v] += ref_of<Real>(fs, v);  // stored deviation -> state (FP32)
            s_mean[v * BT + tid] = u[0][v];
        }
#pragma unroll
        for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) R[i][v] = Real(0);
        const Real j00 = (Real)r0.x, j01 = (Real)r0.y, j10 = (Real)r1.x, j11 = (Real)r1.y;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            Real w[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Real s = Real(0);
#pragma unroll
                for (int i = 0; i < NB; ++i) s += tb.vphi[q][i] * u[i][v];
                w[v] = s;
            }
            Real ri = rcp_(w[0]);
            Real vx = w[1] * ri, vy = w[2] * ri;
            Real p = gm1 * (w[3] - Real(0.5) * (w[1] * vx + w[2] * vy));
            Real F[4] = {w[1], w[1] * vx + p, w[2] * vx, (w[3] + p) * vx};
            Real G[4] = {w[2], w[1] * vy, w[2] * vy + p, (w[3] + p) * vy};
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Real fx = j00 * F[v] + j01 * G[v];
                Real fy = j10 * F[v] + j11 * G[v];
#pragma unroll
                for (int i = 1; i < NB; ++i) R[i][v] += fx * tb.vdxi[q][i] + fy * tb.veta[q][i];
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int g = 0; g < NG; ++g)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    Real s = Real(0);
#pragma unroll
                    for (int i = 0; i < NB; ++i) s += tb.ephi[k][g][i] * u[i][v];
                    s_tr[((k * NG + g) * 4 + v) * BT + tid] = s;
                }
    }
    __syncthreads();  // s_ephi visible below; own traces complete
    {
        const int h0 = d1.x, nh = d1.y;
        for (int h = tid; h < nh; h += BT) {
            const int2 hh = __ldg(ta.halo + h0 + h);
            Real un[NB][4];
            load_state<Real, NB>(U, a.ld, hh.x, un);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                un[0][v] += ref_of<Real>(fs, v);
                s_hmean[v * HM + h] = un[0][v];
            }
#pragma unroll
            for (int g = 0; g < NG; ++g)
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    Real s = Real(0);
#pragma unroll
                    for (int i = 0; i < NB; ++i) s += s_ephi[hh.y][g][i] * un[i][v];
                    s_htr[(g * 4 + v) * HM + h] = s;
                }
        }
    }
    __syncthreads();

    // ------------------------------------------------------------ phase B
    {
        const int t0 = d1.z, nt = d1.w;
        for (int j = tid; j < nt; j += BT) {
            const int tk = __ldg(ta.task + t0 + j);
            const int le = tk >> 2, k = tk & 3;
            const int c = __ldg(&ta.code[e0 + le].x + k);
            const int kind = c & 3, se = (c >> 2) & 3, idx = c >> 4;
            // physical normal N = n * length of edge k of element le from the
            // FP64 J^-1 and area (N_k / area = 2(r0 + r1), -2 r0, -2 r1);
            // its length and direction in the working precision
            const double a0 = s_jinv[0 * BT + le], a1 = s_jinv[1 * BT + le];
            const double b0 = s_jinv[2 * BT + le], b1 = s_jinv[3 * BT + le];
            const double area2 = s_area2[le];
            double Nxd, Nyd;
            if (k == 0) {
                Nxd = (a0 + b0) * area2;
                Nyd = (a1 + b1) * area2;
            } else if (k == 1) {
                Nxd = -a0 * area2;
                Nyd = -a1 * area2;
            } else {
                Nxd = -b0 * area2;
                Nyd = -b1 * area2;
            }
            const Real Nx = (Real)Nxd, Ny = (Real)Nyd;
            const Real len = sqrt_(Nx * Nx + Ny * Ny);
            const Real il = rcp_(len);
            const Real nx = Nx * il, ny = Ny * il;
            Real mL[4], mR[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) mL[v] = s_mean[v * BT + le];
            if (kind == EDGE_IN_OWNER) {
#pragma unroll
                for (int v = 0; v < 4; ++v) mR[v] = s_mean[v * BT + idx];
            } else if (kind == EDGE_HALO) {
#pragma unroll
                for (int v = 0; v < 4; ++v) mR[v] = s_hmean[v * HM + idx];
            } else {
                ghost<Real>(se, mL, far, nx, ny, mR);
            }
            Real alpha = Real(0);
            if (FLUX == RKDG_FLUX_LLF) {
                // LLF coefficient from the average of the two cell means
                // (src/kernelfunctions.cu:370-387), scaled by the edge length
                Real rho = Real(0.5) * (mL[0] + mR[0]);
                Real ir = rcp_(rho);
                Real vx = Real(0.5) * (mL[1] + mR[1]) * ir;
                Real vy = Real(0.5) * (mL[2] + mR[2]) * ir;
                Real E = Real(0.5) * (mL[3] + mR[3]);
                Real p = gm1 * (E - Real(0.5) * rho * (vx * vx + vy * vy));
                alpha = fabs(vx * Nx + vy * Ny) + sqrt_(gamma * p * ir) * len;
            }
#pragma unroll
            for (int g = 0; g < NG; ++g) {
                Real uL[4], uR[4];
                Real* slot = s_tr + (k * NG + g) * 4 * BT + le;
#pragma unroll
                for (int v = 0; v < 4; ++v) uL[v] = slot[v * BT];
                // the neighbour's point NG-1-g on its edge se pairs with ours
                // (src/kernelfunctions.cu:545-549)
                if (kind == EDGE_IN_OWNER) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) uR[v] = s_tr[((se * NG + NG - 1 - g) * 4 + v) * BT + idx];
                } else if (kind == EDGE_HALO) {
#pragma unroll
                    for (int v = 0; v < 4; ++v) uR[v] = s_htr[((NG - 1 - g) * 4 + v) * HM + idx];
                } else {
                    ghost<Real>(se, uL, far, nx, ny, uR);
                }
                Real fh[4];
                if (FLUX == RKDG_FLUX_LLF) {
                    Real fL[4], fR[4], pL, pR;
                    normal_flux<Real>(uL, Nx, Ny, gm1, fL, pL);
                    normal_flux<Real>(uR, Nx, Ny, gm1, fR, pR);
#pragma unroll
                    for (int v = 0; v < 4; ++v) fh[v] = Real(0.5) * (fL[v] + fR[v] - alpha * (uR[v] - uL[v]));
                } else {
                    hllc<Real>(uL, uR, nx, ny, gamma, fh);
#pragma unroll
                    for (int v = 0; v < 4; ++v) fh[v] *= len;
                }
#pragma unroll
                for (int v = 0; v < 4; ++v) slot[v * BT] = fh[v];
            }
        }
    }
    __syncthreads();

    // ------------------------------------------------------------ phase C
    const int4 cd = __ldg(ta.code + ee);
    const Real inv_area = (Real)(2.0 / s_area2[tid]);  // 1 / area
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int c = k == 0 ? cd.x : (k == 1 ? cd.y : cd.z);
        const int kind = c & 3, se = (c >> 2) & 3, idx = c >> 4;
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            Real f[4];
            if (kind == EDGE_IN_OTHER) {
#pragma unroll
                for (int v = 0; v < 4; ++v) f[v] = -s_tr[((se * NG + NG - 1 - g) * 4 + v) * BT + idx];
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) f[v] = s_tr[((k * NG + g) * 4 + v) * BT + tid];
            }
            const Real wg = tb.ew[g] * inv_area;
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Real cw = wg * f[v];
#pragma unroll
                for (int i = 0; i < NB; ++i) R[i][v] -= cw * tb.ephi[k][g][i];
            }
        }
    }

    Real* __restrict__ Uout = static_cast<Real*>(a.Unew);
    if (MODE == MODE_RESIDUAL) {
        if (active) store_state<Real, NB>(Uout, a.ld, e, R);
        return;
    }
    const double dtd = ctl->dt;
    const Real dt = (Real)dtd, ca = (Real)a.a, cb = (Real)a.b;
    Real u0m[4] = {Real(0), Real(0), Real(0), Real(0)};
    {
        Real u[NB][4];
        load_state<Real, NB>(U, a.ld, ee, u);  // stored values (L1/L2 hit: read in phase A)
        if (a.U0 != nullptr) {
            Real u0[NB][4];
            load_state<Real, NB>(static_cast<const Real*>(a.U0), a.ld, ee, u0);
#pragma unroll
            for (int i = 0; i < NB; ++i)
#pragma unroll
                for (int v = 0; v < 4; ++v) R[i][v] = ca * u0[i][v] + cb * (u[i][v] + dt * R[i][v]);
#pragma unroll
            for (int v = 0; v < 4; ++v) u0m[v] = u0[0][v];
        } else {
#pragma unroll
            for (int i = 0; i < NB; ++i)
#pragma unroll
                for (int v = 0; v < 4; ++v) R[i][v] = cb * (u[i][v] + dt * R[i][v]);
        }
    }
    if (active) store_state<Real, NB>(Uout, a.ld, e, R);
    if (a.last_stage) {
        double wv = 0.0, m0 = 0.0, m1 = 0.0;
        if (active) {
            bool bad;
            wv = wave_measure((double)R[0][0] + (double)ref_of<Real>(fs, 0),
                              (double)R[0][1] + (double)ref_of<Real>(fs, 1),
                              (double)R[0][2] + (double)ref_of<Real>(fs, 2),
                              (double)R[0][3] + (double)ref_of<Real>(fs, 3), a.gamma, r0, r1, bad);
            if (bad) atomicOr(&ctl->error, 1);
            m0 = fabs((double)R[0][0] - (double)u0m[0]);
            m1 = fabs((double)R[0][3] - (double)u0m[3]);
        }
        block_max3_atomic(wv, m0, m1, &ctl->wave_bits, &ctl->mon_bits[0], &ctl->mon_bits[1]);
    }
}

// ORD: 1 = P1 tiles only, 2 = P2 tiles only, 3 = both (dispatch per tile;
// P2 tiles use the NQ2-point volume rule, P1 tiles the 3/2-point rules).
template <typename Real, int NQ2, int FLUX, int MODE, int ORD>
__global__ void __launch_bounds__(kTile, TiledOccupancy<Real, ORD>::value)
    tiled_stage_kernel(const StageArgs a, const TileArgs ta) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ntiles = ta.ntiles_dev ? *ta.ntiles_dev : ta.ntiles;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int4 d0 = __ldg(ta.desc + 2 * tile), d1 = __ldg(ta.desc + 2 * tile + 1);
        if (ORD == 2 || (ORD == 3 && d0.w == 2))
            tile_stage<Real, 6, NQ2, 3, FLUX, MODE>(a, ta, d0, d1, smem_raw);
        else
            tile_stage<Real, 3, 3, 2, FLUX, MODE>(a, ta, d0, d1, smem_raw);
        __syncthreads();  // shared memory is reused by the next tile
    }
}
