// Tile-staged fused stage kernel (included by kernels.cu).
//
// A tile is up to BT consecutive (locality-ordered) elements of one
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
//
// Staging pipeline: a tile's own state rows are contiguous 16-byte rows in
// HBM (pack p of element e at (p ld + e) 16), so one thread moves them into
// shared memory with bulk asynchronous copies (cp.async.bulk, completion
// counted in bytes on an mbarrier).  The copies for the CTA's next tile are
// issued once the current tile's halo traces are formed, and run under its
// flux and update work; the next tile's J^-1, edge-code and U^n rows and its
// halo and task lists are prefetched into L2 at the same time.

// ------------------------------------------------------------- staging --
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// 16-byte asynchronous gather into shared memory (completion per thread).
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Orders this thread's earlier generic-proxy shared-memory accesses before
// later asynchronous-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the barrier phase of the given parity; gives up after limit_ns
// nanoseconds (two seconds for the stage kernel's staging waits) or 2^26
// polls, returning false.
constexpr uint64_t kStageWaitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = kStageWaitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 1; it < (1u << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0 && global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// Self-test of the bounded wait: one thread arms an mbarrier for 16 bytes
// that no copy ever delivers and waits on it with the given limit; out[0] =
// 1 if the wait gave up, out[1] = nanoseconds waited.  Nothing is in flight
// when it returns.
__global__ void wait_selftest_kernel(uint64_t limit_ns, unsigned long long* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_expect_tx(&bar, 16);
    const uint64_t t0 = global_ns();
    const bool ok = mbar_wait(&bar, 0, limit_ns);
    out[0] = ok ? 0ull : 1ull;
    out[1] = global_ns() - t0;
}

// Shared memory of one CTA: the work area (edge normals, edge codes, flux
// tasks, own traces and means, as 4-vectors), sized for the largest tile
// layout the kernel dispatches (P1 tiles of a mixed pack use a prefix),
// then the staging area.  The staging area first receives the tile's own
// state rows by bulk copy (SROWS rows of 16 bytes per element); once phase A
// has read them, the halo neighbours' states by 16-byte gathers ([SROWS][hm]
// rows).  Each halo thread then overwrites its own neighbour's first rows
// with that neighbour's traces (and mean: put_htr), which phase B reads, and
// the next tile's rows are copied in after phase B.  This keeps an FP32 CTA
// within the shared memory of six per SM (P2) and an FP64 one within that of
// three (P2) or four (P1).  J^-1 and the edge codes are read per thread (L2
// hits, prefetched with the rows) while the rows arrive.
template <typename Real>
struct alignas(16) Vec4 {
    Real x, y, z, w;
};
template <typename Real>
__device__ __forceinline__ void put4(Vec4<Real>* p, const Real a[4]) {
    Vec4<Real> t;
    t.x = a[0], t.y = a[1], t.z = a[2], t.w = a[3];
    *p = t;
}
template <typename Real>
__device__ __forceinline__ void get4(const Vec4<Real>* p, Real a[4]) {
    const Vec4<Real> t = *p;
    a[0] = t.x, a[1] = t.y, a[2] = t.z, a[3] = t.w;
}
// Per-element linear algebra on 4-vectors (the conservative components).
// FP32 runs it in lane pairs (components 0-1 and 2-3) with the f32x2
// helpers and the paired tables; FP64 runs the scalar form.  (Pairing the
// two sides of the HLLC flux the same way executed fewer instructions but
// more register moves and ran slower.)
__device__ __forceinline__ float2 lo2(const float a[4]) { return make_float2(a[0], a[1]); }
__device__ __forceinline__ float2 hi2(const float a[4]) { return make_float2(a[2], a[3]); }
__device__ __forceinline__ void set4(float a[4], float2 l, float2 h) { a[0] = l.x, a[1] = l.y, a[2] = h.x, a[3] = h.y; }
// out = c + sum_{i >= 1} tab[i] u_i
template <int NB>
__device__ __forceinline__ void comb_rows(const float2* tab, const float u[NB][4], float2 cl, float2 ch,
                                          float out[4]) {
#pragma unroll
    for (int i = 1; i < NB; ++i) {
        cl = f2fma(tab[i], lo2(u[i]), cl);
        ch = f2fma(tab[i], hi2(u[i]), ch);
    }
    set4(out, cl, ch);
}
// R_i += f tab[i] for i >= I0
template <int I0, int NB>
__device__ __forceinline__ void acc_rows(float R[NB][4], const float f[4], const float2* tab) {
    const float2 fl = lo2(f), fh = hi2(f);
#pragma unroll
    for (int i = I0; i < NB; ++i) set4(R[i], f2fma(fl, tab[i], lo2(R[i])), f2fma(fh, tab[i], hi2(R[i])));
}

template <typename Real, int BT>
struct TiledLayout {
    // edge normals per element: (Nx, Ny) per edge, the length formed where
    // used (as it was formed when stored: the same bits); this keeps an FP64
    // P2 CTA with the LLF means within the shared memory of three per SM
    static constexpr int NC = 2;
    static constexpr size_t code_off = (sizeof(Real) * 3 * NC * BT + 15) / 16 * 16;
};

// Cell means (own and halo) are kept only where the LLF coefficient needs
// them.
template <typename Real, int ORD, int FLUX, int BT>
struct TiledSmem {
    static constexpr int NG = ORD == 1 ? 2 : 3;
    static constexpr int SROWS = (ORD == 1 ? 3 : 6) * (int)(sizeof(Real) / 4);
    static constexpr int MEANS = FLUX == RKDG_FLUX_LLF ? 1 : 0;
    __host__ __device__ static constexpr size_t work(int) {
        return TiledLayout<Real, BT>::code_off + sizeof(int4) * BT + sizeof(uint16_t) * 3 * BT +
               sizeof(Vec4<Real>) * ((size_t)3 * NG * BT + MEANS * BT);
    }
    __host__ __device__ static constexpr size_t stage_offset(int hm) { return (work(hm) + 127) / 128 * 128; }
    __host__ __device__ static constexpr size_t stage_rows(int hm) {
        return (size_t)SROWS * (BT > hm ? BT : hm);
    }
    __host__ __device__ static constexpr size_t bytes(int hm) { return stage_offset(hm) + stage_rows(hm) * 16; }
};

// Resident CTAs per SM the register allocation is held to: in FP32 24 warps
// per SM for kernels with P2 tiles (80 registers; 128-element tiles at most
// 37 KB of shared memory per CTA) and 32 for P1-only kernels (64 registers;
// their tiles need about 27 KB, and the extra warps hide more of the tile
// pipeline's latency: 11 % faster on the limited Mach-3 step); in FP64 12
// (P2: 168 registers, about 100 B of spills per thread, 17 % faster than
// 8 warps at 236 registers on large meshes) and 16 (P1: 128 registers);
// whatever the tile size.  LAT (FP64 only): 8 and 12 warps without spills,
// for launches whose tiles all fit on the device at once, where a tile's
// latency rather than the throughput of many sets the time.
template <typename Real, int ORD, int BT, int LAT = 0>
struct TiledOccupancy {
    static constexpr int warps = sizeof(Real) == 8 ? (LAT ? (ORD == 1 ? 12 : 8) : (ORD == 1 ? 16 : 12))
                                                   : (ORD == 1 ? 32 : 24);
    static constexpr int value = warps * 32 / BT > 0 ? warps * 32 / BT : 1;
};

// Issues the bulk copies of tile d's state rows into the staging area (one
// thread; completion counted on bar).
template <typename Real, int BT>
__device__ __forceinline__ void stage_copy(const StageArgs& a, const int4 d, unsigned char* stg, uint64_t* bar) {
    const int rows = (d.w == 2 ? 6 : 3) * (int)(sizeof(Real) / 4);
    const uint32_t rb = (uint32_t)d.y * 16u;
    mbar_expect_tx(bar, rb * (uint32_t)rows);
    const char* U = static_cast<const char*>(a.U);
    for (int r = 0; r < rows; ++r)
        bulk_g2s(stg + (size_t)r * BT * 16, U + ((size_t)r * a.ld + d.x) * 16, rb, bar);
}
// L2 prefetches of tile d's J^-1 and edge-code rows, U^n rows, the rows of
// the means' low parts (RKDG_FP32C) and halo and task lists, and with STATE
// its state rows (one thread; the tables are padded so that the 16-byte
// rounding stays inside them).
template <typename Real, bool STATE>
__device__ __forceinline__ void stage_prefetch(const StageArgs& a, const TileArgs& ta, const int4 d,
                                               const int4 dd) {
    const int rows = (d.w == 2 ? 6 : 3) * (int)(sizeof(Real) / 4);
    const uint32_t rb = (uint32_t)d.y * 16u;
    if constexpr (STATE) {
        const char* U = static_cast<const char*>(a.U);
        for (int r = 0; r < rows; ++r) bulk_prefetch_l2(U + ((size_t)r * a.ld + d.x) * 16, rb);
    }
    const char* J = reinterpret_cast<const char*>(a.jinv);
    bulk_prefetch_l2(J + (size_t)d.x * 16, rb);
    bulk_prefetch_l2(J + ((size_t)a.ld + d.x) * 16, rb);
    bulk_prefetch_l2(ta.code + d.x, rb);
    if (a.U0 != nullptr) {
        const char* U0 = static_cast<const char*>(a.U0);
        for (int r = 0; r < rows; ++r) bulk_prefetch_l2(U0 + ((size_t)r * a.ld + d.x) * 16, rb);
    }
    if (a.lo_row >= 0) {  // RKDG_FP32C: the low parts of the means, read by the update
        const size_t lo = ((size_t)a.lo_row * a.ld + d.x) * 16;
        bulk_prefetch_l2(static_cast<const char*>(a.U) + lo, rb);
        if (a.U0 != nullptr) bulk_prefetch_l2(static_cast<const char*>(a.U0) + lo, rb);
    }
    if (dd.y > 0) {
        const uintptr_t b = reinterpret_cast<uintptr_t>(ta.halo + dd.x) & ~uintptr_t(15);
        const uintptr_t e = (reinterpret_cast<uintptr_t>(ta.halo + dd.x + dd.y) + 15) & ~uintptr_t(15);
        bulk_prefetch_l2(reinterpret_cast<const void*>(b), (uint32_t)(e - b));
    }
    if (dd.w > 0) {
        const uintptr_t b = reinterpret_cast<uintptr_t>(ta.task + dd.z) & ~uintptr_t(15);
        const uintptr_t e = (reinterpret_cast<uintptr_t>(ta.task + dd.z + dd.w) + 15) & ~uintptr_t(15);
        bulk_prefetch_l2(reinterpret_cast<const void*>(b), (uint32_t)(e - b));
    }
}

// A halo neighbour's trace (slot g < NG) or cell mean (slot NG) in the
// staging area, over that neighbour's own staged state rows (entry h of the
// [rows][HM] gather): FP32 one 16-byte row per slot (row g), FP64 two (rows
// 2g and 2g + 1).  Each halo thread writes only its own entry, after it has
// read the rows there.
template <typename Real>
__device__ __forceinline__ void put_htr(unsigned char* stg, int HM, int g, int h, const Real t[4]) {
    if constexpr (sizeof(Real) == 8) {
        double2* p = reinterpret_cast<double2*>(stg);
        p[(2 * g) * HM + h] = make_double2(t[0], t[1]);
        p[(2 * g + 1) * HM + h] = make_double2(t[2], t[3]);
    } else {
        reinterpret_cast<float4*>(stg)[g * HM + h] = make_float4(t[0], t[1], t[2], t[3]);
    }
}
template <typename Real>
__device__ __forceinline__ void get_htr(const unsigned char* stg, int HM, int g, int h, Real t[4]) {
    if constexpr (sizeof(Real) == 8) {
        const double2* p = reinterpret_cast<const double2*>(stg);
        const double2 a = p[(2 * g) * HM + h], b = p[(2 * g + 1) * HM + h];
        t[0] = a.x, t[1] = a.y, t[2] = b.x, t[3] = b.y;
    } else {
        const float4 a = reinterpret_cast<const float4*>(stg)[g * HM + h];
        t[0] = a.x, t[1] = a.y, t[2] = a.z, t[3] = a.w;
    }
}

// Element x's state from the staging rows.
template <typename Real, int NB, int BT>
__device__ __forceinline__ void load_staged(const unsigned char* stg, int x, Real u[NB][4]) {
    if constexpr (sizeof(Real) == 8) {
        const double2* p = reinterpret_cast<const double2*>(stg);
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            const double2 a = p[(2 * i) * BT + x], b = p[(2 * i + 1) * BT + x];
            u[i][0] = a.x;
            u[i][1] = a.y;
            u[i][2] = b.x;
            u[i][3] = b.y;
        }
    } else {
        const float4* p = reinterpret_cast<const float4*>(stg);
#pragma unroll
        for (int i = 0; i < NB; ++i) {
            const float4 a = p[i * BT + x];
            u[i][0] = a.x;
            u[i][1] = a.y;
            u[i][2] = a.z;
            u[i][3] = a.w;
        }
    }
}

// The part of a tile's work that needs only its descriptors, J^-1 rows and
// edge codes: edge normals and codes into shared memory, the solve's
// reference state, the halo and task list entries.  Formed while the tile's
// state rows are still in flight.
template <typename Real>
struct TilePre {
    RefState<Real> rs;
    Real inv_area, j00, j01, j10, j11;  // 1 / area; rows of 2 area J^-1
    double det;                         // det J^-1 = 1 / (2 area)
    int2 hh[3];
};
template <typename Real, int BT>
__device__ __forceinline__ TilePre<Real> tile_pre(const StageArgs& a, const TileArgs& ta, const int4 d0,
                                                  const int4 d1, const double2 r0, const double2 r1,
                                                  const int4 code, unsigned char* smem_raw) {
    constexpr int NC = TiledLayout<Real, BT>::NC;
    const int tid = threadIdx.x;
    TilePre<Real> t;
    // far-field / reference state by value (a pointer into the parameter
    // block would put the parameter array in local memory)
    double fs[4];
    if (a.far_sid) {
        const double* p = a.far_sid + 4 * d0.z;
        fs[0] = p[0], fs[1] = p[1], fs[2] = p[2], fs[3] = p[3];
    } else {
        fs[0] = a.far[0], fs[1] = a.far[1], fs[2] = a.far[2], fs[3] = a.far[3];
    }
    t.rs = ref_state<Real>(fs, a.gamma);
    // the halo and task lists (L2 hits: prefetched with the tile's rows)
    const int h0 = d1.x, nh = d1.y, t0 = d1.z, nt = d1.w;
    int4* s_code = reinterpret_cast<int4*>(smem_raw + TiledLayout<Real, BT>::code_off);  // [BT]
    uint16_t* s_task = reinterpret_cast<uint16_t*>(s_code + BT);                         // [3 BT]
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const int h = tid + r * BT;
        t.hh[r] = h < nh ? __ldg(ta.halo + h0 + h) : make_int2(0, 0);
        // the flux tasks straight into the work area (not the staging area)
        if (h < nt) s_task[h] = __ldg(ta.task + t0 + h);
    }
    s_code[tid] = code;
    // edge normals N_k (length = edge length; N_k / area = 2(r0 + r1), -2 r0,
    // -2 r1) from the FP64 J^-1 rows, kept in the working precision.  The
    // residual is accumulated scaled by 2 area (= 1 / det J^-1): the volume
    // term through 2 area J^-1 = (-N_1; -N_2), the surface term through the
    // table 2 w_g psi_i, and the factor det J^-1 applied once in the update.
    Real* s_nrm = reinterpret_cast<Real*>(smem_raw);  // [3][NC][BT] Nx, Ny
    t.det = r0.x * r1.y - r0.y * r1.x;
    t.inv_area = (Real)(2.0 * t.det);
    // FP64 forms them in FP64; FP32 from the rounded J^-1 rows (a few ulp,
    // without the FP64 reciprocal)
    const Real area2 = rcp_((Real)t.det);
    const Real ax = (Real)r0.x, ay = (Real)r0.y, bx = (Real)r1.x, by = (Real)r1.y;
    const Real cx[3] = {ax + bx, -ax, -bx}, cy[3] = {ay + by, -ay, -by};
    Real Nx[3], Ny[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Nx[k] = cx[k] * area2, Ny[k] = cy[k] * area2;
        s_nrm[(NC * k + 0) * BT + tid] = Nx[k];
        s_nrm[(NC * k + 1) * BT + tid] = Ny[k];
    }
    t.j00 = -Nx[1], t.j01 = -Ny[1], t.j10 = -Nx[2], t.j11 = -Ny[2];
    return t;
}

// Returns, when the stage is followed by the TVB limiter (a.tile_flags set),
// whether the limiter may change this thread's element (tvb_keeps fails).
template <typename Real, int NB, int NQ, int NG, int FLUX, int MODE, int BT>
__device__ __forceinline__ bool tile_stage(const StageArgs& a, const TileArgs& ta, const int4 d0,
                                           const int4 d1, unsigned char* smem_raw, unsigned char* stg,
                                           const int nxt, const int ntiles, uint64_t* bar,
                                           const TilePre<Real>& pre, Real (*s_red)[3], const double* s_dt) {
    constexpr int CFG = cfg_index(NQ, NG);
    using V4 = Vec4<Real>;
    const Tab<Real>& tb = tab<Real>(CFG);
    const int HM = ta.max_halo;
    constexpr int NC = TiledLayout<Real, BT>::NC;
    Real* s_nrm = reinterpret_cast<Real*>(smem_raw);                       // [3][NC][BT] Nx, Ny
    int4* s_code = reinterpret_cast<int4*>(smem_raw + TiledLayout<Real, BT>::code_off);  // [BT]
    uint16_t* s_task = reinterpret_cast<uint16_t*>(s_code + BT);           // [3 BT] flux tasks
    V4* s_tr = reinterpret_cast<V4*>(s_task + 3 * BT);                     // [3][NG][BT] own traces
    constexpr int MEANS = FLUX == RKDG_FLUX_LLF ? 1 : 0;                   // LLF needs cell means
    V4* s_mean = s_tr + 3 * NG * BT;                                       // [BT] (LLF)
    // halo traces and means: in the staging rows, over each neighbour's own
    // staged state (put_htr / get_htr; FP32 also through these pointers,
    // trace g of halo h in row g, entry h)
    V4* s_htr = reinterpret_cast<V4*>(stg);
    V4* s_hmean = s_htr + NG * HM;
    constexpr bool PK = sizeof(Real) == 4;  // FP32: lane-pair arithmetic, paired tables
    const Tab2& t2 = c_tab_f2[CFG];
    using SE = typename std::conditional<PK, float2, Real>::type;
    __shared__ SE s_ephi[3][NG][NB];  // neighbour-side edge table (runtime edge index)
    for (int x = threadIdx.x; x < 3 * NG * NB; x += BT) {
        int k = x / (NG * NB), g = (x / NB) % NG, i = x % NB;
        if constexpr (PK) s_ephi[k][g][i] = t2.ephi[k][g][i];
        else s_ephi[k][g][i] = tb.ephi[k][g][i];
    }
    const int sid = d0.z;
    StepCtl* ctl = a.ctl + sid;

    const int tid = threadIdx.x;
    const int e0 = d0.x;
    const int e = e0 + tid;
    const bool active = tid < d0.y;
    const int ee = active ? e : e0;
    const int sx = active ? tid : 0;  // staging row index
    const Real* __restrict__ U = static_cast<const Real*>(a.U);
    const Real gamma = (Real)a.gamma, gm1 = gamma - Real(1);
    // FP32: traces and fluxes in deviation form about the reference state
    constexpr bool DEV = stores_deviation<Real>();
    const RefState<Real> rs = pre.rs;
    const Real far[4] = {rs.rho, rs.mx, rs.my, rs.E};
    Real refv[4];  // the offset of a stored mean (FP32: the far field)
#pragma unroll
    for (int v = 0; v < 4; ++v) refv[v] = DEV ? far[v] : Real(0);

    // ------------------------------------------------------------ phase A
    constexpr int SR = NB * (int)(sizeof(Real) / 4);  // 16-byte rows of a state
    const int nh = d1.y, nt = d1.w;
    const int2* hh = pre.hh;
    Real R[NB][4];
    Real u[NB][4];
    const double det = pre.det;
    const Real inv_area = pre.inv_area;
    const Real j00 = pre.j00, j01 = pre.j01, j10 = pre.j10, j11 = pre.j11;  // rows of 2 area J^-1
    // psi_0 is the constant K00 at every volume and edge point: its term is
    // formed once per state
    const Real k00 = tb.vphi[0][0];
    {
        load_staged<Real, NB, BT>(stg, sx, u);
        __syncthreads();  // staged rows consumed: the area takes the halo states
        {
            const char* Ub = static_cast<const char*>(a.U);
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const int h = tid + r * BT;
                if (h < nh) {
#pragma unroll
                    for (int q = 0; q < SR; ++q)
                        cp_async16(stg + ((size_t)q * HM + h) * 16, Ub + ((size_t)q * a.ld + hh[r].x) * 16);
                }
            }
        }
        {
            Real mfull[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                mfull[v] = u[0][v] + refv[v];  // the cell mean itself
                if constexpr (!DEV) u[0][v] = mfull[v];
            }
            if constexpr (MEANS) put4(s_mean + tid, mfull);
        }
#pragma unroll
        for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) R[i][v] = Real(0);
        Real c0[4];
        if constexpr (PK) {
            const float2 kk = make_float2(k00, k00);
            set4(c0, f2mul(kk, lo2(u[0])), f2mul(kk, hi2(u[0])));
        } else {
#pragma unroll
            for (int v = 0; v < 4; ++v) c0[v] = k00 * u[0][v];
        }
        // FP32: the quadrature loop is unrolled by two only (a smaller body
        // keeps the instruction cache warm across the CTAs on an SM; full
        // unrolling is 2 % slower, none 1 %); FP64 unrolls it.  Each product
        // is its own fused multiply-add, and psi_1 (a function of xi alone)
        // has no eta-derivative term.
        constexpr int VOL_UNROLL = sizeof(Real) == 4 ? 2 : NQ;
#pragma unroll VOL_UNROLL
        for (int q = 0; q < NQ; ++q) {
            Real w[4];
            if constexpr (PK) {
                comb_rows<NB>(t2.vphi[q], u, lo2(c0), hi2(c0), w);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    Real s = c0[v];
#pragma unroll
                    for (int i = 1; i < NB; ++i) s += tb.vphi[q][i] * u[i][v];
                    w[v] = s;
                }
            }
            Real fx[4], fy[4];
            if constexpr (DEV) {
                // flux deviations through the rows of 2 area J^-1
                const DevPrims<Real> pw = dev_prims(w, rs, gm1);
                dev_flux(w, pw, rs, j00, j01, fx);
                dev_flux(w, pw, rs, j10, j11, fy);
            } else {
                Real ri = rcp_(w[0]);
                Real vx = w[1] * ri, vy = w[2] * ri;
                Real p = gm1 * (w[3] - Real(0.5) * (w[1] * vx + w[2] * vy));
                Real F[4] = {w[1], w[1] * vx + p, w[2] * vx, (w[3] + p) * vx};
                Real G[4] = {w[2], w[1] * vy, w[2] * vy + p, (w[3] + p) * vy};
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    fx[v] = j00 * F[v] + j01 * G[v];
                    fy[v] = j10 * F[v] + j11 * G[v];
                }
            }
            if constexpr (PK) {
                acc_rows<1, NB>(R, fx, t2.vdxi[q]);
                acc_rows<2, NB>(R, fy, t2.veta[q]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) {
#pragma unroll
                    for (int i = 1; i < NB; ++i) R[i][v] += fx[v] * tb.vdxi[q][i];
#pragma unroll
                    for (int i = 2; i < NB; ++i) R[i][v] += fy[v] * tb.veta[q][i];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int g = 0; g < NG; ++g) {
                Real t[4];
                if constexpr (PK) {
                    comb_rows<NB>(t2.ephi[k][g], u, lo2(c0), hi2(c0), t);
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        Real s = c0[v];
#pragma unroll
                        for (int i = 1; i < NB; ++i) s += tb.ephi[k][g][i] * u[i][v];
                        t[v] = s;
                    }
                }
                put4(s_tr + (k * NG + g) * BT + tid, t);
            }
    }
    cp_async_wait_all();
    __syncthreads();  // s_ephi visible below; own traces complete; halo states landed
    {
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            const int h = tid + r * BT;
            if (h < nh) {
                Real un[NB][4];
                if constexpr (sizeof(Real) == 8) {
                    const double2* p = reinterpret_cast<const double2*>(stg);
#pragma unroll
                    for (int i = 0; i < NB; ++i) {
                        const double2 x = p[(2 * i) * HM + h], y = p[(2 * i + 1) * HM + h];
                        un[i][0] = x.x, un[i][1] = x.y, un[i][2] = y.x, un[i][3] = y.y;
                    }
                } else {
                    const float4* p = reinterpret_cast<const float4*>(stg);
#pragma unroll
                    for (int i = 0; i < NB; ++i) {
                        const float4 x = p[i * HM + h];
                        un[i][0] = x.x, un[i][1] = x.y, un[i][2] = x.z, un[i][3] = x.w;
                    }
                }
                {
                    Real mfull[4];
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        mfull[v] = un[0][v] + refv[v];
                        if constexpr (!DEV) un[0][v] = mfull[v];
                    }
                    if constexpr (MEANS) put_htr<Real>(stg, HM, NG, h, mfull);
                }
                const int he = hh[r].y;
                Real c0[4];
                if constexpr (PK) {
                    const float2 kk = make_float2(k00, k00);
                    set4(c0, f2mul(kk, lo2(un[0])), f2mul(kk, hi2(un[0])));
                } else {
#pragma unroll
                    for (int v = 0; v < 4; ++v) c0[v] = k00 * un[0][v];
                }
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    Real t[4];
                    if constexpr (PK) {
                        comb_rows<NB>(s_ephi[he][g], un, lo2(c0), hi2(c0), t);
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            Real s = c0[v];
#pragma unroll
                            for (int i = 1; i < NB; ++i) s += s_ephi[he][g][i] * un[i][v];
                            t[v] = s;
                        }
                    }
                    put_htr<Real>(stg, HM, g, h, t);
                }
            }
        }
    }
    __syncthreads();  // halo traces complete
    int4 nd0 = make_int4(0, 0, 0, 0);
    if (tid == 0 && nxt < ntiles) {  // the CTA's next tile (only this thread reads its descriptor)
        nd0 = __ldg(ta.desc + 2 * nxt);
        stage_prefetch<Real, true>(a, ta, nd0, __ldg(ta.desc + 2 * nxt + 1));
    }

    // ------------------------------------------------------------ phase B
    {
        for (int j = tid; j < nt; j += BT) {
            const int tkj = s_task[j];
            const int le = tkj >> 2, k = tkj & 3;
            const int c = reinterpret_cast<const int*>(s_code + le)[k];
            const int kind = c & 3, se = (c >> 2) & 3, idx = c >> 4;
            // physical normal N (|N| = edge length) and unit normal of edge k
            const Real Nx = s_nrm[(NC * k + 0) * BT + le], Ny = s_nrm[(NC * k + 1) * BT + le];
            const Real len = sqrt_(Nx * Nx + Ny * Ny);
            const Real il = rcp_(len);
            const Real nx = Nx * il, ny = Ny * il;
            Real mL[4], mR[4];
            if constexpr (MEANS) {
                get4(s_mean + le, mL);
                if (kind == EDGE_BOUNDARY) ghost<Real>(se, mL, far, nx, ny, mR);
                else if constexpr (sizeof(Real) == 4) get4(kind == EDGE_HALO ? s_hmean + idx : s_mean + idx, mR);
                else if (kind == EDGE_HALO) get_htr<Real>(stg, HM, NG, idx, mR);
                else get4(s_mean + idx, mR);
            }
            Real alpha = Real(0);
            if constexpr (FLUX == RKDG_FLUX_LLF) {
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
                V4* slot = s_tr + (k * NG + g) * BT + le;
                get4(slot, uL);
                // the neighbour's point NG-1-g on its edge se pairs with ours
                // (src/kernelfunctions.cu:545-549)
                V4* nslot = sizeof(Real) == 4 && kind == EDGE_HALO ? s_htr + (NG - 1 - g) * HM + idx
                                                                   : s_tr + (se * NG + NG - 1 - g) * BT + idx;
                if (kind == EDGE_BOUNDARY) {
                    if constexpr (DEV) ghost_dev<Real>(se, uL, rs, nx, ny, uR);
                    else ghost<Real>(se, uL, far, nx, ny, uR);
                }
                else if (sizeof(Real) == 8 && kind == EDGE_HALO) get_htr<Real>(stg, HM, NG - 1 - g, idx, uR);
                else get4(nslot, uR);
                Real fh[4], fn[4];  // the flux out of this side and into the neighbour
                if (FLUX == RKDG_FLUX_LLF) {
                    Real fL[4], fR[4];
                    if constexpr (DEV) {
                        dev_flux(uL, dev_prims(uL, rs, gm1), rs, Nx, Ny, fL);
                        dev_flux(uR, dev_prims(uR, rs, gm1), rs, Nx, Ny, fR);
                    } else {
                        Real pL, pR;
                        normal_flux<Real>(uL, Nx, Ny, gm1, fL, pL);
                        normal_flux<Real>(uR, Nx, Ny, gm1, fR, pR);
                    }
                    if constexpr (PK) {
                        const float2 na = make_float2(-alpha, -alpha);
                        const float2 tl = f2fma(na, f2sub(lo2(uR), lo2(uL)), f2add(lo2(fL), lo2(fR)));
                        const float2 th = f2fma(na, f2sub(hi2(uR), hi2(uL)), f2add(hi2(fL), hi2(fR)));
                        const float2 hp = make_float2(0.5f, 0.5f), hn = make_float2(-0.5f, -0.5f);
                        set4(fh, f2mul(hp, tl), f2mul(hp, th));
                        set4(fn, f2mul(hn, tl), f2mul(hn, th));
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            const Real t = fL[v] + fR[v] - alpha * (uR[v] - uL[v]);
                            fh[v] = Real(0.5) * t;
                            fn[v] = Real(-0.5) * t;
                        }
                    }
                } else {
                    Real f[4];
                    if constexpr (DEV) hllc_dev<Real>(uL, uR, nx, ny, gamma, rs, f);
                    else hllc<Real>(uL, uR, nx, ny, gamma, f);
                    if constexpr (PK) {
                        const float2 l = make_float2(len, len), nl = make_float2(-len, -len);
                        set4(fh, f2mul(lo2(f), l), f2mul(hi2(f), l));
                        set4(fn, f2mul(lo2(f), nl), f2mul(hi2(f), nl));
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            fh[v] = f[v] * len;
                            fn[v] = f[v] * -len;
                        }
                    }
                }
                // each slot of an edge is read by this task alone: the
                // computing side's slot takes the flux, an in-tile
                // neighbour's slot its negation
                put4(slot, fh);
                if (kind == EDGE_IN_OWNER) put4(nslot, fn);
            }
        }
    }
    __syncthreads();  // fluxes complete, halo traces read: the staging area takes the next tile's rows
    if (tid == 0 && nxt < ntiles) {
        fence_proxy_async();
        stage_copy<Real, BT>(a, nd0, stg, bar);
    }

    // ------------------------------------------------------------ phase C
    // every own slot now holds the outward flux of its edge point
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int g = 0; g < NG; ++g) {
            Real f[4];
            get4(s_tr + (k * NG + g) * BT + tid, f);
            if constexpr (PK) {
                acc_rows<0, NB>(R, f, t2.nephiw[k][g]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v)
#pragma unroll
                    for (int i = 0; i < NB; ++i) R[i][v] -= f[v] * tb.ephiw[k][g][i];
            }
        }

    Real* __restrict__ Uout = static_cast<Real*>(a.Unew);
    if (MODE == MODE_RESIDUAL) {
        const Real sc = (Real)det;
#pragma unroll
        for (int i = 0; i < NB; ++i)
#pragma unroll
            for (int v = 0; v < 4; ++v) R[i][v] *= sc;
        if (active) store_state<Real, NB>(Uout, a.ld, e, R);
        return false;
    }
    const double dtd = *s_dt;
    // a U^n + b (U + dt L) as U^n + b ((U - U^n) + dt L): a + b = 1 holds
    // exactly (1/3 and 2/3 both round up in FP32, and a scale of 1 + 3e-8
    // per step would accumulate into the state); L = det J^-1 R
    const Real dt = (Real)(dtd * det), cb = (Real)a.b;
    Real u0m[4] = {Real(0), Real(0), Real(0), Real(0)};
    // RKDG_FP32C (comp): row 0 is updated in FP64 below, not here
    constexpr bool comp = PK && (MODE & MODE_STAGE_COMP);
    {
        load_state<Real, NB>(U, a.ld, ee, u);  // stored values (L2 hit)
        if (a.U0 != nullptr) {
            Real u0[NB][4];
            load_state<Real, NB>(static_cast<const Real*>(a.U0), a.ld, ee, u0);
            if constexpr (PK) {
                const float2 dt2 = make_float2(dt, dt), cb2 = make_float2(cb, cb);
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    const float2 l = f2fma(cb2, f2fma(dt2, lo2(R[i]), f2sub(lo2(u[i]), lo2(u0[i]))), lo2(u0[i]));
                    const float2 h = f2fma(cb2, f2fma(dt2, hi2(R[i]), f2sub(hi2(u[i]), hi2(u0[i]))), hi2(u0[i]));
                    if (i > 0 || !comp) set4(R[i], l, h);
                }
            } else {
#pragma unroll
                for (int i = 0; i < NB; ++i)
#pragma unroll
                    for (int v = 0; v < 4; ++v) R[i][v] = u0[i][v] + cb * ((u[i][v] - u0[i][v]) + dt * R[i][v]);
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) u0m[v] = u0[0][v];
        } else {
            if constexpr (PK) {
                const float2 dt2 = make_float2(dt, dt), cb2 = make_float2(cb, cb);
#pragma unroll
                for (int i = 0; i < NB; ++i) {
                    const float2 l = f2mul(cb2, f2fma(dt2, lo2(R[i]), lo2(u[i])));
                    const float2 h = f2mul(cb2, f2fma(dt2, hi2(R[i]), hi2(u[i])));
                    if (i > 0 || !comp) set4(R[i], l, h);
                }
            } else {
#pragma unroll
                for (int i = 0; i < NB; ++i)
#pragma unroll
                    for (int v = 0; v < 4; ++v) R[i][v] = cb * (u[i][v] + dt * R[i][v]);
            }
        }
    }
    if constexpr (comp) {
        // RKDG_FP32C: the cell mean is the unevaluated sum of its stored high
        // part (row 0) and low part (row lo_row).  Rows 1.. are stored as
        // updated above; R[0] still holds the mean's residual, and the
        // mean's update runs in FP64 from both parts, split again into a
        // high and a low float, so the mean's storage rounding does not
        // accumulate over the stages.
        if (active) store_rows<Real, 1, NB>(Uout, a.ld, e, R);
        const size_t lr = (size_t)a.lo_row * a.ld;
        // the high parts: the stage input's and U^n's row 0 as loaded for
        // the update above (U^n's is zero in a first stage)
        const float4 h = make_float4(u[0][0], u[0][1], u[0][2], u[0][3]);
        const float4 h0 = make_float4(u0m[0], u0m[1], u0m[2], u0m[3]);
        const float4 l = __ldg(reinterpret_cast<const float4*>(a.U) + lr + ee);
        float4 l0 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a.U0 != nullptr) l0 = __ldg(reinterpret_cast<const float4*>(a.U0) + lr + ee);
        const double dtdet = dtd * det;
        const float hv[4] = {h.x, h.y, h.z, h.w}, lv[4] = {l.x, l.y, l.z, l.w};
        const float h0v[4] = {h0.x, h0.y, h0.z, h0.w}, l0v[4] = {l0.x, l0.y, l0.z, l0.w};
        float nl[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const double m = (double)hv[v] + (double)lv[v], m0 = (double)h0v[v] + (double)l0v[v];
            const double y = m0 + a.b * ((m - m0) + dtdet * (double)R[0][v]);
            const float yh = (float)y;
            R[0][v] = yh;
            nl[v] = (float)(y - (double)yh);
        }
        if (active) {
            reinterpret_cast<float4*>(a.Unew)[e] = make_float4(R[0][0], R[0][1], R[0][2], R[0][3]);
            reinterpret_cast<float4*>(a.Unew)[lr + e] = make_float4(nl[0], nl[1], nl[2], nl[3]);
        }
    } else {
        if (active) store_state<Real, NB>(Uout, a.ld, e, R);
    }
    if (a.last_stage) {
        // CFL wave maximum (and the residual monitor when asked) of the new
        // state: a max over each warp in the working precision into s_red;
        // after the tile's closing barrier one thread takes the max over the
        // warps and makes one atomic per tile on the solve's control block
        // (a solve's atomics meet at one address, so their number is kept
        // small)
        Real wv = Real(0), m0 = Real(0), m1 = Real(0);
        if (active) {
            bool bad;
            Real m[4], len[3];
#pragma unroll
            for (int v = 0; v < 4; ++v) m[v] = R[0][v] + refv[v];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const Real Nx = s_nrm[(NC * k + 0) * BT + tid], Ny = s_nrm[(NC * k + 1) * BT + tid];
                len[k] = sqrt_(Nx * Nx + Ny * Ny);
            }
            wv = (Real)wave_of<Real>(m, gamma, len, inv_area, bad);
            if (bad) atomicOr(&ctl->error, 1);
            if (a.monitor) {
                m0 = fabs(R[0][0] - u0m[0]);
                m1 = fabs(R[0][3] - u0m[3]);
            }
        }
        wv = warp_max(wv);
        if (a.monitor) {
            m0 = warp_max(m0);
            m1 = warp_max(m1);
        }
        if ((tid & 31) == 0) {
            s_red[tid >> 5][0] = wv;
            s_red[tid >> 5][1] = m0;
            s_red[tid >> 5][2] = m1;
        }
    }
    bool need = false;
    if constexpr (MODE & MODE_LIMITED) {
      if (active && (a.limiter_on == nullptr || a.limiter_on[sid])) {
        // the limiter's exact test on the new state (its P1 part at the edge
        // midpoints, the mean, the TVB thresholds from the rows of 2 area
        // J^-1: the columns of J are (j11, -j10) and (-j01, j00))
        Real mean[4], tmax = Real(0);
#pragma unroll
        for (int v = 0; v < 4; ++v) mean[v] = R[0][v] + refv[v];
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int v = 0; v < 4; ++v) tmax = fmax(tmax, fabs(tb.mphi[k][0] * R[1][v] + tb.mphi[k][1] * R[2][v]));
        Real dirx[3], diry[3], thr[3];
        tvb_geometry<Real>(j11, -j10, -j01, j00, (Real)a.tvb_m, dirx, diry, thr);
        need = !tvb_keeps<Real>(mean, gamma, tmax, fmin(fmin(thr[0], thr[1]), thr[2]));
      }
    }
    return need;
}

// The tile's maxima from s_red into its solve's control block (one thread,
// after the barrier that closes the tile; bits of a non-negative double
// order like the values).
template <typename Real, int BT>
__device__ __forceinline__ void tile_maxima_atomic(const StageArgs& a, StepCtl* ctl, const Real (*s_red)[3]) {
    Real w = s_red[0][0], m0 = s_red[0][1], m1 = s_red[0][2];
#pragma unroll
    for (int k = 1; k < BT / 32; ++k) {
        w = fmax(w, s_red[k][0]);
        m0 = fmax(m0, s_red[k][1]);
        m1 = fmax(m1, s_red[k][2]);
    }
    atomicMax(&ctl->wave_bits, (unsigned long long)__double_as_longlong((double)w));
    if (a.monitor) {
        atomicMax(&ctl->mon_bits[0], (unsigned long long)__double_as_longlong((double)m0));
        atomicMax(&ctl->mon_bits[1], (unsigned long long)__double_as_longlong((double)m1));
    }
}

// ORD: 1 = P1 tiles only, 2 = P2 tiles only, 3 = both (dispatch per tile;
// P2 tiles use the NQ2-point volume rule, P1 tiles the 3/2-point rules).
// BT: elements per tile = threads per CTA.
// A barrier wait that times out sets bit 1 of the solve's error word and
// ends the CTA (all threads together).
template <typename Real, int NQ2, int FLUX, int MODE, int ORD, int BT, int LAT = 0>
__global__ void __launch_bounds__(BT, TiledOccupancy<Real, ORD, BT, LAT>::value)
    tiled_stage_kernel(const StageArgs a, const TileArgs ta) {
    using SM = TiledSmem<Real, ORD, FLUX, BT>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t s_bar;
    __shared__ Real s_red[BT / 32][3];  // per-warp maxima of a last stage
    __shared__ double s_dt;             // the tile's solve's dt (read before the staging wait)
    unsigned char* stg = smem_raw + SM::stage_offset(ta.max_halo);
    const int ntiles = ta.ntiles_dev ? *ta.ntiles_dev : ta.ntiles;
    int tile = blockIdx.x;
    if (tile >= ntiles) return;
    if (threadIdx.x == 0) mbar_init(&s_bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int4 fd = __ldg(ta.desc + 2 * tile);
        stage_copy<Real, BT>(a, fd, stg, &s_bar);
        // the first tile's table prefetch: a gain for FP64 (measured at two
        // CTAs per SM), a loss for FP32
        if constexpr (sizeof(Real) == 8) stage_prefetch<Real, false>(a, ta, fd, __ldg(ta.desc + 2 * tile + 1));
    }
    const double2* jinv2 = reinterpret_cast<const double2*>(a.jinv);
    uint32_t parity = 0;
    for (; tile < ntiles; tile += gridDim.x) {
        const int4 d0 = __ldg(ta.desc + 2 * tile), d1 = __ldg(ta.desc + 2 * tile + 1);
        const int nxt = tile + gridDim.x;
        // this thread's J^-1 rows and edge codes, and the work that needs
        // only them, while the state rows arrive
        const int ex = d0.x + ((int)threadIdx.x < d0.y ? (int)threadIdx.x : 0);
        const double2 r0 = __ldg(jinv2 + ex), r1 = __ldg(jinv2 + a.ld + ex);
        const int4 code = __ldg(ta.code + ex);
        const int done = MODE != MODE_RESIDUAL ? a.ctl[d0.z].done : 0;
        if (MODE != MODE_RESIDUAL && threadIdx.x == 0) s_dt = a.ctl[d0.z].dt;
        const TilePre<Real> pre = tile_pre<Real, BT>(a, ta, d0, d1, r0, r1, code, smem_raw);
        const bool ok = mbar_wait(&s_bar, parity);
        if (__syncthreads_or(!ok)) {  // also: every thread has seen this phase complete
            if (threadIdx.x == 0) atomicOr(&a.ctl[d0.z].error, 2);
            return;
        }
        parity ^= 1u;
        if (done) {  // finished solve: pass the tile on
            if (threadIdx.x == 0 && nxt < ntiles) stage_copy<Real, BT>(a, __ldg(ta.desc + 2 * nxt), stg, &s_bar);
            continue;
        }
        bool need;
        if (ORD == 2 || (ORD == 3 && d0.w == 2))
            need = tile_stage<Real, 6, NQ2, 3, FLUX, MODE, BT>(a, ta, d0, d1, smem_raw, stg, nxt, ntiles, &s_bar, pre,
                                                              s_red, &s_dt);
        else
            need = tile_stage<Real, 3, 3, 2, FLUX, MODE, BT>(a, ta, d0, d1, smem_raw, stg, nxt, ntiles, &s_bar, pre,
                                                            s_red, &s_dt);
        // shared memory is reused by the next tile (with the limiter the
        // barrier also ORs its test over the tile)
        if constexpr (MODE & MODE_LIMITED) {
            const int any = __syncthreads_or(need);
            if (threadIdx.x == 0 && any && atomicExch(a.tile_flags + tile, 1) == 0) {
                const int slot = atomicAdd(a.tile_list, 1);
                if (slot < a.tile_cap) a.tile_list[kListHead + slot] = tile;
            }
        } else {
            __syncthreads();
        }
        if (MODE != MODE_RESIDUAL && a.last_stage && threadIdx.x == 0)
            tile_maxima_atomic<Real, BT>(a, a.ctl + d0.z, s_red);
    }
}
