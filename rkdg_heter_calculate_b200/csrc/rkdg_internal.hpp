// Internal declarations shared by the host C++ and CUDA translation units of
// librkdg.so.  Nothing here crosses the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "rkdg.h"

namespace rkdg {

constexpr int kMaxNB = 6;   // P2
constexpr int kMaxNQ = 7;   // degree-5 volume rule
constexpr int kMaxNG = 3;   // 3-point Gauss-Legendre per edge

// ---------------------------------------------------------------- errors --
void set_error(const std::string& msg);
struct Error {
    int code;
    std::string msg;
};
// A failed call's error is also taken off the runtime's per-thread last
// error (cudaGetLastError), so that a non-sticky error reported here is not
// reported again by a later, unrelated check.
#define RKDG_CUDA_TRY(expr)                                                              \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            cudaGetLastError();                                                          \
            throw ::rkdg::Error{RKDG_ERR_CUDA, std::string(#expr) + ": " +               \
                                                   cudaGetErrorString(e_)};              \
        }                                                                                \
    } while (0)

// ----------------------------------------------------------- quadrature --
// Reference-element tables of the native basis (orthonormal under the area
// average on the triangle (0,0),(1,0),(0,1), hierarchical: the first 3
// functions span P1).  Volume points carry their normalised weight folded
// into the gradient tables.
struct RuleTables {
    // volume: value and weighted gradients, [q][i]
    double vphi[kMaxNQ][kMaxNB];
    double vdxi_w[kMaxNQ][kMaxNB];
    double veta_w[kMaxNQ][kMaxNB];
    double vw[kMaxNQ];
    // edges: value at point g of edge k, [k][g][i]; normalised weights [g]
    double ephi[3][kMaxNG][kMaxNB];
    double ew[kMaxNG];
    // P1 part at the three edge midpoints [k][1..2] and its least-squares
    // inverse (2 x 3) for the limiter
    double mphi[3][2];
    double minv[2][3];
};

void volume_rule(int nq, double l[][3], double* w);
void edge_rule(int ng, double* s, double* w);
// native basis: coefficients on monomials 1, xi, eta, xi^2, xi*eta, eta^2
const double (*native_coeff())[6];
void native_eval(int nbasis, double xi, double eta, double* val, double* dxi, double* deta);
RuleTables make_tables(int nq, int ng);

// ------------------------------------------------------------- geometry --
// Per-element FP64 quantities computed on the host once.
struct HostGeometry {
    std::vector<double> jinv;   // [T][4]: rows of J^-1, (r0x, r0y, r1x, r1y)
    std::vector<double> area;   // [T]
    std::vector<double> conv_in;   // [T][6][6] native <- reference: b_j = sum_i a_i C[i][j]
    std::vector<double> conv_out;  // [T][6][6] reference <- native: a_i = sum_j b_j D[i][j]
    std::vector<double> lim;       // [T][3][2] limiter (alpha, beta) per edge (see kernels)
    std::vector<uint8_t> lim_pair; // [T] bit k: edge k pairs with edge (k+2)%3, else (k+1)%3
};

// ------------------------------------------------------------------ mesh --
struct HostMesh {
    int T = 0;
    std::vector<double> xy;       // [T][3][2] per-triangle vertex coordinates
    std::vector<int32_t> nbr;     // [T][3]
    std::vector<int8_t> bc;       // [T][3]
    std::vector<int8_t> shared;   // [T][3] neighbour-local edge index (or -1)
    std::vector<int32_t> perm;    // internal index -> caller index
    std::vector<int32_t> tri_vertex;  // [T][3] caller's vertex ids (output only)
    std::vector<double> vertices;     // [V][2] caller's vertices (output only)
};

// Builds HostMesh from the C descriptor in caller order; validates it.
HostMesh build_mesh(const rkdg_mesh_desc& d);
// Morton order of the centroids; returns perm (new -> old).
std::vector<int32_t> morton_order(const HostMesh& m);
HostMesh permute_mesh(const HostMesh& m, const std::vector<int32_t>& perm);
HostGeometry build_geometry(const HostMesh& m, int order, bool with_conversion, bool with_limiter);
// Packed connectivity word: bits 0-5 shared edge (2 bits per edge),
// bits 6-11 boundary tag (2 bits per edge), bits 12-14 the limiter's edge
// pairing (HostGeometry::lim_pair).
uint32_t pack_info(const int8_t* shared3, const int8_t* bc3, uint32_t lim_pair = 0);
// The limiter table on the device: rows k = 0..2 of (alpha, beta) per
// element, double2 (prec RKDG_FP64) or float2 (RKDG_FP32), row k of element
// e at index k ld + e; uploads elements [e0, e0 + T) from lim [T][3][2] and
// waits for the copy.
void upload_limiter(void* dev, int ld, int64_t e0, const std::vector<double>& lim, int T, int prec,
                    cudaStream_t stream);

// ---------------------------------------------------------------- tiles --
// Work decomposition of the tile-staged stage kernel: a CTA owns kTile
// consecutive (locality-ordered) elements.  For every element edge k a code
// says where the trace across it comes from:
//   bits 0-1 kind: 0 in-tile neighbour, this side computes the flux (lower index)
//                  1 in-tile neighbour, the other side computes it
//                  2 out-of-tile (halo) neighbour, this side computes
//                  3 boundary edge, this side computes
//   bits 2-3 neighbour-local edge (kinds 0-2) or boundary tag (kind 3)
//   bits 4.. local index of the in-tile neighbour, or the halo slot
constexpr int kTile = 128;
// Bytes added to the halo and task tables so that the stage kernel's L2
// prefetch of a tile's list, rounded out to 16-byte boundaries, stays inside.
constexpr size_t kTablePad = 64;
enum { EDGE_IN_OWNER = 0, EDGE_IN_OTHER = 1, EDGE_HALO = 2, EDGE_BOUNDARY = 3 };

// Tiles of one solve.  Element indices are global in the packed element
// space (elem_offset + local), halo and task ranges index pool arrays at the
// given offsets, so the tables of many solves concatenate.
// desc per tile (8 ints): e0, count, solve id, order, halo_begin, nhalo,
// task_begin, ntask.
struct TileTables {
    int tile = kTile;                  // elements per tile
    int ntiles = 0;
    int max_halo = 0;                  // rounded up to a multiple of 4
    std::vector<int32_t> code;         // [T][4] (code of edges 0..2, unused)
    std::vector<int32_t> desc;         // [ntiles][8]
    std::vector<int32_t> halo;         // [nhalo][2] (global element, its edge)
    std::vector<uint16_t> task;        // local element * 4 + edge, sorted by edge
};
// n_tiled >= 0: only elements [0, n_tiled) are tiled (a partition's owned
// elements; the rest are halo copies that other tiles read as neighbours).
TileTables build_tiles(const HostMesh& m, int elem_offset = 0, int sid = 0, int order = 2,
                       int halo_offset = 0, int task_offset = 0, int n_tiled = -1, int tile = kTile);

// ------------------------------------------------------------- device --
struct StepCtl {
    double t;                  // simulated time after the last step
    double t_final;            // <= 0: no final time
    double dt;                 // dt of the current step
    double dt_fixed;           // > 0: use this dt instead of the CFL one
    double cfl;
    unsigned long long wave_bits;   // max (|u|+c) perimeter/area of the state, as bits
    unsigned long long mon_bits[2]; // residual monitor, as bits
    int step;
    int done;
    int error;                 // bit 0: non-physical state seen; bit 1: a device wait timed out;
                               // bit 2: a halo-exchange row index out of range
    int pad;
};

// Throws the error a solve's control word reports (no-op when clean).
inline void throw_ctl_error(int error, const std::string& who) {
    if (error & 4) throw Error{RKDG_ERR_INVALID, who + ": a row index given to a halo exchange is out of range"};
    if (error & 2) throw Error{RKDG_ERR_CUDA, who + ": a device-side wait on staged data timed out"};
    if (error) throw Error{RKDG_ERR_STATE, who + ": non-physical state (NaN or non-positive density/pressure)"};
}

struct DeviceArrays {
    void* U[3] = {nullptr, nullptr, nullptr};  // state buffers (A holds U^n)
    double* jinv = nullptr;     // [2][ld][2]
    int4* conn = nullptr;       // [ld]
    void* lim = nullptr;        // [3][ld] (alpha, beta) of the limiter (when enabled)
    int* tile_flags = nullptr;  // [ntiles] the stage kernel's per-tile limiter test (when enabled)
    int* tile_list = nullptr;   // [2 + ntiles] the tiles the limiter must visit (LimitList)
    int32_t* perm = nullptr;    // [T]
    double* conv_in = nullptr;  // [T][36]
    double* conv_out = nullptr; // [T][36]
    double* staging = nullptr;  // [4][6][T] dense FP64 host-layout staging
    double* partial = nullptr;  // block partial sums for deterministic totals
    StepCtl* ctl = nullptr;
    double* far = nullptr;      // [4] far-field / reference state (device copy)
    // tile tables
    int4* tcode = nullptr;
    int4* tdesc = nullptr;
    int2* halo = nullptr;
    uint16_t* task = nullptr;
    size_t bytes = 0;
};

// The tiles a stage's TVB limiter must visit, built by the stage kernel:
// int[2 + cap] = {count, CTAs done, tile ids...}.  A tile whose limiter test
// fails (tvb_keeps false for an element) sets its flag (tile_flags, 0 -> 1)
// and appends itself once; the limiter visits the listed tiles, clears their
// flags, and its last CTA to finish resets count and done, so every flag is
// 0 and the list empty when the next stage starts.
constexpr int kListHead = 2;

struct TileArgs {
    const int4* code;   // [elements] per-edge source codes
    const int4* desc;   // [ntiles][2] tile descriptors
    const int2* halo;   // halo pool
    const uint16_t* task;  // task pool
    int max_halo;
    int ntiles;
    const int* ntiles_dev;  // when set, kernels read the tile count here (graph-stable)
    int tile = kTile;       // elements per tile (threads per CTA of the stage kernel): 128 or 256
};

struct StageArgs {
    int T, ld;
    const void* U;       // stage input
    const void* U0;      // U^n (may equal nullptr when a == 0)
    void* Unew;          // stage output (residual output in residual mode)
    const double* jinv;
    const int4* conn;
    StepCtl* ctl;
    double a, b;         // Unew = a U0 + b (U + dt L(U)), formed as U0 + b ((U - U0) + dt L); a = 1 - b
    double gamma;
    double far[4];
    const double* far_sid;  // per-solve far-field states [solves][4], or nullptr
    int last_stage;      // compute wave max / error (and the monitor when asked) in the epilogue
    int monitor;         // last stage: also form the residual monitor max |d mean| (rho, rhoE)
    int lo_row;          // RKDG_FP32C: state row of the cell means' low parts (in U, U0, Unew), else -1
    int* tile_flags;     // with the TVB limiter: per tile of the launch, 1 while the tile is in tile_list
    int* tile_list;      // with tile_flags: the LimitList the stage appends its limiter-changeable tiles to
    int tile_cap;        // entries of tile_list
    const int* limiter_on;  // per solve: the test is made only for solves with the limiter (null: all)
    double tvb_m;        // the TVB constant of that test
};

// Arithmetic type of the kernels for a precision setting: RKDG_FP32C runs
// the FP32 kernels (its extra cell-mean row is read and written in the
// stage update only).
inline int kernel_prec(int precision) { return precision == RKDG_FP64 ? RKDG_FP64 : RKDG_FP32; }
// 16-byte state rows per element: FP64 two per basis function, FP32 one,
// FP32C one plus the row of the cell means' low parts.
inline int state_rows(int precision, int nb) {
    return precision == RKDG_FP64 ? 2 * nb : (precision == RKDG_FP32C ? nb + 1 : nb);
}

// Launchers (kernels.cu).  All asynchronous on `stream`.  `prec` is the
// arithmetic type of a kernel (RKDG_FP64 or RKDG_FP32; kernel_prec maps the
// RKDG_FP32C setting to RKDG_FP32).
void upload_tables(int nq, int ng);
// The tile-staged stage kernel: one CTA per tile of kTile elements (each
// interior flux once per tile, traces shared in shared memory), `ctas` CTAs
// per launch looping over the tiles (0 = one CTA per tile).  `order` 1 or 2,
// or 3 for a pack of P1 and P2 tiles (P2 tiles use nq, P1 tiles the
// 3/2-point rules).
void launch_stage(const StageArgs& a, const TileArgs& t, int order, int nq, int flux, int prec, int ctas,
                  cudaStream_t stream);
void launch_residual(const StageArgs& a, const TileArgs& t, int order, int nq, int flux, int prec, int ctas,
                     cudaStream_t stream);
// CFL measure per solve, one CTA per tile (resets the wave slots of solves
// 0..nsolves-1 first; nsolves 0 leaves them as they are)
// FP32 states store cell means as deviations from a per-solve reference
// state (the far field); `refs` ([solves][4], device) / `ref` (4, host) give it.
void launch_wave(const TileArgs& t, int ld, const void* U, int prec, const double* jinv,
                 double gamma, StepCtl* ctl, int nsolves, const double* refs, cudaStream_t stream);
void launch_step_begin(StepCtl* ctl, int nsolves, cudaStream_t stream);
// bounded device wait on data that never arrives (see rkdg_wait_selftest)
void wait_selftest(double limit_s, int* timed_out, double* waited_s);
// dynamic shared memory per CTA of the tiled stage kernel for a tile size
// and halo list length (order 3: mixed pack); the launchers refuse a
// configuration above the device's per-CTA limit with RKDG_ERR_INVALID
size_t tiled_smem_bytes(int prec, int order, int flux, int max_halo, int tile);
bool tiled_fits(int prec, int order, int flux, int max_halo, int tile);
// resident CTAs per SM of the tiled stage kernel (order 3: mixed pack) for
// tiles of `tile` elements
int tiled_max_ctas_per_sm(int prec, int order, int nq, int flux, int max_halo, int tile = kTile);
int sm_count();  // SMs of the current device
// TVB limiter over tiles; flags[solve] (may be null: all on) enables it per
// solve, solves whose control block (ctl may be null) says done are skipped,
// and tiles whose tile_flags entry (may be null) is 0 -- the stage kernel
// that wrote the state found the limiter would change none of their
// elements -- are skipped; ctas 0 = one CTA per tile
void launch_tiled_limiter(const TileArgs& t, int ctas, int ld, void* U, const int4* conn,
                          const void* lim, const double* jinv, const int* flags,
                          const double* refs, int prec, int nq2, double gamma, double tvb_m,
                          const StepCtl* ctl, int* tile_flags, int* tile_list, int tile_cap,
                          cudaStream_t stream);
// Caller layout [4][nb][ldh] FP64 <-> HBM state packs.  lo_row >= 0: the
// state is RKDG_FP32C and row lo_row holds the low part of each cell mean
// (import splits the FP64 mean into high and low floats, export and the
// totals add them back).
void launch_import(int T, int ld, const double* staging, int ldh, const double* conv,
                   const int32_t* perm, void* U, int order, int prec, const double* ref, int lo_row,
                   cudaStream_t stream);
void launch_export(int T, int ld, const void* U, const double* conv, const int32_t* perm,
                   double* staging, int ldh, int order, int prec, int residual_scale,
                   const double* jinv, const double* ref, int lo_row, cudaStream_t stream);
void launch_totals(int T, int ld, const void* U, int order, int prec, const double* jinv,
                   double* partial, double* out4, const double* ref, int lo_row, cudaStream_t stream);
int totals_partial_count(int T);
// Halo exchange of a partition: rows 0..nrows-1 of elements idx[0..n) of U
// to (gather) or from (scatter) buf [n][nrows] 16-byte packs; bad indices
// set bit 2 of *err.
void launch_rows(bool gather, void* U, int ld, int T, const int* idx, int n, int nrows, void* buf, int* err,
                 cudaStream_t stream);

}  // namespace rkdg
