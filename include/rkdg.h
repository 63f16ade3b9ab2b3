/*
 * rkdg.h -- C ABI of librkdg.so, the B200 (sm_100a) RKDG residual and
 * time-step path for the 2D Euler equations on unstructured triangles.
 *
 * Every entry point is plain C: pointers, sizes and status codes; nothing
 * throws across the boundary.  Each function returns RKDG_OK (0) or an
 * error code; rkdg_last_error() gives the message of the calling thread's
 * last failure.  Contexts share no global state, so different contexts may
 * be driven from different host threads.
 *
 * Data layout at the boundary is the reference's (multi_gpuRkdg/):
 *   - DOFs and residuals are four SoA blocks freedom_{rho,rhou,rhov,rhoE},
 *     each [basis i][cell] with leading dimension ld >= ntri, i.e. the host
 *     array is [var][basis][ld] (src/cudarkdgsolver.cu:253-264, 336-339);
 *   - "reference basis" is the reference's per-element orthogonal basis,
 *     built by Gram-Schmidt in physical coordinates
 *     (src/triangleinfo.cpp:281-602); basis row 0 is the cell mean;
 *   - residuals are R = R_volume - R_edge before the mass division, the
 *     reference's rhs_edge_* (src/kernelfunctions.cu:584-637).
 * Internally the state lives in HBM in a reference-element orthonormal basis
 * (RKDG_BASIS_NATIVE), which represents the same functions.
 */
#ifndef RKDG_H
#define RKDG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define RKDG_OK 0
#define RKDG_ERR_INVALID 1     /* bad argument, mesh or configuration          */
#define RKDG_ERR_CUDA 2        /* CUDA runtime error (message has details)     */
#define RKDG_ERR_NOMEM 3       /* device or host allocation failed / budget    */
#define RKDG_ERR_STATE 4       /* non-physical state (NaN, rho<=0, p<=0) seen  */
#define RKDG_ERR_NODEVICE 5    /* no usable sm_100 device                      */
#define RKDG_ERR_IO 6          /* file could not be read or written            */
#define RKDG_ERR_BUSY 7        /* resource (slot, budget) not available now    */

/* ---- enumerations ------------------------------------------------------ */
#define RKDG_FLUX_LLF 0        /* local Lax-Friedrichs, alpha from cell means */
#define RKDG_FLUX_HLLC 1       /* HLLC, Davis wave-speed bounds (Toro 10.48)  */
#define RKDG_LIMITER_NONE 0
#define RKDG_LIMITER_TVB 1     /* TVB minmod on characteristic variables      */
#define RKDG_FP64 0            /* FP64 state and arithmetic                   */
#define RKDG_FP32 1            /* FP32 state/arithmetic, FP64 geometry and dt */
#define RKDG_FP32C 2           /* as RKDG_FP32, with each cell mean stored as a
                                  high + low float pair (about 48 significant
                                  bits) and updated in FP64: the state's
                                  storage rounding no longer accumulates over
                                  long runs; one more 16-byte row per element */
#define RKDG_BASIS_REFERENCE 0 /* the reference's per-element basis           */
#define RKDG_BASIS_NATIVE 1    /* reference-element orthonormal basis         */

/* boundary tags of an edge; the values are the reference's cell tags
 * (inc/defines.h:48-54) */
#define RKDG_BC_INTERIOR 0
#define RKDG_BC_FARFIELD 1     /* given state (far field / supersonic inflow) */
#define RKDG_BC_OUTFLOW 2      /* zero-gradient copy                          */
#define RKDG_BC_REFLECTION 3   /* slip wall                                   */

/* ---- mesh -------------------------------------------------------------- */
/* A triangle mesh.  Edge k of a triangle is the edge opposite its vertex k
 * (edge 0 = v1->v2, 1 = v2->v0, 2 = v0->v1), vertices counter-clockwise.
 * tri_neighbour[3t+k] is the triangle across edge k or -1 on a boundary; if
 * NULL it is built from shared vertex ids (no periodicity then).  Periodic
 * meshes pass explicit neighbours and per-triangle (unwrapped) vertices.
 * bc[3t+k] tags boundary edges (RKDG_BC_*); if NULL, the reference's rule is
 * used: far field when the reflected (ghost) triangle's barycentre lies
 * outside |x|,|y| <= 15, else wall (src/unstructuredgrid.cpp:729-760). */
typedef struct rkdg_mesh_desc {
    int32_t ntri;
    int32_t nvert;
    const double* vertices;      /* [nvert][2]                       */
    const int32_t* tri_vertex;   /* [ntri][3]                        */
    const int32_t* tri_neighbour;/* [ntri][3] or NULL                */
    const int8_t* bc;            /* [ntri][3] or NULL                */
} rkdg_mesh_desc;

/* Discretisation and physics.  Replaces the compile-time constants of
 * inc/defines.h:17-32 and the keys of input/main.conf read by
 * CCUDARkdgSolver::initConfig (src/cudarkdgsolver.cu:93-156). */
typedef struct rkdg_params {
    int32_t order;        /* 1 (P1) or 2 (P2)                                */
    int32_t nq;           /* volume rule: 3 (deg 2), 6 (deg 4) or 7 (deg 5)  */
    int32_t ng;           /* Gauss points per edge: 2 or 3                   */
                          /* supported: P2 with nq 7|6, ng 3; P1 nq 3, ng 2 */
    int32_t flux;         /* RKDG_FLUX_*                                     */
    int32_t limiter;      /* RKDG_LIMITER_*                                  */
    int32_t rk;           /* 2 or 3 (SSP Runge-Kutta stages)                 */
    int32_t precision;    /* RKDG_FP64, RKDG_FP32 or RKDG_FP32C              */
    int32_t reorder;      /* 1: Morton-reorder elements in HBM for locality  */
    double gamma;
    double cfl;           /* dt = cfl / max (|u|+c) perimeter/area           */
    double tvb_m;         /* TVB constant M                                  */
    double farfield[4];   /* conservative far-field / inflow state           */
} rkdg_params;

/* Fills p with the reference's defaults: P2, 7/3-point rules, LLF, no
 * limiter, SSP-RK3, FP64, gamma 1.4, cfl 0.18 (src/cudarkdgsolver.cu:3-32). */
void rkdg_default_params(rkdg_params* p);

typedef struct rkdg_ctx rkdg_ctx;

/* ---- lifetime ---------------------------------------------------------- */
/* Builds connectivity (O(T) edge hashing), FP64 geometry and device arrays,
 * and binds the calling thread's current CUDA device.
 * Replaces CCUDARkdgSolver::run + runNext (src/cudarkdgsolver.cu:158-230):
 * CUnstructuredGrid::initializeGrid/initializeGridNext, initializeTriangleInfos,
 * markLocalBoundaryTriangles, CCUDAArrays::allocateMemory and
 * copyTriangleInfosToGPU. */
int rkdg_create(const rkdg_mesh_desc* mesh, const rkdg_params* params, rkdg_ctx** out);

/* Replaces ~CCUDARkdgSolver / ~CCUDAArrays (src/cudaarrays.cpp:227-292). */
int rkdg_destroy(rkdg_ctx* ctx);

/* Thread-local message of the last failing call on this thread. */
const char* rkdg_last_error(void);

/* Sizes: triangles, basis functions per variable, device bytes held. */
int rkdg_get_sizes(const rkdg_ctx* ctx, int32_t* ntri, int32_t* nbasis, size_t* device_bytes);

/* The cudaStream_t (as void*) every call of this context is ordered on. */
int rkdg_get_stream(const rkdg_ctx* ctx, void** stream);

/* ---- state ------------------------------------------------------------- */
/* Free-stream initial condition: cell mean = farfield state, higher modes 0.
 * Replaces CCUDARkdgSolver::initRKDG (src/cudarkdgsolver.cu:326-368). */
int rkdg_init_freestream(rkdg_ctx* ctx);

/* Host <-> device state in the reference layout [4][nbasis][ld].  basis is
 * RKDG_BASIS_REFERENCE or RKDG_BASIS_NATIVE.  rkdg_get_state replaces
 * CCUDARkdgSolver::copyFreedomToHost (src/cudarkdgsolver.cu:253-264). */
int rkdg_set_state(rkdg_ctx* ctx, const double* U, int32_t ld, int32_t basis);
int rkdg_get_state(rkdg_ctx* ctx, double* U, int32_t ld, int32_t basis);

/* ---- hot path ---------------------------------------------------------- */
/* R(U) of the current state, [4][nbasis][ld], not divided by the mass.
 * One evaluation of the chain calculateConVars -> boundaryCondition ->
 * calculateVolumeRHS -> calculateLFCoeff -> calculateEdgeFG ->
 * calculateFlux x2 -> calculateEdgeRHS (src/cudarkdgsolver.cu:382-553,
 * src/rkdgadvance.cpp:135-159), here one fused kernel. */
int rkdg_residual(rkdg_ctx* ctx, double* R, int32_t ld, int32_t basis);

/* CFL time step of the current state.  Replaces CCUDARkdgSolver::getTimeStep
 * + the dt read-back (src/cudarkdgsolver.cu:370-380, src/rkdgadvance.cpp:165-168). */
int rkdg_compute_dt(rkdg_ctx* ctx, double* dt);

/* Saves the current state as U^n (src/rkdgadvance.cpp:104-107). */
int rkdg_save_old(rkdg_ctx* ctx);

/* Stage s (0-based) of the SSP-RK scheme against the saved U^n:
 * R(U) and the stage update fused (and the limiter when enabled).
 * Replaces one RK iteration of src/rkdgadvance.cpp:132-195
 * (rkdgStepOne/Two/Three, src/cudarkdgsolver.cu:555-599). */
int rkdg_stage(rkdg_ctx* ctx, int32_t s, double dt);

/* Applies the TVB limiter to the current state. */
int rkdg_limit(rkdg_ctx* ctx);

/* One full time step.  dt <= 0 uses the CFL time step of the current state.
 * dt_used and monitor (max |d rho_mean|, max |d rhoE_mean|, the reference's
 * residual monitor, src/kernelfunctions.cu:751-867) may be NULL.
 * Replaces one iteration of RkdgAdvance::advance (src/rkdgadvance.cpp:91-243). */
int rkdg_step(rkdg_ctx* ctx, double dt, double* dt_used, double* monitor);

/* nsteps steps on the device with no host round trip (CUDA graph of the
 * whole step), stopping early at t_final when t_final > 0 (dt clipped to
 * land on it).  Returns the simulated time reached and steps taken.
 * Replaces RkdgAdvance::advance's loop (src/rkdgadvance.cpp:91-243). */
int rkdg_advance(rkdg_ctx* ctx, int32_t nsteps, double t_final, double* t, int32_t* steps_done);

/* Simulated time and step counter of the context (device-resident). */
int rkdg_get_time(rkdg_ctx* ctx, double* t, int32_t* steps);
int rkdg_set_time(rkdg_ctx* ctx, double t);

/* FP64 conservation totals sum_e area_e * mean_e for the 4 variables,
 * deterministic (fixed-order reduction). */
int rkdg_conservation_totals(rkdg_ctx* ctx, double totals[4]);

/* Benchmark helper: launches the fused kernel of stage s (0-based) `reps`
 * times back to back on the context's stream, writing to a scratch buffer
 * (the state is not advanced; the last stage includes its CFL and monitor
 * epilogue), and returns the mean device time per launch in milliseconds
 * measured with CUDA events on that stream.  No reference
 * counterpart (the reference times nothing on the device). */
int rkdg_time_stage(rkdg_ctx* ctx, int32_t s, int32_t reps, double* ms_per_launch);

/* Allocation-free FP64 conservation totals.  No counterpart in the
 * reference.  For callers that cannot allocate device memory -- an embedding
 * application whose device memory is all owned by its own allocator, or a
 * loop that must not allocate once running: the caller passes device arrays
 * d_means [4][ld] (the cell means of rho, rhou, rhov, rhoE: row 0 of each
 * freedom block) and d_area [ntri], and receives sum_e area_e * mean_e in
 * d_totals[4] (device), ordered on `stream` (a cudaStream_t, NULL = legacy
 * default stream) and reduced in a fixed order (deterministic).  Scratch is
 * a static 128 KiB device array inside this library, held by every GPU that
 * loads it until exit; ntri is limited to 1,048,576 (larger meshes are
 * rejected with RKDG_ERR_INVALID).  The first call on a device looks up that
 * array's device address (cudaGetSymbolAddress), so make it before any
 * stream capture; the address is kept for the process, so resetting the
 * device (cudaDeviceReset) between calls is not supported.  Calls that
 * overlap on one GPU share the array and race; serialise them.  Calls no
 * cudaMalloc/cudaFree.  The means may be the caller's whole state in the
 * reference layout [4][nbasis][ld0], passed in place with ld = nbasis ld0. */
int rkdg_conservation_totals_noalloc(int32_t ntri, const double* d_means, int32_t ld,
                                     const double* d_area, double* d_totals, void* stream);

/* ---- domain decomposition (one partition of a mesh per device) ---------- */
/* A partition of a mesh shared by several devices (one process per GPU):
 * elements [0, n_owned) are the partition's own, in the caller's order (no
 * reordering: the caller orders them for locality), and elements
 * [n_owned, ntri) are halo copies of the neighbouring partitions' elements
 * that share an edge with an owned one (their other edges may be given as
 * boundary edges with any tag; they are never used).  Halo copies are not
 * updated, and are left out of the CFL maximum and the conservation totals.
 * The caller refreshes them before every stage from their owners
 * (rkdg_gather_rows on the owner, a device-to-device transfer such as NCCL
 * send/recv, rkdg_scatter_rows here), takes the minimum of the partitions'
 * rkdg_compute_dt for each step, and advances with rkdg_save_old and
 * rkdg_stage; with the TVB limiter, rkdg_stage leaves it out, and the caller
 * refreshes the halo means (the first mean_rows rows) of the stage output
 * and then calls rkdg_limit.  rkdg_step and rkdg_advance refuse a
 * partition.
 * Replaces the reference's per-rank set-up of its MPI decomposition
 * (partition file and interface elements, src/unstructuredgrid.cpp:290-318;
 * inner-boundary ghost cells, src/unstructuredgrid.cpp:502-526; the
 * interface-index handshake, src/sendboundaryindex.cpp:8-37). */
int rkdg_create_part(const rkdg_mesh_desc* mesh, const rkdg_params* params, int32_t n_owned,
                     rkdg_ctx** out);
/* 16-byte state rows per element: all of them (a full halo refresh) and the
 * leading rows that hold the cell means (a means-only refresh). */
int rkdg_part_rows(const rkdg_ctx* ctx, int32_t* state_rows, int32_t* mean_rows);
/* Rows 0..nrows-1 of the current state of elements d_index[0..n) (device
 * int32, caller element numbers of a partition) to or from the device
 * buffer d_buf [n][nrows][16 bytes], ordered on the context's stream and
 * asynchronous (rkdg_sync waits and reports an index out of range as
 * RKDG_ERR_INVALID).  They replace the device-host copies and the buffer
 * packing around the reference's MPI_Isend/MPI_Irecv halo exchange
 * (RkdgAdvance::commuInfo, src/rkdgadvance.cpp:287-409). */
int rkdg_gather_rows(rkdg_ctx* ctx, const int32_t* d_index, int32_t n, int32_t nrows, void* d_buf);
int rkdg_scatter_rows(rkdg_ctx* ctx, const int32_t* d_index, int32_t n, int32_t nrows, const void* d_buf);
/* Waits for the context's stream and reports any error its kernels flagged. */
int rkdg_sync(rkdg_ctx* ctx);
/* Stream-ordered steps of a partition: every call below only enqueues work
 * on the context's stream (no host round trip; errors surface at rkdg_sync
 * or rkdg_part_time), so a decomposed step runs with the halo transfers
 * (NCCL send/recv) and one all-reduce on the same streams.  Per step, on
 * every partition: refresh the halo copies; rkdg_part_wave(ctx, d_w, 0)
 * writes the partition's CFL wave-speed maximum over its owned elements
 * (one double, device memory); the caller reduces it to the maximum over
 * all partitions (an all-reduce MAX) and hands it back with
 * rkdg_part_wave(ctx, d_w, 1); rkdg_part_begin_step forms dt = cfl / that
 * maximum, clips it to the final time set by rkdg_part_set_final_time,
 * advances the device-resident time and step count and keeps the state as
 * U^n; then per RK stage a halo refresh and rkdg_part_stage (which never
 * applies the limiter), and with the TVB limiter a means refresh and
 * rkdg_part_limit.  Every partition forms the same dt.  A finished solve
 * (time at its final time) skips later steps.  This replaces the
 * reference's per-step dt read-back and its host-staged MPI exchange
 * (src/rkdgadvance.cpp:165-168, 287-409), and the dt reduction it left
 * commented out (src/rkdgadvance.cpp:226-234). */
int rkdg_part_set_final_time(rkdg_ctx* ctx, double t_final);
int rkdg_part_wave(rkdg_ctx* ctx, double* d_wave, int32_t to_context);
int rkdg_part_begin_step(rkdg_ctx* ctx);
int rkdg_part_stage(rkdg_ctx* ctx, int32_t stage);
/* The same stage in two halves, so that the halo refresh overlaps work:
 * rkdg_part_stage_begin launches the partition's tiles that read no halo
 * copy (they need only the owned elements' current state), and
 * rkdg_part_stage_end, once the halo copies are current, the rest, which
 * completes the stage.  Per stage: start the transfers (gather, send and
 * receive), begin, finish the transfers (scatter), end.  The result equals
 * rkdg_part_stage's bit for bit.  The reference exchanges the whole
 * interface through the host before each stage and then runs every
 * element (src/rkdgadvance.cpp:287-409). */
int rkdg_part_stage_begin(rkdg_ctx* ctx, int32_t stage);
int rkdg_part_stage_end(rkdg_ctx* ctx, int32_t stage);
int rkdg_part_limit(rkdg_ctx* ctx);
/* Waits, reports flagged errors, and returns the time, the step count and
 * whether the final time has been reached (any pointer may be NULL). */
int rkdg_part_time(rkdg_ctx* ctx, double* t, int32_t* steps, int32_t* done);

/* ---- output ------------------------------------------------------------ */
/* Writes the cell means as the reference's Tecplot solution.plt
 * (CCUDARkdgSolver::outputSolution, src/cudarkdgsolver.cu:860-1001). */
int rkdg_write_solution(rkdg_ctx* ctx, const char* path);
/* Residual history, as the reference's residual file (RkdgAdvance::advance,
 * src/rkdgadvance.cpp:10-17,201-211): the file starts with the line
 * "N, rho" and then takes one line per step taken by rkdg_step or
 * rkdg_advance, "<step>   <log10(max |change of a cell-mean density| /
 * far-field density)>" (the reference labels step k's value k+1 and omits
 * the last step).  While a history file is open, rkdg_advance launches one
 * step at a time.  NULL closes it. */
int rkdg_set_residual_log(rkdg_ctx* ctx, const char* path);

/* ---- checkpoint / resume ----------------------------------------------- */
/* No reference counterpart (the reference writes no restart files).
 * rkdg_checkpoint_save writes the context's full state to path: a header
 * (format tag, triangle count, order, precision, a hash of the mesh in its
 * internal order, time, step count, the CFL wave maximum and monitor, the
 * far-field state, the quadrature rules, flux, limiter, RK scheme, gamma,
 * CFL number and TVB constant) followed by the state rows exactly as held on
 * the device.  A run restored from it continues bit for bit as if never
 * stopped.  rkdg_checkpoint_load restores such a file into a context built
 * on the same mesh, order, precision, method and physics (RKDG_ERR_INVALID
 * otherwise; an FP32 or FP32C file also needs the same far-field state, its
 * cell means being stored relative to it); RKDG_ERR_IO when the file cannot
 * be read or written. */
int rkdg_checkpoint_save(rkdg_ctx* ctx, const char* path);
int rkdg_checkpoint_load(rkdg_ctx* ctx, const char* path);

/* ---- batched independent solves ----------------------------------------- */
/* Many independent solves on meshes of uneven size and mixed order (P1
 * and P2) packed into one element space: every RK stage of all solves is
 * one launch of the tile-staged kernel over the concatenated tiles (a
 * persistent pass when the autotuner picks fewer CTAs than tiles), each
 * solve with its own dt, time, final time and monitor, and the whole step
 * captured as one CUDA graph.  A solve's arithmetic does not depend on the
 * others: its result equals the same solve run alone, bit for bit.
 * No reference counterpart: the reference runs one solve per process
 * (src/main.cpp:24-159). */
typedef struct rkdg_batch rkdg_batch;

/* orders[s]: 1 or 2 per solve; P2 solves use params->nq (6 or 7 for a
 * P2-only batch, 6 when P1 and P2 are mixed) and 3 edge points, P1 solves
 * the 3/2-point rules.  params->precision, flux, rk, gamma, cfl and reorder
 * (Morton order within each solve) are shared; farfields [nsolves][4] gives
 * each solve's far-field state (NULL: params). */
int rkdg_batch_create(int32_t nsolves, const rkdg_mesh_desc* meshes, const int32_t* orders,
                      const double* farfields, const rkdg_params* params, rkdg_batch** out);
int rkdg_batch_destroy(rkdg_batch* b);
/* Native-basis state of one solve, [4][nbasis(solve)][ld] in its caller order. */
int rkdg_batch_set_state(rkdg_batch* b, int32_t solve, const double* U, int32_t ld);
int rkdg_batch_get_state(rkdg_batch* b, int32_t solve, double* U, int32_t ld);
/* nsteps device-resident steps of every solve; t_final[s] > 0 stops solve s
 * there (NULL: none).  t[s] and steps[s] (may be NULL) receive each solve's
 * time and step count. */
int rkdg_batch_advance(rkdg_batch* b, int32_t nsteps, const double* t_final, double* t,
                       int32_t* steps);
int rkdg_batch_set_time(rkdg_batch* b, int32_t solve, double t);
/* Picks the tile size (128 or 256 elements, one thread per element), the
 * persistent grid size and the tile order by timing candidate launch shapes
 * on this batch's live state; returns the chosen CTA count (0: one per
 * tile), tile order (0 solve order, 1 P2 tiles first, 2 P2 tiles first and
 * the P2 and P1 tiles of a mixed pack as two concurrent launches of the
 * single-order kernels) and tile size (any pointer may be NULL).  Every
 * shape gives the same bits for a given tile size.  The reference fixes its
 * block size from its configuration file (threadsperblock,
 * src/cudarkdgsolver.cu:22). */
int rkdg_batch_autotune(rkdg_batch* b, int32_t* ctas, int32_t* tile_order, int32_t* tile);
int rkdg_batch_set_shape(rkdg_batch* b, int32_t ctas, int32_t tile_order);
/* Rebuilds the tile tables for tiles of 128 or 256 elements.  A solve's
 * result does not depend on the tile size beyond rounding (interface
 * fluxes are formed once per tile pair). */
int rkdg_batch_set_tile(rkdg_batch* b, int32_t tile);
/* Mean device milliseconds of one launch of stage s over all solves (the
 * last stage with its CFL and monitor epilogue, as it runs in a step). */
int rkdg_batch_time_stage(rkdg_batch* b, int32_t s, int32_t reps, double* ms_per_launch);
int rkdg_batch_get_sizes(const rkdg_batch* b, int64_t* elements, int32_t* ntiles, size_t* device_bytes);
int rkdg_batch_get_stream(const rkdg_batch* b, void** stream);

/* ---- serving: continuous batching of solve requests --------------------- */
/* A request loop on its own host thread.  It admits solve requests into a
 * device pool sized by an HBM budget (elements, halo and flux-task entries,
 * solve slots), keeps every admitted solve's state resident in HBM, and
 * advances all in-flight solves together: one launch per RK stage over the
 * packed tiles (CUDA graph; the set of tiles changes without recapture).
 * Requests that arrive while others run are admitted as soon as a slot and
 * memory are free; each solve runs to its own final time and is retired
 * (state copied back, memory freed) by the loop.  A solve's arithmetic is
 * independent of what else is in flight: its result equals the same solve
 * run alone.  No reference counterpart (the reference runs one solve per
 * process). */
typedef struct rkdg_server rkdg_server;

/* params: precision, rk, gamma, cfl, tvb_m and nq (P2 rule, 6) shared by
 * all requests, flux the default of rkdg_server_submit; hbm_budget_bytes
 * bounds the pool; max_slots bounds the number of solves in flight. */
int rkdg_server_create(const rkdg_params* params, size_t hbm_budget_bytes, int32_t max_slots,
                       rkdg_server** out);
/* Stops the loop (in-flight solves are abandoned) and frees everything. */
int rkdg_server_destroy(rkdg_server* s);
/* Queues a solve: mesh, order (1 or 2), native-basis initial state
 * [4][nbasis][ntri] (caller triangle order), final time, far-field /
 * inflow state, limiter flag.  Host preprocessing (connectivity, geometry,
 * tiles) runs in the calling thread.  Returns the request id. */
int rkdg_server_submit(rkdg_server* s, const rkdg_mesh_desc* mesh, int32_t order, const double* U0,
                       double t_final, const double* farfield, int32_t limiter, int64_t* id);
/* As rkdg_server_submit, with the request's own Riemann flux (RKDG_FLUX_*;
 * rkdg_server_submit uses params->flux).  The loop runs the LLF and the
 * HLLC requests' tiles as two launches per stage on two streams, joined
 * before the next stage. */
int rkdg_server_submit_method(rkdg_server* s, const rkdg_mesh_desc* mesh, int32_t order, const double* U0,
                              double t_final, const double* farfield, int32_t limiter, int32_t flux,
                              int64_t* id);
/* Waits up to timeout_s (< 0: forever) for request id; status 0 queued,
 * 1 running, 2 done, 3 failed.  On done, U (may be NULL) receives the final
 * state [4][nbasis][ntri], and times[3] (may be NULL) the submit, admit and
 * completion times in seconds on the loop's steady clock; steps the number
 * of time steps taken.  A fetched request is released. */
int rkdg_server_wait(rkdg_server* s, int64_t id, double timeout_s, int32_t* status, double* U,
                     double* times, int32_t* steps);
/* Aggregate counters: DOF-stage updates done, seconds with work in flight,
 * requests completed, peak solves in flight, pool capacity in elements. */
int rkdg_server_stats(rkdg_server* s, double* dof_stage_updates, double* busy_seconds,
                      int64_t* completed, int32_t* peak_in_flight, int64_t* capacity_elements);
/* Seconds on the loop's steady clock (the clock of rkdg_server_wait's times). */
double rkdg_server_clock(void);
/* Where the loop's time went: seconds uploading admitted requests (tables,
 * state, tile lists; the device idles meanwhile), seconds retiring finished
 * ones (state export and copy back), seconds of step chunks (graph launches
 * and the control-block read that ends each chunk of 4 steps), and the
 * number of chunks. */
int rkdg_server_timing(rkdg_server* s, double* admit_s, double* retire_s, double* step_s, int64_t* chunks);
/* Health of the loop: RKDG_OK while it runs, with the number of queued and
 * in-flight requests (either may be NULL).  Once the loop has stopped on an
 * error (a failed CUDA call) it returns that error's code, with the message
 * in rkdg_last_error(), and zero counts: every request that was queued or in
 * flight then has status 3 (failed), later submits are refused, and the
 * server can only be destroyed. */
int rkdg_server_status(rkdg_server* s, int32_t* queued, int32_t* in_flight);
/* Test support, no reference counterpart: the loop stops as on a failed CUDA
 * call before launching its (after_chunks + 1)-th next chunk of steps.
 * Nothing is done to the device; it exercises the failure handling above. */
int rkdg_server_inject_fault(rkdg_server* s, int32_t after_chunks);

/* ---- diagnostics ------------------------------------------------------- */
/* No reference counterpart.  The stage kernels wait on an mbarrier for each
 * tile's staged rows, and every such wait gives up after 2 s, sets an error
 * bit in the solve's control word (reported as RKDG_ERR_CUDA at the next host
 * sync) and ends the CTA instead of hanging the device.  This self-test runs
 * one such wait on data that never arrives, with limit_s (<= 10) seconds:
 * *timed_out = 1 and *waited_s >= limit_s when the bound works; the device
 * stays usable afterwards. */
int rkdg_wait_selftest(double limit_s, int32_t* timed_out, double* waited_s);

/* ---- mesh files -------------------------------------------------------- */
/* Reads the reference's mesh set: the mesh configuration file
 * (trianglenum, verticenum, edgenum and the five file names) and the five
 * files it names, relative to base_dir (CUnstructuredGrid::initializeGrid
 * and readers, src/unstructuredgrid.cpp:14-60, 193-288).  Header lines are
 * detected rather than assumed, so files with or without the '#...' first
 * line are accepted; ids may be 0- or 1-based.  The arrays are allocated
 * with malloc and owned by the caller (free with rkdg_free_mesh). */
int rkdg_read_mesh(const char* base_dir, const char* mesh_conf, rkdg_mesh_desc* out);
void rkdg_free_mesh(rkdg_mesh_desc* mesh);

/* Host-only: the connectivity rkdg_create would build (no device needed).
 * neighbour [ntri][3], shared [ntri][3] (the neighbour-local index of each
 * shared edge, -1 on boundaries: the reference's sharedEdge,
 * src/unstructuredgrid.cpp:934-976) and bc [ntri][3]; any output may be NULL. */
int rkdg_build_connectivity(const rkdg_mesh_desc* mesh, int32_t* neighbour, int8_t* shared,
                            int8_t* bc);

/* Host-only: the locality (Morton) order the context stores elements in;
 * perm[new] = caller index.  The single-device replacement of the
 * reference's partition file (src/unstructuredgrid.cpp:290-305). */
int rkdg_locality_order(const rkdg_mesh_desc* mesh, int32_t* perm);

/* ---- native basis (for projections done by the caller) ----------------- */
/* Values of the first nbasis native basis functions at npts reference-
 * element points (xi, eta) on the triangle (0,0),(1,0),(0,1); out[npts][nbasis]. */
int rkdg_native_basis(int32_t nbasis, int32_t npts, const double* xi, const double* eta,
                      double* out);

#ifdef __cplusplus
}
#endif
#endif /* RKDG_H */
