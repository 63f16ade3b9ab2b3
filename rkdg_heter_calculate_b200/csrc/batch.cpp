// Batched independent solves (include/rkdg.h, rkdg_batch_*).
//
// Every solve's elements (Morton-ordered within the solve) are packed into
// one element space with the P2 row layout, its tiles' descriptors carry the
// solve id and order, and one tile-staged launch per RK stage covers all of
// them.  Per-solve control blocks hold dt, time, final time, the CFL measure
// and the monitor, so solves advance with their own time steps inside one
// CUDA graph of whole steps (one, and eight for long runs).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "rkdg_internal.hpp"

using namespace rkdg;

struct rkdg_batch {
    rkdg_params p{};
    int S = 0, device = 0, word = 8, ord = 2;
    int64_t total = 0;
    int ld = 0, ntiles = 0, max_halo = 4;
    std::vector<int> order, T, off;
    std::vector<double> far_host;  // [S][4]
    std::vector<int32_t> desc_solve;  // descriptors in solve order [ntiles][8]
    size_t bytes = 0;
    void* U[3] = {nullptr, nullptr, nullptr};
    double* jinv = nullptr;
    int4* tcode = nullptr;
    int4* tdesc = nullptr;
    int2* halo = nullptr;
    uint16_t* task = nullptr;
    int32_t* perm = nullptr;
    double* far = nullptr;
    double* staging = nullptr;
    StepCtl* ctl = nullptr;
    StepCtl* h_ctl = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;    // tile order 2: the P1 tiles' launches, forked and joined
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int n2tiles = 0;                   // P2 tiles (the first ones in tile orders 1 and 2)
    cudaGraphExec_t graph = nullptr;   // one step
    cudaGraphExec_t graph_n = nullptr; // kGraphSteps steps (fewer graph launches and boundaries)
    // tile order: 0 = solve order, 1 = P2 tiles first, 2 = P2 tiles first
    // and the P2 and P1 tiles as two launches of the single-order kernels on
    // forked streams (mixed packs)
    int ctas = 0, tile_order = 0, tile = kTile;
    std::vector<HostMesh> topo;  // per solve (internal order): T, neighbours, shared edges, tags
    size_t table_bytes = 0;      // device bytes of the tile tables (rebuilt with the tile size)
    bool wave_valid = false;
    std::vector<bool> have_state;
    TileArgs tiles{};
};

namespace {

template <class F>
int guarded(F&& f) {
    try {
        f();
        return RKDG_OK;
    } catch (const Error& e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return RKDG_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return RKDG_ERR_INVALID;
    }
}

void* balloc(rkdg_batch* b, size_t bytes) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{RKDG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                                        cudaGetErrorString(e)};
    }
    b->bytes += bytes;
    return p;
}

template <class T>
void h2d(rkdg_batch* b, T* dst, const std::vector<T>& src) {
    if (!src.empty())
        RKDG_CUDA_TRY(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, b->stream));
}

// the P2 row layout for every solve (RKDG_FP32C: row 6 holds the low parts
// of the cell means, for P1 and P2 solves alike)
size_t state_bytes(const rkdg_batch* b) { return (size_t)16 * state_rows(b->p.precision, 6) * b->ld; }
int kprec(const rkdg_batch* b) { return kernel_prec(b->p.precision); }
int lo_row(const rkdg_batch* b) { return b->p.precision == RKDG_FP32C ? 6 : -1; }

void sync(rkdg_batch* b) { RKDG_CUDA_TRY(cudaStreamSynchronize(b->stream)); }

void pull(rkdg_batch* b) {
    RKDG_CUDA_TRY(cudaMemcpyAsync(b->h_ctl, b->ctl, sizeof(StepCtl) * b->S, cudaMemcpyDeviceToHost, b->stream));
    sync(b);
}

void push(rkdg_batch* b) {
    RKDG_CUDA_TRY(cudaMemcpyAsync(b->ctl, b->h_ctl, sizeof(StepCtl) * b->S, cudaMemcpyHostToDevice, b->stream));
}

// uploads the descriptors in the chosen tile order
void upload_desc(rkdg_batch* b) {
    std::vector<int32_t> d(b->desc_solve.size());
    std::vector<int> idx(b->ntiles);
    std::iota(idx.begin(), idx.end(), 0);
    if (b->tile_order != 0)  // P2 tiles first: the expensive tiles start early
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) {
            return b->desc_solve[8 * x + 3] > b->desc_solve[8 * y + 3];
        });
    b->n2tiles = 0;
    for (int i = 0; i < b->ntiles; ++i) b->n2tiles += b->desc_solve[8 * i + 3] == 2;
    for (int i = 0; i < b->ntiles; ++i)
        std::memcpy(&d[8 * i], &b->desc_solve[8 * idx[i]], 8 * sizeof(int32_t));
    h2d(b, reinterpret_cast<int32_t*>(b->tdesc), d);
}

StageArgs stage_args(const rkdg_batch* b) {
    StageArgs a{};
    a.T = (int)b->total;
    a.ld = b->ld;
    a.jinv = b->jinv;
    a.conn = nullptr;
    a.ctl = b->ctl;
    a.gamma = b->p.gamma;
    for (int v = 0; v < 4; ++v) a.far[v] = b->p.farfield[v];
    a.far_sid = b->far;
    a.lo_row = lo_row(b);
    return a;
}

void coeffs(int rk, int s, double& a, double& c) {
    if (s == 0) a = 0, c = 1;
    else if (rk == 2) a = 0.5, c = 0.5;
    else if (s == 1) a = 0.75, c = 0.25;
    else a = 1.0 / 3.0, c = 2.0 / 3.0;
}

// One stage over every tile of the pack: one launch of the kernel for the
// pack's orders, or in tile order 2 (a mixed pack) the P2 tiles with the
// P2 kernel on the batch's stream and the P1 tiles with the P1 kernel (more
// resident CTAs per SM) on a second stream forked from it and joined after
// them.  A tile's arithmetic is the same in every kernel that runs it.
void launch_pack_stage(rkdg_batch* b, const StageArgs& a) {
    if (b->tile_order != 2 || b->ord != 3) {
        launch_stage(a, b->tiles, b->ord, b->p.nq, b->p.flux, kprec(b), b->ctas, b->stream);
        return;
    }
    TileArgs t2 = b->tiles, t1 = b->tiles;
    t2.ntiles = b->n2tiles;
    t1.desc = b->tdesc + 2 * (size_t)b->n2tiles;
    t1.ntiles = b->ntiles - b->n2tiles;
    RKDG_CUDA_TRY(cudaEventRecord(b->ev_fork, b->stream));
    RKDG_CUDA_TRY(cudaStreamWaitEvent(b->stream2, b->ev_fork, 0));
    if (t2.ntiles > 0) launch_stage(a, t2, 2, b->p.nq, b->p.flux, kprec(b), b->ctas, b->stream);
    if (t1.ntiles > 0) launch_stage(a, t1, 1, b->p.nq, b->p.flux, kprec(b), b->ctas, b->stream2);
    RKDG_CUDA_TRY(cudaEventRecord(b->ev_join, b->stream2));
    RKDG_CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
}

void enqueue_stage(rkdg_batch* b, int s, int in, int u0, int out, bool last) {
    StageArgs a = stage_args(b);
    coeffs(b->p.rk, s, a.a, a.b);
    a.U = b->U[in];
    a.U0 = s == 0 ? nullptr : b->U[u0];
    a.Unew = b->U[out];
    a.last_stage = last ? 1 : 0;
    launch_pack_stage(b, a);
}

void enqueue_step(rkdg_batch* b) {
    launch_step_begin(b->ctl, b->S, b->stream);
    if (b->p.rk == 3) {
        enqueue_stage(b, 0, 0, 0, 1, false);
        enqueue_stage(b, 1, 1, 0, 2, false);
        enqueue_stage(b, 2, 2, 0, 0, true);
    } else {
        enqueue_stage(b, 0, 0, 0, 1, false);
        enqueue_stage(b, 1, 1, 0, 0, true);
    }
}

// (Re)builds the tile tables of every solve for tiles of b->tile elements
// and uploads them: edge codes, descriptors (in the chosen tile order), halo
// and flux-task lists.
void build_batch_tiles(rkdg_batch* b) {
    std::vector<int32_t> code, halo;
    std::vector<uint16_t> task;
    b->desc_solve.clear();
    b->ntiles = 0;
    b->max_halo = 4;
    for (int s = 0; s < b->S; ++s) {
        TileTables tt = build_tiles(b->topo[s], b->off[s], s, b->order[s], (int)(halo.size() / 2),
                                    (int)task.size(), -1, b->tile);
        code.insert(code.end(), tt.code.begin(), tt.code.end());
        halo.insert(halo.end(), tt.halo.begin(), tt.halo.end());
        task.insert(task.end(), tt.task.begin(), tt.task.end());
        b->desc_solve.insert(b->desc_solve.end(), tt.desc.begin(), tt.desc.end());
        b->max_halo = std::max(b->max_halo, tt.max_halo);
        b->ntiles += tt.ntiles;
    }
    code.resize((size_t)4 * b->ld, 0);
    for (void* p : {(void*)b->tcode, (void*)b->tdesc, (void*)b->halo, (void*)b->task}) cudaFree(p);
    b->bytes -= b->table_bytes;
    const size_t before = b->bytes;
    b->tcode = (int4*)balloc(b, sizeof(int32_t) * code.size());
    h2d(b, reinterpret_cast<int32_t*>(b->tcode), code);
    b->tdesc = (int4*)balloc(b, sizeof(int32_t) * b->desc_solve.size());
    upload_desc(b);
    b->halo = (int2*)balloc(b, sizeof(int32_t) * std::max<size_t>(2, halo.size()) + kTablePad);
    h2d(b, reinterpret_cast<int32_t*>(b->halo), halo);
    b->task = (uint16_t*)balloc(b, sizeof(uint16_t) * std::max<size_t>(1, task.size()) + kTablePad);
    h2d(b, b->task, task);
    b->table_bytes = b->bytes - before;
    b->tiles.code = b->tcode;
    b->tiles.desc = b->tdesc;
    b->tiles.halo = b->halo;
    b->tiles.task = b->task;
    b->tiles.max_halo = b->max_halo;
    b->tiles.ntiles = b->ntiles;
    b->tiles.tile = b->tile;
    sync(b);  // host tables go out of scope
}

constexpr int kGraphSteps = 8;

// A graph of `steps` whole steps on the batch's stream.
cudaGraphExec_t capture_steps(rkdg_batch* b, int steps) {
    cudaGraph_t g;
    RKDG_CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    try {
        for (int i = 0; i < steps; ++i) enqueue_step(b);
    } catch (...) {
        cudaStreamEndCapture(b->stream, &g);
        throw;
    }
    RKDG_CUDA_TRY(cudaStreamEndCapture(b->stream, &g));
    cudaGraphExec_t e = nullptr;
    cudaError_t err = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    RKDG_CUDA_TRY(err);
    return e;
}

void drop_graph(rkdg_batch* b) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (b->graph_n) {
        cudaGraphExecDestroy(b->graph_n);
        b->graph_n = nullptr;
    }
}

void destroy_batch(rkdg_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    drop_graph(b);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (void* p : {b->U[0], b->U[1], b->U[2]}) cudaFree(p);
    for (void* p : {(void*)b->jinv, (void*)b->tcode, (void*)b->tdesc, (void*)b->halo, (void*)b->task,
                    (void*)b->perm, (void*)b->far, (void*)b->staging, (void*)b->ctl})
        cudaFree(p);
    if (b->h_ctl) cudaFreeHost(b->h_ctl);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->stream2) cudaStreamDestroy(b->stream2);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

void check_solve(const rkdg_batch* b, int s) {
    if (!b) throw Error{RKDG_ERR_INVALID, "null batch"};
    if (s < 0 || s >= b->S) throw Error{RKDG_ERR_INVALID, "solve index out of range"};
}

}  // namespace

extern "C" {

int rkdg_batch_create(int32_t nsolves, const rkdg_mesh_desc* meshes, const int32_t* orders,
                      const double* farfields, const rkdg_params* params, rkdg_batch** out) {
    rkdg_batch* b = nullptr;
    int rc = guarded([&] {
        if (nsolves <= 0 || !meshes || !orders || !params || !out)
            throw Error{RKDG_ERR_INVALID, "rkdg_batch_create: bad arguments"};
        *out = nullptr;
        const rkdg_params& p = *params;
        if (p.precision != RKDG_FP32 && p.precision != RKDG_FP64 && p.precision != RKDG_FP32C)
            throw Error{RKDG_ERR_INVALID, "unknown precision"};
        if (p.rk != 2 && p.rk != 3) throw Error{RKDG_ERR_INVALID, "rk must be 2 or 3"};
        if (p.limiter != RKDG_LIMITER_NONE) throw Error{RKDG_ERR_INVALID, "batches run without the limiter"};
        if (!(p.gamma > 1.0) || !(p.cfl > 0.0)) throw Error{RKDG_ERR_INVALID, "gamma > 1 and cfl > 0 required"};
        bool has1 = false, has2 = false;
        for (int s = 0; s < nsolves; ++s) {
            if (orders[s] == 1) has1 = true;
            else if (orders[s] == 2) has2 = true;
            else throw Error{RKDG_ERR_INVALID, "orders must be 1 or 2"};
        }
        if (has2 && p.nq != 6 && p.nq != 7) throw Error{RKDG_ERR_INVALID, "P2 solves need nq 6 or 7"};
        if (has1 && has2 && p.nq != 6) throw Error{RKDG_ERR_INVALID, "mixed P1/P2 batches use nq 6 for P2"};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{RKDG_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
        }
        cudaDeviceProp prop;
        RKDG_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
        if (prop.major < 10) throw Error{RKDG_ERR_NODEVICE, "this library is built for sm_100a"};

        b = new rkdg_batch();
        b->device = dev;
        b->p = p;
        b->S = nsolves;
        b->word = p.precision == RKDG_FP64 ? 8 : 4;
        b->ord = has1 && has2 ? 3 : (has2 ? 2 : 1);
        b->order.assign(orders, orders + nsolves);
        b->have_state.assign(nsolves, false);
        RKDG_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        RKDG_CUDA_TRY(cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking));
        RKDG_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        RKDG_CUDA_TRY(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
        RKDG_CUDA_TRY(cudaMallocHost(&b->h_ctl, sizeof(StepCtl) * nsolves));
        std::memset(b->h_ctl, 0, sizeof(StepCtl) * nsolves);
        if (has2) upload_tables(p.nq, 3);
        if (has1) upload_tables(3, 2);

        // pack the solves
        std::vector<double> jv;      // [total][4]
        std::vector<int32_t> perm;
        int64_t total = 0;
        int maxT = 0;
        for (int s = 0; s < nsolves; ++s) {
            HostMesh m = build_mesh(meshes[s]);
            if (p.reorder) m = permute_mesh(m, morton_order(m));
            HostGeometry g = build_geometry(m, orders[s], false, false);
            b->T.push_back(m.T);
            b->off.push_back((int)total);
            maxT = std::max(maxT, m.T);
            jv.insert(jv.end(), g.jinv.begin(), g.jinv.end());
            perm.insert(perm.end(), m.perm.begin(), m.perm.end());
            // the connectivity the tile tables are built from (tile size may change)
            HostMesh t;
            t.T = m.T;
            t.nbr = std::move(m.nbr);
            t.shared = std::move(m.shared);
            t.bc = std::move(m.bc);
            b->topo.push_back(std::move(t));
            total += b->T.back();
            if (total > (int64_t)1 << 30) throw Error{RKDG_ERR_INVALID, "batch too large"};
        }
        b->total = total;
        b->ld = (int)((total + 127) / 128 * 128);
        const int ld = b->ld;
        for (int k = 0; k < 3; ++k) {
            b->U[k] = balloc(b, state_bytes(b));
            RKDG_CUDA_TRY(cudaMemsetAsync(b->U[k], 0, state_bytes(b), b->stream));
        }
        std::vector<double> jp((size_t)4 * ld, 0.0);
        for (int64_t t = 0; t < total; ++t) {
            jp[2 * t] = jv[4 * t];
            jp[2 * t + 1] = jv[4 * t + 1];
            jp[2 * (ld + t)] = jv[4 * t + 2];
            jp[2 * (ld + t) + 1] = jv[4 * t + 3];
        }
        b->jinv = (double*)balloc(b, sizeof(double) * jp.size());
        h2d(b, b->jinv, jp);
        build_batch_tiles(b);
        b->perm = (int32_t*)balloc(b, sizeof(int32_t) * perm.size());
        h2d(b, b->perm, perm);
        std::vector<double> far((size_t)4 * nsolves);
        for (int s = 0; s < nsolves; ++s)
            for (int v = 0; v < 4; ++v) far[4 * s + v] = farfields ? farfields[4 * s + v] : p.farfield[v];
        b->far = (double*)balloc(b, sizeof(double) * far.size());
        h2d(b, b->far, far);
        b->far_host = far;
        b->staging = (double*)balloc(b, sizeof(double) * 24 * (size_t)maxT);
        b->ctl = (StepCtl*)balloc(b, sizeof(StepCtl) * nsolves);
        for (int s = 0; s < nsolves; ++s) b->h_ctl[s].cfl = p.cfl;
        push(b);
        sync(b);
        *out = b;
    });
    if (rc != RKDG_OK && b) destroy_batch(b);
    return rc;
}

int rkdg_batch_destroy(rkdg_batch* b) {
    return guarded([&] { destroy_batch(b); });
}

int rkdg_batch_set_state(rkdg_batch* b, int32_t s, const double* U, int32_t ld) {
    return guarded([&] {
        check_solve(b, s);
        if (!U || ld < b->T[s]) throw Error{RKDG_ERR_INVALID, "rkdg_batch_set_state: bad arguments"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        const int T = b->T[s], nb = b->order[s] == 1 ? 3 : 6;
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(b->staging, sizeof(double) * T, U, sizeof(double) * ld,
                                        sizeof(double) * T, 4 * nb, cudaMemcpyHostToDevice, b->stream));
        char* base = static_cast<char*>(b->U[0]) + (size_t)16 * b->off[s];
        launch_import(T, b->ld, b->staging, T, nullptr, b->perm + b->off[s], base, b->order[s],
                      kprec(b), &b->far_host[4 * s], lo_row(b), b->stream);
        b->have_state[s] = true;
        b->wave_valid = false;
        sync(b);
    });
}

int rkdg_batch_get_state(rkdg_batch* b, int32_t s, double* U, int32_t ld) {
    return guarded([&] {
        check_solve(b, s);
        if (!U || ld < b->T[s]) throw Error{RKDG_ERR_INVALID, "rkdg_batch_get_state: bad arguments"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        const int T = b->T[s], nb = b->order[s] == 1 ? 3 : 6;
        const char* base = static_cast<const char*>(b->U[0]) + (size_t)16 * b->off[s];
        launch_export(T, b->ld, base, nullptr, b->perm + b->off[s], b->staging, T, b->order[s],
                      kprec(b), 0, nullptr, &b->far_host[4 * s], lo_row(b), b->stream);
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(U, sizeof(double) * ld, b->staging, sizeof(double) * T,
                                        sizeof(double) * T, 4 * nb, cudaMemcpyDeviceToHost, b->stream));
        sync(b);
    });
}

int rkdg_batch_set_time(rkdg_batch* b, int32_t s, double t) {
    return guarded([&] {
        check_solve(b, s);
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        pull(b);
        b->h_ctl[s].t = t;
        b->h_ctl[s].done = 0;
        push(b);
        sync(b);
    });
}

int rkdg_batch_advance(rkdg_batch* b, int32_t nsteps, const double* t_final, double* t, int32_t* steps) {
    return guarded([&] {
        if (!b || nsteps < 0) throw Error{RKDG_ERR_INVALID, "rkdg_batch_advance: bad arguments"};
        for (int s = 0; s < b->S; ++s)
            if (!b->have_state[s]) throw Error{RKDG_ERR_INVALID, "solve " + std::to_string(s) + " has no state"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        if (!b->wave_valid) {
            launch_wave(b->tiles, b->ld, b->U[0], kprec(b), b->jinv, b->p.gamma, b->ctl, b->S,
                        b->far, b->stream);
            b->wave_valid = true;
        }
        pull(b);
        std::vector<int> step0(b->S);
        bool any_final = false;
        for (int s = 0; s < b->S; ++s) {
            step0[s] = b->h_ctl[s].step;
            b->h_ctl[s].dt_fixed = 0.0;
            b->h_ctl[s].t_final = (t_final && t_final[s] > 0) ? t_final[s] : 0.0;
            any_final = any_final || b->h_ctl[s].t_final > 0;
            b->h_ctl[s].done = 0;
        }
        push(b);
        if (!b->graph) b->graph = capture_steps(b, 1);
        if (!b->graph_n && nsteps >= kGraphSteps) b->graph_n = capture_steps(b, kGraphSteps);
        int left = nsteps;
        const int chunk = any_final ? 32 : std::max(1, nsteps);
        while (left > 0) {
            const int n = std::min(left, chunk);
            for (int i = 0; i < n / kGraphSteps; ++i) RKDG_CUDA_TRY(cudaGraphLaunch(b->graph_n, b->stream));
            for (int i = 0; i < n % kGraphSteps; ++i) RKDG_CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
            left -= n;
            if (any_final && left > 0) {
                pull(b);
                bool all = true;
                for (int s = 0; s < b->S; ++s) all = all && (b->h_ctl[s].done || b->h_ctl[s].error);
                if (all) break;
            }
        }
        pull(b);
        for (int s = 0; s < b->S; ++s) {
            if (t) t[s] = b->h_ctl[s].t;
            if (steps) steps[s] = b->h_ctl[s].step - step0[s];
        }
        for (int s = 0; s < b->S; ++s) throw_ctl_error(b->h_ctl[s].error, "solve " + std::to_string(s));
    });
}

int rkdg_batch_time_stage(rkdg_batch* b, int32_t s, int32_t reps, double* ms) {
    return guarded([&] {
        if (!b || !ms || s < 0 || s >= b->p.rk || reps <= 0)
            throw Error{RKDG_ERR_INVALID, "rkdg_batch_time_stage: bad arguments"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        pull(b);
        for (int k = 0; k < b->S; ++k) {
            if (!(b->h_ctl[k].dt > 0)) b->h_ctl[k].dt = 1e-6;
            b->h_ctl[k].done = 0;
        }
        push(b);
        StageArgs a = stage_args(b);
        coeffs(b->p.rk, s, a.a, a.b);
        a.U = b->U[0];
        a.U0 = s == 0 ? nullptr : b->U[0];
        a.Unew = b->U[1];
        a.last_stage = s == (int)b->p.rk - 1;  // the last stage with its CFL/monitor epilogue
        cudaEvent_t e0, e1;
        RKDG_CUDA_TRY(cudaEventCreate(&e0));
        RKDG_CUDA_TRY(cudaEventCreate(&e1));
        launch_pack_stage(b, a);
        RKDG_CUDA_TRY(cudaEventRecord(e0, b->stream));
        for (int i = 0; i < reps; ++i) launch_pack_stage(b, a);
        RKDG_CUDA_TRY(cudaEventRecord(e1, b->stream));
        RKDG_CUDA_TRY(cudaEventSynchronize(e1));
        float tms = 0;
        RKDG_CUDA_TRY(cudaEventElapsedTime(&tms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)tms / reps;
    });
}

int rkdg_batch_set_shape(rkdg_batch* b, int32_t ctas, int32_t tile_order) {
    return guarded([&] {
        if (!b || ctas < 0 || tile_order < 0 || tile_order > 2)
            throw Error{RKDG_ERR_INVALID, "rkdg_batch_set_shape: bad arguments"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        if (tile_order != b->tile_order) {
            b->tile_order = tile_order;
            upload_desc(b);
        }
        b->ctas = ctas;
        drop_graph(b);
        sync(b);
    });
}

int rkdg_batch_set_tile(rkdg_batch* b, int32_t tile) {
    return guarded([&] {
        if (!b || (tile != 128 && tile != 256)) throw Error{RKDG_ERR_INVALID, "rkdg_batch_set_tile: 128 or 256"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        if (tile == b->tile) return;
        sync(b);
        const int old = b->tile;
        b->tile = tile;
        drop_graph(b);
        build_batch_tiles(b);
        b->wave_valid = false;  // the CFL measure is redone over the new tiles at the next advance
        if (!tiled_fits(kprec(b), b->ord, b->p.flux, b->max_halo, tile)) {
            const int mh = b->max_halo;
            b->tile = old;
            build_batch_tiles(b);
            throw Error{RKDG_ERR_INVALID, "tiles of " + std::to_string(tile) + " elements: halo lists of " +
                                              std::to_string(mh) + " entries exceed the shared memory of a CTA"};
        }
    });
}

int rkdg_batch_autotune(rkdg_batch* b, int32_t* ctas_out, int32_t* order_out, int32_t* tile_out) {
    return guarded([&] {
        if (!b) throw Error{RKDG_ERR_INVALID, "null batch"};
        for (int s = 0; s < b->S; ++s)
            if (!b->have_state[s]) throw Error{RKDG_ERR_INVALID, "autotune needs every solve's state"};
        RKDG_CUDA_TRY(cudaSetDevice(b->device));
        cudaDeviceProp prop;
        RKDG_CUDA_TRY(cudaGetDeviceProperties(&prop, b->device));
        double best = 1e300;
        int bc = 0, bo = 0, bt = b->tile;
        const int stage = b->p.rk > 1 ? 1 : 0;  // a stage that also reads U^n
        for (int tile : {128, 256}) {
            int rc = rkdg_batch_set_tile(b, tile);
            if (rc == RKDG_ERR_INVALID) continue;  // this tile size does not fit the batch's halo lists
            if (rc != RKDG_OK) throw Error{rc, "autotune: set_tile failed"};
            const int per_sm = std::max(1, tiled_max_ctas_per_sm(kprec(b), b->ord, b->p.nq, b->p.flux,
                                                                  b->tiles.max_halo, tile));
            const int wave = prop.multiProcessorCount * per_sm;
            std::vector<int> cand_order = {0};
            if (b->ord == 3) {
                cand_order.push_back(1);
                cand_order.push_back(2);
            }
            for (int o : cand_order)
                for (int c : {0, wave, 2 * wave, 4 * wave}) {
                    if (c > 0 && c >= b->ntiles) continue;
                    rc = rkdg_batch_set_shape(b, c, o);
                    if (rc != RKDG_OK) throw Error{rc, "autotune: set_shape failed"};
                    double ms = 0;
                    rc = rkdg_batch_time_stage(b, stage, 5, &ms);
                    if (rc != RKDG_OK) throw Error{rc, "autotune: timing failed"};
                    if (ms < best) {
                        best = ms;
                        bc = c;
                        bo = o;
                        bt = tile;
                    }
                }
        }
        int rc = rkdg_batch_set_tile(b, bt);
        if (rc == RKDG_OK) rc = rkdg_batch_set_shape(b, bc, bo);
        if (rc != RKDG_OK) throw Error{rc, "autotune: set_shape failed"};
        if (ctas_out) *ctas_out = bc;
        if (order_out) *order_out = bo;
        if (tile_out) *tile_out = bt;
    });
}

int rkdg_batch_get_sizes(const rkdg_batch* b, int64_t* elements, int32_t* ntiles, size_t* bytes) {
    return guarded([&] {
        if (!b) throw Error{RKDG_ERR_INVALID, "null batch"};
        if (elements) *elements = b->total;
        if (ntiles) *ntiles = b->ntiles;
        if (bytes) *bytes = b->bytes;
    });
}

int rkdg_batch_get_stream(const rkdg_batch* b, void** stream) {
    return guarded([&] {
        if (!b || !stream) throw Error{RKDG_ERR_INVALID, "null argument"};
        *stream = (void*)b->stream;
    });
}

}  // extern "C"
