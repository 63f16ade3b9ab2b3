// C ABI of librkdg.so (include/rkdg.h): context lifetime, state transfer,
// the fused stage path, the device-resident time loop and solution output.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "rkdg_internal.hpp"

namespace rkdg {

namespace {
thread_local std::string g_last_error;
}

void set_error(const std::string& msg) { g_last_error = msg; }

}  // namespace rkdg

using namespace rkdg;

struct rkdg_ctx {
    rkdg_params p{};
    int T = 0, ld = 0, nb = 0;
    int T_own = 0;  // elements the context updates; [T_own, T) are a partition's halo copies
    int device = 0;
    HostMesh mesh;  // internal (possibly reordered) order
    std::vector<double> area;
    DeviceArrays d;
    cudaStream_t stream = nullptr;
    int cur = 0;   // buffer holding the current state
    int old = 0;   // buffer holding U^n for manual stages
    bool conv_ready = false;
    bool wave_valid = false;
    bool have_state = false;
    cudaGraphExec_t graph = nullptr;    // one step
    cudaGraphExec_t graph_n = nullptr;  // kGraphSteps steps (fewer graph launches and boundaries)
    StepCtl* h_ctl = nullptr;  // pinned mirror of the device control block
    TileArgs tiles{};
    int ctas = 0;     // tiled grid size (0: one CTA per tile)
    int n_int_tiles = 0;     // a partition's tiles that read no halo copy (they come first)
    int pending_stage = -1;  // rkdg_part_stage_begin's stage until rkdg_part_stage_end
    int pending_out = -1;
    std::unique_ptr<std::ofstream> reslog;  // residual history file (rkdg_set_residual_log)
    bool graph_monitor = false;  // the captured step forms the residual monitor
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

void* dev_alloc(rkdg_ctx* c, size_t bytes) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{RKDG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                                        cudaGetErrorString(e)};
    }
    c->d.bytes += bytes;
    return p;
}

size_t state_bytes(const rkdg_ctx* c) { return (size_t)16 * state_rows(c->p.precision, c->nb) * c->ld; }

// arithmetic type of the kernels, and the RKDG_FP32C row of the means' low parts
int kprec(const rkdg_ctx* c) { return kernel_prec(c->p.precision); }
int lo_row(const rkdg_ctx* c) { return c->p.precision == RKDG_FP32C ? c->nb : -1; }

void check_params(const rkdg_params& p) {
    if (p.order != 1 && p.order != 2) throw Error{RKDG_ERR_INVALID, "order must be 1 or 2"};
    if (p.nq != 3 && p.nq != 6 && p.nq != 7) throw Error{RKDG_ERR_INVALID, "nq must be 3, 6 or 7"};
    if (p.ng != 2 && p.ng != 3) throw Error{RKDG_ERR_INVALID, "ng must be 2 or 3"};
    const bool rule_ok = (p.order == 2 && p.ng == 3 && (p.nq == 7 || p.nq == 6)) ||
                         (p.order == 1 && p.nq == 3 && p.ng == 2);
    if (!rule_ok)
        throw Error{RKDG_ERR_INVALID,
                    "supported rules: P2 with nq 7 or 6 and ng 3; P1 with nq 3 and ng 2"};
    if (p.flux != RKDG_FLUX_LLF && p.flux != RKDG_FLUX_HLLC) throw Error{RKDG_ERR_INVALID, "unknown flux"};
    if (p.limiter != RKDG_LIMITER_NONE && p.limiter != RKDG_LIMITER_TVB)
        throw Error{RKDG_ERR_INVALID, "unknown limiter"};
    if (p.rk != 2 && p.rk != 3) throw Error{RKDG_ERR_INVALID, "rk must be 2 or 3"};
    if (p.precision != RKDG_FP64 && p.precision != RKDG_FP32 && p.precision != RKDG_FP32C)
        throw Error{RKDG_ERR_INVALID, "unknown precision"};
    if (!(p.gamma > 1.0) || !(p.cfl > 0.0)) throw Error{RKDG_ERR_INVALID, "gamma > 1 and cfl > 0 required"};
    if (!(p.farfield[0] > 0.0)) throw Error{RKDG_ERR_INVALID, "far-field density must be positive"};
}

void sync(rkdg_ctx* c) { RKDG_CUDA_TRY(cudaStreamSynchronize(c->stream)); }

void ensure_staging(rkdg_ctx* c) {
    if (!c->d.staging) c->d.staging = (double*)dev_alloc(c, sizeof(double) * 4 * c->nb * (size_t)c->T);
}

void ensure_conversion(rkdg_ctx* c) {
    if (c->conv_ready) return;
    HostGeometry g = build_geometry(c->mesh, c->p.order, true, false);
    c->d.conv_in = (double*)dev_alloc(c, sizeof(double) * 36 * (size_t)c->T);
    c->d.conv_out = (double*)dev_alloc(c, sizeof(double) * 36 * (size_t)c->T);
    RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.conv_in, g.conv_in.data(), sizeof(double) * 36 * c->T,
                                  cudaMemcpyHostToDevice, c->stream));
    RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.conv_out, g.conv_out.data(), sizeof(double) * 36 * c->T,
                                  cudaMemcpyHostToDevice, c->stream));
    sync(c);
    c->conv_ready = true;
}

void pull_ctl(rkdg_ctx* c) {
    RKDG_CUDA_TRY(cudaMemcpyAsync(c->h_ctl, c->d.ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, c->stream));
    sync(c);
}

void push_ctl(rkdg_ctx* c) {
    RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.ctl, c->h_ctl, sizeof(StepCtl), cudaMemcpyHostToDevice, c->stream));
}

void require_state(const rkdg_ctx* c) {
    if (!c->have_state) throw Error{RKDG_ERR_INVALID, "no state: call rkdg_set_state or rkdg_init_freestream"};
}

// moves the current state into buffer 0 (the step path keeps U^n there)
void normalise_buffers(rkdg_ctx* c) {
    if (c->cur != 0) {
        RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.U[0], c->d.U[c->cur], state_bytes(c),
                                      cudaMemcpyDeviceToDevice, c->stream));
        c->cur = 0;
    }
    c->old = 0;
}

void ensure_wave(rkdg_ctx* c) {
    if (c->wave_valid) return;
    launch_wave(c->tiles, c->ld, c->d.U[c->cur], kprec(c), c->d.jinv, c->p.gamma, c->d.ctl, 1,
                c->d.far, c->stream);
    c->wave_valid = true;
}

StageArgs base_args(const rkdg_ctx* c) {
    StageArgs a{};
    a.T = c->T;
    a.ld = c->ld;
    a.jinv = c->d.jinv;
    a.conn = c->d.conn;
    a.ctl = c->d.ctl;
    a.gamma = c->p.gamma;
    for (int v = 0; v < 4; ++v) a.far[v] = c->p.farfield[v];
    a.lo_row = lo_row(c);
    a.tvb_m = c->p.tvb_m;
    return a;
}

void stage_coeffs(int rk, int s, double& a, double& b) {
    if (s == 0) {
        a = 0, b = 1;
    } else if (rk == 2) {
        a = 0.5, b = 0.5;
    } else if (s == 1) {
        a = 0.75, b = 0.25;
    } else {
        a = 1.0 / 3.0, b = 2.0 / 3.0;
    }
}

void launch_one_stage(rkdg_ctx* c, int s, int in, int u0, int out, bool monitor = true, bool part_stage = false) {
    StageArgs a = base_args(c);
    stage_coeffs(c->p.rk, s, a.a, a.b);
    a.U = c->d.U[in];
    a.U0 = s == 0 ? nullptr : c->d.U[u0];
    a.Unew = c->d.U[out];
    a.last_stage = s == c->p.rk - 1;
    a.monitor = monitor ? 1 : 0;
    // a partition applies its limiter by rkdg_limit once the halo means of
    // the stage output have been exchanged
    const bool limit = c->p.limiter == RKDG_LIMITER_TVB && c->T_own == c->T && !part_stage;
    // the stage lists the tiles its limiter test finds changeable; the
    // limiter visits those
    a.tile_flags = limit ? c->d.tile_flags : nullptr;
    a.tile_list = limit ? c->d.tile_list : nullptr;
    a.tile_cap = c->tiles.ntiles;
    launch_stage(a, c->tiles, c->p.order, c->p.nq, c->p.flux, kprec(c), c->ctas, c->stream);
    if (limit)
        launch_tiled_limiter(c->tiles, 0, c->ld, c->d.U[out], c->d.conn, c->d.lim, c->d.jinv, nullptr,
                             c->d.far, kprec(c), c->p.nq, c->p.gamma, c->p.tvb_m, c->d.ctl, c->d.tile_flags,
                             c->d.tile_list, c->tiles.ntiles, c->stream);
}

// one full step on the stream with the state in buffer 0 (graph-capturable);
// monitor: also form the residual monitor in the last stage
void enqueue_step(rkdg_ctx* c, bool monitor) {
    launch_step_begin(c->d.ctl, 1, c->stream);
    if (c->p.rk == 3) {
        launch_one_stage(c, 0, 0, 0, 1, monitor);
        launch_one_stage(c, 1, 1, 0, 2, monitor);
        launch_one_stage(c, 2, 2, 0, 0, monitor);
    } else {
        launch_one_stage(c, 0, 0, 0, 1, monitor);
        launch_one_stage(c, 1, 1, 0, 0, monitor);
    }
}

constexpr int kGraphSteps = 8;

// A graph of `steps` whole steps on the context's stream.
cudaGraphExec_t capture_steps(rkdg_ctx* c, int steps, bool monitor) {
    cudaGraph_t g;
    RKDG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
        for (int i = 0; i < steps; ++i) enqueue_step(c, monitor);
    } catch (...) {
        cudaStreamEndCapture(c->stream, &g);
        throw;
    }
    RKDG_CUDA_TRY(cudaStreamEndCapture(c->stream, &g));
    cudaGraphExec_t e = nullptr;
    cudaError_t err = cudaGraphInstantiate(&e, g, 0);
    cudaGraphDestroy(g);
    RKDG_CUDA_TRY(err);
    return e;
}

void check_error_flag(rkdg_ctx* c) {
    throw_ctl_error(c->h_ctl->error, "solve");
}

// the buffer a stage writes: the last stage of a step overwrites U^n in
// place (each element reads its own U^n first), the others a free buffer
int stage_output(const rkdg_ctx* c, int s) {
    if (s == c->p.rk - 1 && s > 0 && c->old != c->cur) return c->old;
    int out = 0;
    while (out == c->cur || out == c->old) ++out;
    return out;
}

// Stage s of a partition over its tiles [first, last) of the list (the
// interior tiles come first), writing buffer out; the limiter is left to
// the caller (rkdg_part_limit), as in rkdg_part_stage.
void launch_part_tiles(rkdg_ctx* c, int s, int out, int first, int last) {
    if (last <= first) return;
    StageArgs a = base_args(c);
    stage_coeffs(c->p.rk, s, a.a, a.b);
    a.U = c->d.U[c->cur];
    a.U0 = s == 0 ? nullptr : c->d.U[c->old];
    a.Unew = c->d.U[out];
    a.last_stage = s == c->p.rk - 1;
    a.monitor = 1;
    TileArgs t = c->tiles;
    t.desc = c->tiles.desc + 2 * (size_t)first;
    t.ntiles = last - first;
    launch_stage(a, t, c->p.order, c->p.nq, c->p.flux, kprec(c), c->ctas, c->stream);
}

// One line of the residual history for the step just taken (the control
// block on the host is current): the step number and log10 of the largest
// cell-mean density change over the step relative to the far-field density.
void log_residual(rkdg_ctx* c) {
    if (!c->reslog) return;
    double m0;
    std::memcpy(&m0, &c->h_ctl->mon_bits[0], sizeof(double));
    *c->reslog << c->h_ctl->step << "   " << std::log10(m0 / c->p.farfield[0]) << "\n";
}

void destroy_ctx(rkdg_ctx* c) {
    if (!c) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    if (c->graph) cudaGraphExecDestroy(c->graph);
    if (c->graph_n) cudaGraphExecDestroy(c->graph_n);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (void* p : {c->d.U[0], c->d.U[1], c->d.U[2]}) cudaFree(p);
    cudaFree(c->d.jinv);
    cudaFree(c->d.conn);
    cudaFree(c->d.lim);
    cudaFree(c->d.tile_flags);
    cudaFree(c->d.tile_list);
    cudaFree(c->d.perm);
    cudaFree(c->d.conv_in);
    cudaFree(c->d.conv_out);
    cudaFree(c->d.staging);
    cudaFree(c->d.partial);
    cudaFree(c->d.ctl);
    cudaFree(c->d.far);
    cudaFree(c->d.tcode);
    cudaFree(c->d.tdesc);
    cudaFree(c->d.halo);
    cudaFree(c->d.task);
    if (c->h_ctl) cudaFreeHost(c->h_ctl);
    if (c->stream) cudaStreamDestroy(c->stream);
    cudaSetDevice(prev);
    delete c;
}

}  // namespace

extern "C" {

const char* rkdg_last_error(void) { return g_last_error.c_str(); }

void rkdg_default_params(rkdg_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->order = 2;
    p->nq = 7;
    p->ng = 3;
    p->flux = RKDG_FLUX_LLF;
    p->limiter = RKDG_LIMITER_NONE;
    p->rk = 3;
    p->precision = RKDG_FP64;
    p->reorder = 1;
    p->gamma = 1.4;
    p->cfl = 0.18;
    p->tvb_m = 50.0;
    // the reference's default far field: Mach 0.4, alpha 5 deg, rho = p = 1,
    // formed by its own expressions (src/cudarkdgsolver.cu:3-32,116,
    // src/rkdgadvance.cpp:31-34: ut = sqrt(gamma pref / rhoref) mach,
    // rhoE = 1/2 rhoref ut^2 + pref / (gamma - 1))
    const double gamma = p->gamma, ut = std::sqrt(gamma * 1.0 / 1.0) * 0.4;
    const double al = 5.0 * std::atan(1.0) * 4 / 180;
    p->farfield[0] = 1.0;
    p->farfield[1] = 1.0 * ut * std::cos(al);
    p->farfield[2] = 1.0 * ut * std::sin(al);
    p->farfield[3] = 0.5 * 1.0 * ut * ut + 1.0 / (gamma - 1);
}

}  // extern "C"

namespace {

// rkdg_create and rkdg_create_part: n_owned < 0 for a whole mesh.
int create_ctx(const rkdg_mesh_desc* mesh, const rkdg_params* params, int32_t n_owned, rkdg_ctx** out) {
    rkdg_ctx* c = nullptr;
    int rc = guarded([&] {
        if (!mesh || !params || !out) throw Error{RKDG_ERR_INVALID, "rkdg_create: null argument"};
        *out = nullptr;
        check_params(*params);
        if (n_owned >= 0 && (n_owned == 0 || n_owned > mesh->ntri))
            throw Error{RKDG_ERR_INVALID, "rkdg_create_part: n_owned must be in [1, ntri]"};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{RKDG_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
        }
        cudaDeviceProp prop;
        RKDG_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
        if (prop.major < 10)
            throw Error{RKDG_ERR_NODEVICE, "device " + std::to_string(dev) + " is sm_" +
                                               std::to_string(prop.major * 10 + prop.minor) +
                                               "; this library is built for sm_100a"};
        c = new rkdg_ctx();
        c->device = dev;
        c->p = *params;
        c->nb = params->order == 1 ? 3 : 6;
        HostMesh m = build_mesh(*mesh);
        // a partition keeps its caller's order: owned elements first, halo copies after
        if (params->reorder && n_owned < 0) m = permute_mesh(m, morton_order(m));
        c->mesh = std::move(m);
        c->T = c->mesh.T;
        c->T_own = n_owned < 0 ? c->T : n_owned;
        c->ld = (c->T + 127) / 128 * 128;
        HostGeometry g = build_geometry(c->mesh, params->order, false,
                                        params->limiter == RKDG_LIMITER_TVB);
        c->area = g.area;
        RKDG_CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        RKDG_CUDA_TRY(cudaMallocHost(&c->h_ctl, sizeof(StepCtl)));
        std::memset(c->h_ctl, 0, sizeof(StepCtl));
        upload_tables(params->nq, params->ng);

        const int T = c->T, ld = c->ld;
        for (int b = 0; b < 3; ++b) {
            c->d.U[b] = dev_alloc(c, state_bytes(c));
            RKDG_CUDA_TRY(cudaMemsetAsync(c->d.U[b], 0, state_bytes(c), c->stream));
        }
        std::vector<double> jp((size_t)4 * ld, 0.0);
        for (int t = 0; t < T; ++t) {
            jp[2 * (size_t)t] = g.jinv[4 * (size_t)t];
            jp[2 * (size_t)t + 1] = g.jinv[4 * (size_t)t + 1];
            jp[2 * ((size_t)ld + t)] = g.jinv[4 * (size_t)t + 2];
            jp[2 * ((size_t)ld + t) + 1] = g.jinv[4 * (size_t)t + 3];
        }
        c->d.jinv = (double*)dev_alloc(c, sizeof(double) * jp.size());
        RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.jinv, jp.data(), sizeof(double) * jp.size(),
                                      cudaMemcpyHostToDevice, c->stream));
        std::vector<int4> cn(ld, make_int4(-1, -1, -1, 0));
        for (int t = 0; t < T; ++t)
            cn[t] = make_int4(c->mesh.nbr[3 * t], c->mesh.nbr[3 * t + 1], c->mesh.nbr[3 * t + 2],
                              (int)pack_info(&c->mesh.shared[3 * t], &c->mesh.bc[3 * t],
                                             g.lim_pair.empty() ? 0u : g.lim_pair[t]));
        c->d.conn = (int4*)dev_alloc(c, sizeof(int4) * ld);
        RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.conn, cn.data(), sizeof(int4) * ld, cudaMemcpyHostToDevice,
                                      c->stream));
        c->d.perm = (int32_t*)dev_alloc(c, sizeof(int32_t) * T);
        RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.perm, c->mesh.perm.data(), sizeof(int32_t) * T,
                                      cudaMemcpyHostToDevice, c->stream));
        if (params->limiter == RKDG_LIMITER_TVB) {
            c->d.lim = dev_alloc(c, (size_t)3 * ld * (kprec(c) == RKDG_FP64 ? 16 : 8));
            upload_limiter(c->d.lim, ld, 0, g.lim, T, kprec(c), c->stream);
        }
        {
            TileTables tt = build_tiles(c->mesh, 0, 0, params->order, 0, 0, c->T_own);
            c->n_int_tiles = tt.ntiles;
            if (c->T_own < c->T) {
                // a partition: the tiles none of whose halo entries is a halo
                // copy first (they can run while the copies are refreshed),
                // then the rest; a tile's arithmetic does not depend on its
                // place in the list
                std::vector<int32_t> inner, outer;
                for (int t = 0; t < tt.ntiles; ++t) {
                    const int32_t* d = &tt.desc[8 * (size_t)t];
                    bool reads_copy = false;
                    for (int h = 0; h < d[5] && !reads_copy; ++h) reads_copy = tt.halo[2 * (size_t)(d[4] + h)] >= c->T_own;
                    (reads_copy ? outer : inner).insert((reads_copy ? outer : inner).end(), d, d + 8);
                }
                c->n_int_tiles = (int)(inner.size() / 8);
                inner.insert(inner.end(), outer.begin(), outer.end());
                tt.desc.swap(inner);
            }
            c->d.tcode = (int4*)dev_alloc(c, sizeof(int32_t) * tt.code.size());
            c->d.tdesc = (int4*)dev_alloc(c, sizeof(int32_t) * tt.desc.size());
            c->d.halo = (int2*)dev_alloc(c, sizeof(int32_t) * std::max<size_t>(2, tt.halo.size()) + kTablePad);
            c->d.task = (uint16_t*)dev_alloc(c, sizeof(uint16_t) * std::max<size_t>(1, tt.task.size()) + kTablePad);
            RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.tcode, tt.code.data(), sizeof(int32_t) * tt.code.size(),
                                          cudaMemcpyHostToDevice, c->stream));
            RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.tdesc, tt.desc.data(), sizeof(int32_t) * tt.desc.size(),
                                          cudaMemcpyHostToDevice, c->stream));
            if (!tt.halo.empty())
                RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.halo, tt.halo.data(), sizeof(int32_t) * tt.halo.size(),
                                              cudaMemcpyHostToDevice, c->stream));
            RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.task, tt.task.data(), sizeof(uint16_t) * tt.task.size(),
                                          cudaMemcpyHostToDevice, c->stream));
            c->tiles.code = c->d.tcode;
            c->tiles.desc = c->d.tdesc;
            c->tiles.halo = c->d.halo;
            c->tiles.task = c->d.task;
            c->tiles.max_halo = tt.max_halo;
            c->tiles.ntiles = tt.ntiles;
            if (params->limiter == RKDG_LIMITER_TVB) {  // flags 0 and the list empty between stages
                const size_t nf = sizeof(int) * std::max(1, tt.ntiles), nl = sizeof(int) * (kListHead + tt.ntiles);
                c->d.tile_flags = (int*)dev_alloc(c, nf);
                c->d.tile_list = (int*)dev_alloc(c, nl);
                RKDG_CUDA_TRY(cudaMemsetAsync(c->d.tile_flags, 0, nf, c->stream));
                RKDG_CUDA_TRY(cudaMemsetAsync(c->d.tile_list, 0, nl, c->stream));
            }
            sync(c);  // host tables go out of scope
        }
        c->d.partial = (double*)dev_alloc(c, sizeof(double) * 4 * (totals_partial_count(T) + 1));
        c->d.ctl = (StepCtl*)dev_alloc(c, sizeof(StepCtl));
        c->d.far = (double*)dev_alloc(c, sizeof(double) * 4);
        RKDG_CUDA_TRY(cudaMemcpyAsync(c->d.far, params->farfield, sizeof(double) * 4,
                                      cudaMemcpyHostToDevice, c->stream));
        c->h_ctl->cfl = params->cfl;
        push_ctl(c);
        sync(c);
        *out = c;
    });
    if (rc != RKDG_OK && c) destroy_ctx(c);
    return rc;
}

}  // namespace

extern "C" {

int rkdg_create(const rkdg_mesh_desc* mesh, const rkdg_params* params, rkdg_ctx** out) {
    return create_ctx(mesh, params, -1, out);
}

int rkdg_create_part(const rkdg_mesh_desc* mesh, const rkdg_params* params, int32_t n_owned, rkdg_ctx** out) {
    return create_ctx(mesh, params, n_owned, out);
}

int rkdg_part_rows(const rkdg_ctx* c, int32_t* state_rows_out, int32_t* mean_rows) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        if (state_rows_out) *state_rows_out = state_rows(c->p.precision, c->nb);
        if (mean_rows) *mean_rows = c->p.precision == RKDG_FP64 ? 2 : 1;
    });
}

int rkdg_gather_rows(rkdg_ctx* c, const int32_t* d_index, int32_t n, int32_t nrows, void* d_out) {
    return guarded([&] {
        if (!c || n < 0 || nrows < 1 || nrows > state_rows(c->p.precision, c->nb) || (n > 0 && (!d_index || !d_out)))
            throw Error{RKDG_ERR_INVALID, "rkdg_gather_rows: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        launch_rows(true, c->d.U[c->cur], c->ld, c->T, d_index, n, nrows, d_out, &c->d.ctl->error, c->stream);
    });
}

int rkdg_scatter_rows(rkdg_ctx* c, const int32_t* d_index, int32_t n, int32_t nrows, const void* d_in) {
    return guarded([&] {
        if (!c || n < 0 || nrows < 1 || nrows > state_rows(c->p.precision, c->nb) || (n > 0 && (!d_index || !d_in)))
            throw Error{RKDG_ERR_INVALID, "rkdg_scatter_rows: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        launch_rows(false, c->d.U[c->cur], c->ld, c->T, d_index, n, nrows, const_cast<void*>(d_in),
                    &c->d.ctl->error, c->stream);
    });
}

int rkdg_part_set_final_time(rkdg_ctx* c, double t_final) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        pull_ctl(c);
        c->h_ctl->t_final = t_final > 0 ? t_final : 0.0;
        c->h_ctl->dt_fixed = 0.0;
        c->h_ctl->done = 0;
        push_ctl(c);
        sync(c);
    });
}

int rkdg_part_wave(rkdg_ctx* c, double* d_wave, int32_t to_context) {
    return guarded([&] {
        if (!c || !d_wave) throw Error{RKDG_ERR_INVALID, "rkdg_part_wave: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        // the maximum is kept as the bits of a non-negative double
        unsigned long long* w = &c->d.ctl->wave_bits;
        if (to_context) {
            RKDG_CUDA_TRY(cudaMemcpyAsync(w, d_wave, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
            c->wave_valid = true;
        } else {
            ensure_wave(c);
            RKDG_CUDA_TRY(cudaMemcpyAsync(d_wave, w, sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
        }
    });
}

int rkdg_part_begin_step(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        require_state(c);
        if (!c->wave_valid) throw Error{RKDG_ERR_STATE, "rkdg_part_begin_step: no wave-speed maximum (rkdg_part_wave)"};
        if (c->pending_stage >= 0) throw Error{RKDG_ERR_STATE, "rkdg_part_begin_step: a stage is still open"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        launch_step_begin(c->d.ctl, 1, c->stream);
        c->old = c->cur;
        c->wave_valid = false;
    });
}

int rkdg_part_stage(rkdg_ctx* c, int32_t s) {
    return guarded([&] {
        if (!c || s < 0 || s >= c->p.rk) throw Error{RKDG_ERR_INVALID, "rkdg_part_stage: bad stage index"};
        require_state(c);
        if (c->pending_stage >= 0) throw Error{RKDG_ERR_STATE, "rkdg_part_stage: a stage is still open"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        const int out = stage_output(c, s);
        launch_one_stage(c, s, c->cur, c->old, out, true, true);
        c->cur = out;
        c->wave_valid = (s == c->p.rk - 1);
    });
}

int rkdg_part_stage_begin(rkdg_ctx* c, int32_t s) {
    return guarded([&] {
        if (!c || s < 0 || s >= c->p.rk) throw Error{RKDG_ERR_INVALID, "rkdg_part_stage_begin: bad stage index"};
        require_state(c);
        if (c->pending_stage >= 0) throw Error{RKDG_ERR_STATE, "rkdg_part_stage_begin: a stage is already open"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        const int out = stage_output(c, s);
        launch_part_tiles(c, s, out, 0, c->n_int_tiles);
        c->pending_stage = s;
        c->pending_out = out;
    });
}

int rkdg_part_stage_end(rkdg_ctx* c, int32_t s) {
    return guarded([&] {
        if (!c || s != c->pending_stage)
            throw Error{RKDG_ERR_STATE, "rkdg_part_stage_end: not the stage rkdg_part_stage_begin opened"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        const int out = c->pending_out;
        c->pending_stage = -1;
        launch_part_tiles(c, s, out, c->n_int_tiles, c->tiles.ntiles);
        c->cur = out;
        c->wave_valid = (s == c->p.rk - 1);
    });
}

int rkdg_part_limit(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        require_state(c);
        if (c->p.limiter != RKDG_LIMITER_TVB) throw Error{RKDG_ERR_INVALID, "context created without limiter"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        launch_tiled_limiter(c->tiles, 0, c->ld, c->d.U[c->cur], c->d.conn, c->d.lim, c->d.jinv,
                             nullptr, c->d.far, kprec(c), c->p.nq, c->p.gamma, c->p.tvb_m,
                             c->d.ctl, nullptr, nullptr, 0, c->stream);
    });
}

int rkdg_part_time(rkdg_ctx* c, double* t, int32_t* steps, int32_t* done) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        pull_ctl(c);
        check_error_flag(c);
        if (t) *t = c->h_ctl->t;
        if (steps) *steps = c->h_ctl->step;
        if (done) *done = c->h_ctl->done;
    });
}

int rkdg_sync(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        pull_ctl(c);
        check_error_flag(c);
    });
}

int rkdg_destroy(rkdg_ctx* ctx) {
    return guarded([&] { destroy_ctx(ctx); });
}

int rkdg_get_sizes(const rkdg_ctx* c, int32_t* ntri, int32_t* nbasis, size_t* bytes) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        if (ntri) *ntri = c->T;
        if (nbasis) *nbasis = c->nb;
        if (bytes) *bytes = c->d.bytes;
    });
}

int rkdg_get_stream(const rkdg_ctx* c, void** stream) {
    return guarded([&] {
        if (!c || !stream) throw Error{RKDG_ERR_INVALID, "null argument"};
        *stream = (void*)c->stream;
    });
}

int rkdg_set_state(rkdg_ctx* c, const double* U, int32_t ld, int32_t basis) {
    return guarded([&] {
        if (!c || !U || ld < c->T) throw Error{RKDG_ERR_INVALID, "rkdg_set_state: bad arguments"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        ensure_staging(c);
        if (basis == RKDG_BASIS_REFERENCE) ensure_conversion(c);
        else if (basis != RKDG_BASIS_NATIVE) throw Error{RKDG_ERR_INVALID, "unknown basis"};
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(c->d.staging, sizeof(double) * c->T, U, sizeof(double) * ld,
                                        sizeof(double) * c->T, 4 * c->nb, cudaMemcpyHostToDevice,
                                        c->stream));
        c->cur = 0;
        c->old = 0;
        c->pending_stage = -1;
        launch_import(c->T, c->ld, c->d.staging, c->T,
                      basis == RKDG_BASIS_REFERENCE ? c->d.conv_in : nullptr, c->d.perm, c->d.U[0],
                      c->p.order, kprec(c), c->p.farfield, lo_row(c), c->stream);
        c->have_state = true;
        c->wave_valid = false;
        ensure_wave(c);
        sync(c);
    });
}

int rkdg_init_freestream(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        std::vector<double> U((size_t)4 * c->nb * c->T, 0.0);
        for (int v = 0; v < 4; ++v)
            std::fill(U.begin() + (size_t)v * c->nb * c->T, U.begin() + ((size_t)v * c->nb + 1) * c->T,
                      c->p.farfield[v]);
        int rc = rkdg_set_state(c, U.data(), c->T, RKDG_BASIS_NATIVE);
        if (rc != RKDG_OK) throw Error{rc, g_last_error};
    });
}

int rkdg_get_state(rkdg_ctx* c, double* U, int32_t ld, int32_t basis) {
    return guarded([&] {
        if (!c || !U || ld < c->T) throw Error{RKDG_ERR_INVALID, "rkdg_get_state: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        ensure_staging(c);
        if (basis == RKDG_BASIS_REFERENCE) ensure_conversion(c);
        else if (basis != RKDG_BASIS_NATIVE) throw Error{RKDG_ERR_INVALID, "unknown basis"};
        launch_export(c->T, c->ld, c->d.U[c->cur], basis == RKDG_BASIS_REFERENCE ? c->d.conv_out : nullptr,
                      c->d.perm, c->d.staging, c->T, c->p.order, kprec(c), 0, c->d.jinv,
                      c->p.farfield, lo_row(c), c->stream);
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(U, sizeof(double) * ld, c->d.staging, sizeof(double) * c->T,
                                        sizeof(double) * c->T, 4 * c->nb, cudaMemcpyDeviceToHost,
                                        c->stream));
        sync(c);
    });
}

int rkdg_residual(rkdg_ctx* c, double* R, int32_t ld, int32_t basis) {
    return guarded([&] {
        if (!c || !R || ld < c->T) throw Error{RKDG_ERR_INVALID, "rkdg_residual: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        ensure_staging(c);
        if (basis == RKDG_BASIS_REFERENCE) ensure_conversion(c);
        else if (basis != RKDG_BASIS_NATIVE) throw Error{RKDG_ERR_INVALID, "unknown basis"};
        // scratch: a buffer that holds neither the current nor the saved state
        int scratch = 0;
        while (scratch == c->cur || scratch == c->old) ++scratch;
        StageArgs a = base_args(c);
        a.U = c->d.U[c->cur];
        a.U0 = nullptr;
        a.Unew = c->d.U[scratch];
        a.a = 0;
        a.b = 1;
        a.lo_row = -1;
        launch_residual(a, c->tiles, c->p.order, c->p.nq, c->p.flux, kprec(c), c->ctas, c->stream);
        launch_export(c->T, c->ld, c->d.U[scratch], basis == RKDG_BASIS_REFERENCE ? c->d.conv_in : nullptr,
                      c->d.perm, c->d.staging, c->T, c->p.order, kprec(c), 1, c->d.jinv,
                      c->p.farfield, -1, c->stream);
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(R, sizeof(double) * ld, c->d.staging, sizeof(double) * c->T,
                                        sizeof(double) * c->T, 4 * c->nb, cudaMemcpyDeviceToHost,
                                        c->stream));
        sync(c);
    });
}

int rkdg_compute_dt(rkdg_ctx* c, double* dt) {
    return guarded([&] {
        if (!c || !dt) throw Error{RKDG_ERR_INVALID, "rkdg_compute_dt: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        c->wave_valid = false;
        ensure_wave(c);
        pull_ctl(c);
        check_error_flag(c);
        double w;
        std::memcpy(&w, &c->h_ctl->wave_bits, sizeof(w));
        *dt = c->p.cfl / w;
    });
}

int rkdg_save_old(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        require_state(c);
        c->old = c->cur;
    });
}

int rkdg_stage(rkdg_ctx* c, int32_t s, double dt) {
    return guarded([&] {
        if (!c || s < 0 || s >= c->p.rk) throw Error{RKDG_ERR_INVALID, "rkdg_stage: bad stage index"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        // the stage reads dt from the control block
        pull_ctl(c);
        c->h_ctl->dt = dt;
        c->h_ctl->done = 0;
        push_ctl(c);
        const int out = stage_output(c, s);
        launch_one_stage(c, s, c->cur, c->old, out);
        c->cur = out;
        // only a last stage leaves the CFL measure of the state it wrote
        c->wave_valid = (s == c->p.rk - 1);
        sync(c);
    });
}

int rkdg_limit(rkdg_ctx* c) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        require_state(c);
        if (c->p.limiter != RKDG_LIMITER_TVB) throw Error{RKDG_ERR_INVALID, "context created without limiter"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        launch_tiled_limiter(c->tiles, 0, c->ld, c->d.U[c->cur], c->d.conn, c->d.lim, c->d.jinv,
                             nullptr, c->d.far, kprec(c), c->p.nq, c->p.gamma, c->p.tvb_m,
                             nullptr, nullptr, nullptr, 0, c->stream);
        sync(c);
    });
}

int rkdg_step(rkdg_ctx* c, double dt, double* dt_used, double* monitor) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        if (c->T_own != c->T)
            throw Error{RKDG_ERR_INVALID, "a partition context advances stage by stage (rkdg_stage) with halo exchanges"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        normalise_buffers(c);
        ensure_wave(c);
        pull_ctl(c);
        c->h_ctl->dt_fixed = dt > 0 ? dt : 0.0;
        c->h_ctl->t_final = 0.0;
        c->h_ctl->done = 0;
        push_ctl(c);
        enqueue_step(c, true);
        c->wave_valid = true;
        pull_ctl(c);
        check_error_flag(c);
        log_residual(c);
        if (dt_used) *dt_used = c->h_ctl->dt;
        if (monitor) {
            std::memcpy(&monitor[0], &c->h_ctl->mon_bits[0], sizeof(double));
            std::memcpy(&monitor[1], &c->h_ctl->mon_bits[1], sizeof(double));
        }
    });
}

int rkdg_advance(rkdg_ctx* c, int32_t nsteps, double t_final, double* t, int32_t* steps_done) {
    return guarded([&] {
        if (!c || nsteps < 0) throw Error{RKDG_ERR_INVALID, "rkdg_advance: bad arguments"};
        if (c->T_own != c->T)
            throw Error{RKDG_ERR_INVALID, "a partition context advances stage by stage (rkdg_stage) with halo exchanges"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        normalise_buffers(c);
        ensure_wave(c);
        pull_ctl(c);
        const int step0 = c->h_ctl->step;
        c->h_ctl->dt_fixed = 0.0;
        c->h_ctl->t_final = t_final > 0 ? t_final : 0.0;
        c->h_ctl->done = 0;
        push_ctl(c);
        if (c->graph && c->graph_monitor != (bool)c->reslog) {  // the history needs the monitor
            cudaGraphExecDestroy(c->graph);
            c->graph = nullptr;
        }
        if (!c->graph) {
            c->graph_monitor = (bool)c->reslog;
            c->graph = capture_steps(c, 1, c->graph_monitor);
        }
        if (!c->graph_n && !c->reslog && nsteps >= kGraphSteps) c->graph_n = capture_steps(c, kGraphSteps, false);
        if (c->reslog) {  // the history needs every step's monitor: one step per launch
            for (int i = 0; i < nsteps; ++i) {
                const int before = c->h_ctl->step;
                RKDG_CUDA_TRY(cudaGraphLaunch(c->graph, c->stream));
                pull_ctl(c);
                if (c->h_ctl->step == before || c->h_ctl->error) break;  // done or failed
                log_residual(c);
            }
            c->reslog->flush();
            nsteps = 0;
        }
        // launch in chunks; with a final time, stop once the device says done
        int left = nsteps;
        const int chunk = t_final > 0 ? 64 : nsteps;
        while (left > 0) {
            int n = std::min(left, chunk > 0 ? chunk : 1);
            for (int i = 0; i < n / kGraphSteps && c->graph_n; ++i)
                RKDG_CUDA_TRY(cudaGraphLaunch(c->graph_n, c->stream));
            for (int i = c->graph_n ? n / kGraphSteps * kGraphSteps : 0; i < n; ++i)
                RKDG_CUDA_TRY(cudaGraphLaunch(c->graph, c->stream));
            left -= n;
            if (t_final > 0 && left > 0) {
                pull_ctl(c);
                if (c->h_ctl->done || c->h_ctl->error) break;
            }
        }
        c->wave_valid = true;
        pull_ctl(c);
        check_error_flag(c);
        if (t) *t = c->h_ctl->t;
        if (steps_done) *steps_done = c->h_ctl->step - step0;
    });
}

int rkdg_time_stage(rkdg_ctx* c, int32_t s, int32_t reps, double* ms) {
    return guarded([&] {
        if (!c || !ms || s < 0 || s >= c->p.rk || reps <= 0)
            throw Error{RKDG_ERR_INVALID, "rkdg_time_stage: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        normalise_buffers(c);
        pull_ctl(c);
        if (!(c->h_ctl->dt > 0)) c->h_ctl->dt = 1e-6;
        c->h_ctl->done = 0;
        push_ctl(c);
        // input buffer 0 (the state), U^n = buffer 0, output buffer 1: a
        // stage that writes neither its input nor U^n, so launches repeat
        StageArgs a = base_args(c);
        stage_coeffs(c->p.rk, s, a.a, a.b);
        a.U = c->d.U[0];
        a.U0 = s == 0 ? nullptr : c->d.U[0];
        a.Unew = c->d.U[1];
        a.last_stage = s == (int)c->p.rk - 1;  // the last stage with its CFL/monitor epilogue
        cudaEvent_t e0, e1;
        RKDG_CUDA_TRY(cudaEventCreate(&e0));
        RKDG_CUDA_TRY(cudaEventCreate(&e1));
        launch_stage(a, c->tiles, c->p.order, c->p.nq, c->p.flux, kprec(c), c->ctas, c->stream);
        RKDG_CUDA_TRY(cudaEventRecord(e0, c->stream));
        for (int i = 0; i < reps; ++i)
            launch_stage(a, c->tiles, c->p.order, c->p.nq, c->p.flux, kprec(c), c->ctas, c->stream);
        RKDG_CUDA_TRY(cudaEventRecord(e1, c->stream));
        RKDG_CUDA_TRY(cudaEventSynchronize(e1));
        float t = 0;
        RKDG_CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = (double)t / reps;
    });
}

int rkdg_get_time(rkdg_ctx* c, double* t, int32_t* steps) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        pull_ctl(c);
        if (t) *t = c->h_ctl->t;
        if (steps) *steps = c->h_ctl->step;
    });
}

int rkdg_set_time(rkdg_ctx* c, double t) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        pull_ctl(c);
        c->h_ctl->t = t;
        c->h_ctl->done = 0;
        push_ctl(c);
        sync(c);
    });
}

int rkdg_conservation_totals(rkdg_ctx* c, double totals[4]) {
    return guarded([&] {
        if (!c || !totals) throw Error{RKDG_ERR_INVALID, "bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        const int n = totals_partial_count(c->T_own);
        double* out4 = c->d.partial + (size_t)4 * n;
        launch_totals(c->T_own, c->ld, c->d.U[c->cur], c->p.order, kprec(c), c->d.jinv,
                      c->d.partial, out4, c->p.farfield, lo_row(c), c->stream);
        RKDG_CUDA_TRY(cudaMemcpyAsync(totals, out4, 4 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        sync(c);
    });
}

int rkdg_write_solution(rkdg_ctx* c, const char* path) {
    return guarded([&] {
        if (!c || !path) throw Error{RKDG_ERR_INVALID, "bad arguments"};
        require_state(c);
        const int T = c->T, nb = c->nb;
        std::vector<double> U((size_t)4 * nb * T);
        int rc = rkdg_get_state(c, U.data(), T, RKDG_BASIS_NATIVE);
        if (rc != RKDG_OK) throw Error{rc, g_last_error};
        std::ofstream f(path);
        if (!f) throw Error{RKDG_ERR_IO, std::string("cannot open ") + path};
        // CCUDARkdgSolver::outputSolution (src/cudarkdgsolver.cu:860-1001):
        // Tecplot FETRIANGLE, BLOCK packing, nodal X/Y then cell-centred
        // rho, u, v, p, Ma, FLAG; six values per line with a line break after
        // the first value; 1-based connectivity.
        const double gamma = c->p.gamma;
        const std::vector<double>& V = c->mesh.vertices;
        const int vnum = (int)(V.size() / 2);
        auto mean = [&](int v, int t) { return U[(size_t)v * nb * T + t]; };
        f << "TITLE=RKDG" << std::endl;
        f << "VARIABLES=X , Y , rho , u , v , p, Ma , FLAG" << std::endl;
        f << "ZONE T= T1 N= " << vnum << " , E= " << T << " , ZONETYPE=FETRIANGLE" << std::endl;
        f << "DATAPACKING=BLOCK" << std::endl;
        f << "VARLOCATION=([1-2]=NODAL,[3-8]=CELLCENTERED)" << std::endl;
        f << "DT=(SINGLE SINGLE SINGLE SINGLE SINGLE SINGLE SINGLE SINGLE)" << std::endl;
        for (int i = 0; i < vnum; ++i) {
            f << V[2 * i] << "  ";
            if (i % 6 == 0) f << std::endl;
        }
        for (int i = 0; i < vnum; ++i) {
            f << V[2 * i + 1] << "  ";
            if (i % 6 == 0) f << std::endl;
        }
        f << std::endl;
        auto column = [&](auto value) {
            for (int i = 0; i < T; ++i) {
                f << value(i) << "  ";
                if (i % 6 == 0) f << std::endl;
            }
            f << std::endl;
        };
        column([&](int i) { return mean(0, i); });
        column([&](int i) { return mean(1, i) / mean(0, i); });
        column([&](int i) { return mean(2, i) / mean(0, i); });
        auto pres = [&](int i) {
            double rho = mean(0, i), u = mean(1, i) / rho, v = mean(2, i) / rho;
            return (gamma - 1) * (mean(3, i) - 0.5 * rho * (u * u + v * v));
        };
        column(pres);
        column([&](int i) {
            double rho = mean(0, i), u = mean(1, i) / rho, v = mean(2, i) / rho;
            return std::sqrt(u * u + v * v) / std::sqrt(gamma * pres(i) / rho);
        });
        for (int i = 0; i < T; ++i) {
            f << "1" << "  ";
            if (i % 6 == 0) f << std::endl;
        }
        f << std::endl;
        const std::vector<int32_t>& tv = c->mesh.tri_vertex;
        for (int i = 0; i < T; ++i)
            f << tv[3 * i] + 1 << "    " << tv[3 * i + 1] + 1 << "    " << tv[3 * i + 2] + 1 << std::endl;
        if (!f) throw Error{RKDG_ERR_IO, std::string("write failed: ") + path};
    });
}

}  // extern "C"

// ------------------------------------------------------ checkpoint / resume
namespace {

// Version 2 also records the method (rules, flux, limiter, RK scheme) and
// the physics (gamma, CFL number, TVB constant) the saved CFL wave maximum
// and state belong to; a context with other settings refuses the file.
struct CheckpointHeader {
    char magic[8];
    uint32_t version;
    int32_t ntri, order, nbasis, precision, packs;
    uint64_t mesh_hash;
    double t;
    int32_t step, pad;
    unsigned long long wave_bits, mon_bits[2];
    double farfield[4];
    int32_t nq, ng, flux, limiter, rk, pad2;
    double gamma, cfl, tvb_m;
};
constexpr uint32_t kCkptVersion = 2;
constexpr char kCkptMagic[8] = {'R', 'K', 'D', 'G', 'C', 'K', 'P', '1'};

// FNV-1a over the internal-order vertex coordinates of every triangle: the
// same caller mesh and ordering setting give the same value.
uint64_t mesh_hash(const HostMesh& m) {
    uint64_t h = 1469598103934665603ull;
    const unsigned char* b = reinterpret_cast<const unsigned char*>(m.xy.data());
    for (size_t i = 0; i < m.xy.size() * sizeof(double); ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

// 16-byte packs per element in the state layout
int state_packs(const rkdg_ctx* c) { return state_rows(c->p.precision, c->nb); }

}  // namespace

int rkdg_checkpoint_save(rkdg_ctx* c, const char* path) {
    return guarded([&] {
        if (!c || !path) throw Error{RKDG_ERR_INVALID, "rkdg_checkpoint_save: bad arguments"};
        require_state(c);
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        ensure_wave(c);
        pull_ctl(c);
        const int packs = state_packs(c);
        std::vector<unsigned char> rows((size_t)packs * c->T * 16);
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(rows.data(), (size_t)c->T * 16, c->d.U[c->cur], (size_t)c->ld * 16,
                                        (size_t)c->T * 16, packs, cudaMemcpyDeviceToHost, c->stream));
        sync(c);
        CheckpointHeader h{};
        std::memcpy(h.magic, kCkptMagic, 8);
        h.version = kCkptVersion;
        h.ntri = c->T;
        h.order = c->p.order;
        h.nbasis = c->nb;
        h.precision = c->p.precision;
        h.packs = packs;
        h.mesh_hash = mesh_hash(c->mesh);
        h.t = c->h_ctl->t;
        h.step = c->h_ctl->step;
        h.wave_bits = c->h_ctl->wave_bits;
        h.mon_bits[0] = c->h_ctl->mon_bits[0];
        h.mon_bits[1] = c->h_ctl->mon_bits[1];
        for (int v = 0; v < 4; ++v) h.farfield[v] = c->p.farfield[v];
        h.nq = c->p.nq;
        h.ng = c->p.ng;
        h.flux = c->p.flux;
        h.limiter = c->p.limiter;
        h.rk = c->p.rk;
        h.gamma = c->p.gamma;
        h.cfl = c->p.cfl;
        h.tvb_m = c->p.tvb_m;
        std::ofstream f(path, std::ios::binary);
        if (!f) throw Error{RKDG_ERR_IO, std::string("cannot open ") + path + " for writing"};
        f.write(reinterpret_cast<const char*>(&h), sizeof(h));
        f.write(reinterpret_cast<const char*>(rows.data()), (std::streamsize)rows.size());
        if (!f) throw Error{RKDG_ERR_IO, std::string("write to ") + path + " failed"};
    });
}

int rkdg_checkpoint_load(rkdg_ctx* c, const char* path) {
    return guarded([&] {
        if (!c || !path) throw Error{RKDG_ERR_INVALID, "rkdg_checkpoint_load: bad arguments"};
        std::ifstream f(path, std::ios::binary);
        if (!f) throw Error{RKDG_ERR_IO, std::string("cannot open ") + path};
        CheckpointHeader h{};
        f.read(reinterpret_cast<char*>(&h), sizeof(h));
        if (!f) throw Error{RKDG_ERR_IO, std::string("short read from ") + path};
        if (std::memcmp(h.magic, kCkptMagic, 8) != 0 || h.version != kCkptVersion)
            throw Error{RKDG_ERR_INVALID, std::string(path) + " is not a checkpoint of this format"};
        const int packs = state_packs(c);
        if (h.ntri != c->T || h.order != c->p.order || h.precision != c->p.precision || h.packs != packs)
            throw Error{RKDG_ERR_INVALID, "checkpoint was written for another triangle count, order or precision"};
        if (h.mesh_hash != mesh_hash(c->mesh))
            throw Error{RKDG_ERR_INVALID, "checkpoint was written for another mesh (or triangle ordering)"};
        if (h.nq != c->p.nq || h.ng != c->p.ng || h.flux != c->p.flux || h.limiter != c->p.limiter ||
            h.rk != c->p.rk || h.gamma != c->p.gamma || h.cfl != c->p.cfl ||
            (c->p.limiter != RKDG_LIMITER_NONE && h.tvb_m != c->p.tvb_m))
            throw Error{RKDG_ERR_INVALID,
                        "checkpoint was written with another method or physics (rules, flux, limiter, RK "
                        "scheme, gamma, CFL number or TVB constant)"};
        if (c->p.precision != RKDG_FP64)
            for (int v = 0; v < 4; ++v)
                if (h.farfield[v] != c->p.farfield[v])
                    throw Error{RKDG_ERR_INVALID, "FP32 checkpoint was written with another far-field state"};
        std::vector<unsigned char> rows((size_t)packs * c->T * 16);
        f.read(reinterpret_cast<char*>(rows.data()), (std::streamsize)rows.size());
        if (!f) throw Error{RKDG_ERR_IO, std::string("short read from ") + path};
        RKDG_CUDA_TRY(cudaSetDevice(c->device));
        RKDG_CUDA_TRY(cudaMemcpy2DAsync(c->d.U[0], (size_t)c->ld * 16, rows.data(), (size_t)c->T * 16,
                                        (size_t)c->T * 16, packs, cudaMemcpyHostToDevice, c->stream));
        c->cur = 0;
        c->old = 0;
        pull_ctl(c);
        c->h_ctl->t = h.t;
        c->h_ctl->step = h.step;
        c->h_ctl->wave_bits = h.wave_bits;
        c->h_ctl->mon_bits[0] = h.mon_bits[0];
        c->h_ctl->mon_bits[1] = h.mon_bits[1];
        c->h_ctl->done = 0;
        c->h_ctl->error = 0;
        push_ctl(c);
        sync(c);
        c->wave_valid = true;
        c->have_state = true;
    });
}

int rkdg_set_residual_log(rkdg_ctx* c, const char* path) {
    return guarded([&] {
        if (!c) throw Error{RKDG_ERR_INVALID, "null context"};
        c->reslog.reset();
        if (!path) return;
        auto f = std::make_unique<std::ofstream>(path);
        if (!*f) throw Error{RKDG_ERR_IO, std::string("cannot open ") + path};
        *f << "N, rho" << std::endl;  // src/rkdgadvance.cpp:10-17
        f->precision(10);
        c->reslog = std::move(f);
    });
}

int rkdg_wait_selftest(double limit_s, int32_t* timed_out, double* waited_s) {
    return guarded([&] {
        if (!timed_out || !waited_s || !(limit_s > 0) || limit_s > 10)
            throw Error{RKDG_ERR_INVALID, "rkdg_wait_selftest: limit must be in (0, 10] s"};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{RKDG_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
        }
        int t = 0;
        wait_selftest(limit_s, &t, waited_s);
        *timed_out = t;
    });
}
