// Serving: a request loop with HBM-budget admission and continuous batching
// (include/rkdg.h, rkdg_server_*).
//
// The pool is allocated once from the budget: per-element arrays (three
// state buffers in the P2 row layout, J^-1, tile codes, global connectivity,
// limiter geometry, caller permutation), halo and flux-task pools, tile
// descriptors and per-slot control blocks.  Admission places a request's
// elements, halo entries and tasks in free ranges (first fit), uploads its
// tables and state, and adds its tiles to the active descriptor list.  The
// engine thread launches a captured graph of whole steps over the active
// tiles (the tile count is read on the device, so membership changes need
// no recapture), checks the per-solve done flags between chunks of steps,
// and retires finished solves.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rkdg_internal.hpp"

using namespace rkdg;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

// First-fit free list over [0, capacity) with coalescing.
class RangeAlloc {
  public:
    explicit RangeAlloc(int64_t cap = 0) { reset(cap); }
    void reset(int64_t cap) {
        free_.clear();
        if (cap > 0) free_[0] = cap;
    }
    int64_t alloc(int64_t n) {
        if (n <= 0) return 0;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= n) {
                int64_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[off + n] = len - n;
                return off;
            }
        }
        return -1;
    }
    void release(int64_t off, int64_t n) {
        if (n <= 0) return;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

  private:
    std::map<int64_t, int64_t> free_;
};

enum { REQ_QUEUED = 0, REQ_RUNNING = 1, REQ_DONE = 2, REQ_FAILED = 3 };

// element ranges start on 32-element boundaries: a warp's 16-byte packs then
// cover whole 512-byte segments
constexpr int64_t kElemAlign = 32;
int64_t elem_span(int T) { return (T + kElemAlign - 1) / kElemAlign * kElemAlign; }
constexpr int kPoolHalo = 160;  // halo entries per tile the pool's kernels stage

// The pool's active tiles are kept in four lists, one per (flux, order):
// list 2 flux + 0 holds P2 tiles, 2 flux + 1 P1 tiles, so each list runs the
// single-order kernel for its tiles (P1 kernels hold more warps per SM).
constexpr int kLists = 4;
int list_of(int flux, int order) { return 2 * flux + (order == 2 ? 0 : 1); }
int list_flux(int l) { return l / 2; }
int list_order(int l) { return l % 2 == 0 ? 2 : 1; }

struct Request {
    int64_t id = 0;
    int order = 2, nb = 6, T = 0;
    int flux = RKDG_FLUX_LLF;
    bool limiter = false;
    double t_final = 0, far[4] = {0, 0, 0, 0};
    std::vector<double> jinv;   // [T][4]
    std::vector<double> lim;    // [T][3][2]
    std::vector<int32_t> conn;  // [T][4] local neighbours + packed info
    std::vector<int32_t> perm;
    TileTables tiles;           // offsets 0
    std::vector<double> U0;     // [4][nb][T]
    std::vector<double> result;
    int status = REQ_QUEUED;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int steps = 0, step_seen = 0;
    int slot = -1;
    int64_t e_off = -1, h_off = -1, k_off = -1;
    std::string error;
    int error_code = RKDG_ERR_STATE;
};

}  // namespace

struct rkdg_server {
    rkdg_params p{};
    int device = 0, word = 4, max_slots = 0, ctas[kLists] = {0, 0, 0, 0};
    int64_t cap = 0, hcap = 0, kcap = 0, tcap = 0, max_T = 0;
    int ld = 0;
    size_t bytes = 0;
    // device pool
    void* U[3] = {nullptr, nullptr, nullptr};
    double* jinv = nullptr;
    int4* tcode = nullptr;
    int4* conn = nullptr;
    void* lim = nullptr;
    int32_t* perm = nullptr;
    int2* halo = nullptr;
    uint16_t* task = nullptr;
    int4* desc = nullptr;
    int* ntiles_dev = nullptr;   // [kLists]: active tiles of each list
    StepCtl* ctl = nullptr;
    double* far = nullptr;
    int* flags = nullptr;
    int* tile_flags = nullptr;   // [kLists][tcap] the stage kernel's per-tile limiter test, per list
    int* tile_list = nullptr;    // [kLists][kListHead + tcap] the tiles each list's limiter visits
    double* staging = nullptr;
    StepCtl* h_ctl = nullptr;
    cudaStream_t stream = nullptr;
    cudaStream_t side[kLists - 1] = {nullptr, nullptr, nullptr};  // lists 1.., forked and joined per stage
    cudaEvent_t ev_fork = nullptr, ev_join[kLists - 1] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t graph = nullptr;
    TileArgs tiles[kLists]{};  // per list (flux, order)
    // host state
    RangeAlloc elems, halos, tasks;
    std::vector<int> free_slots;
    std::vector<std::shared_ptr<Request>> active;  // by slot
    std::deque<std::shared_ptr<Request>> queue;
    std::map<int64_t, std::shared_ptr<Request>> reqs;
    int64_t next_id = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread engine;
    bool stop = false;
    std::string fatal;         // set when the engine thread has stopped on an error
    int fatal_code = RKDG_OK;
    int fault_after = -1;      // rkdg_server_inject_fault: chunks left before a simulated failure
    bool tiles_dirty = false;
    int ntiles[kLists] = {0, 0, 0, 0};
    // stats
    double dof_updates = 0, busy = 0;
    double t_admit = 0, t_retire = 0;  // engine seconds spent uploading and retiring requests
    int64_t chunks = 0;
    int64_t completed = 0;
    int peak = 0;
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

void* salloc(rkdg_server* s, size_t bytes) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes ? bytes : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{RKDG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed: " +
                                        cudaGetErrorString(e)};
    }
    s->bytes += bytes;
    return p;
}

// the P2 row layout for every request (RKDG_FP32C: row 6 holds the low
// parts of the cell means)
size_t state_bytes(const rkdg_server* s) { return (size_t)16 * state_rows(s->p.precision, 6) * s->ld; }
int kprec(const rkdg_server* s) { return kernel_prec(s->p.precision); }
int lo_row(const rkdg_server* s) { return s->p.precision == RKDG_FP32C ? 6 : -1; }

void coeffs(int rk, int st, double& a, double& c) {
    if (st == 0) a = 0, c = 1;
    else if (rk == 2) a = 0.5, c = 0.5;
    else if (st == 1) a = 0.75, c = 0.25;
    else a = 1.0 / 3.0, c = 2.0 / 3.0;
}

// One step of every solve in flight: per RK stage, the stage kernel and the
// limiter over each tile list (flux, order), the first on the server's
// stream and the others on streams forked from it (the lists hold different
// solves, so the launches overlap where one runs out), joined before the
// next stage.
void enqueue_step(rkdg_server* s) {
    launch_step_begin(s->ctl, s->max_slots, s->stream);
    const int plan[3][3] = {{0, 0, 1}, {1, 0, 2}, {2, 0, 0}};
    const int plan2[2][3] = {{0, 0, 1}, {1, 0, 0}};
    for (int st = 0; st < s->p.rk; ++st) {
        const int* pl = s->p.rk == 3 ? plan[st] : plan2[st];
        StageArgs a{};
        a.T = (int)s->cap;
        a.ld = s->ld;
        a.jinv = s->jinv;
        a.ctl = s->ctl;
        a.gamma = s->p.gamma;
        for (int v = 0; v < 4; ++v) a.far[v] = s->p.farfield[v];
        a.far_sid = s->far;
        coeffs(s->p.rk, st, a.a, a.b);
        a.U = s->U[pl[0]];
        a.U0 = st == 0 ? nullptr : s->U[pl[1]];
        a.Unew = s->U[pl[2]];
        a.last_stage = st == s->p.rk - 1;
        a.lo_row = lo_row(s);
        a.tvb_m = s->p.tvb_m;
        a.limiter_on = s->flags;
        RKDG_CUDA_TRY(cudaEventRecord(s->ev_fork, s->stream));
        for (int l = 1; l < kLists; ++l) RKDG_CUDA_TRY(cudaStreamWaitEvent(s->side[l - 1], s->ev_fork, 0));
        for (int l = 0; l < kLists; ++l) {
            cudaStream_t st_l = l == 0 ? s->stream : s->side[l - 1];
            a.tile_flags = s->tile_flags + l * s->tcap;
            a.tile_list = s->tile_list + l * (kListHead + s->tcap);
            a.tile_cap = (int)s->tcap;
            launch_stage(a, s->tiles[l], list_order(l), s->p.nq, list_flux(l), kprec(s), s->ctas[l], st_l);
            launch_tiled_limiter(s->tiles[l], s->ctas[l], s->ld, s->U[pl[2]], s->conn, s->lim, s->jinv, s->flags,
                                 s->far, kprec(s), s->p.nq, s->p.gamma, s->p.tvb_m, s->ctl, a.tile_flags,
                                 a.tile_list, a.tile_cap, st_l);
        }
        for (int l = 1; l < kLists; ++l) {
            RKDG_CUDA_TRY(cudaEventRecord(s->ev_join[l - 1], s->side[l - 1]));
            RKDG_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->ev_join[l - 1], 0));
        }
    }
}

template <class T>
void h2d(rkdg_server* s, T* dst, const T* src, size_t n) {
    if (n) RKDG_CUDA_TRY(cudaMemcpyAsync(dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, s->stream));
}

// Places and uploads one request (engine thread, caller holds no lock on
// device work; the request's host data is owned by the engine from here).
void upload(rkdg_server* s, Request& r) {
    const int T = r.T;
    const int64_t e = r.e_off;
    std::vector<double> j0(2 * (size_t)T), j1(2 * (size_t)T);
    for (int t = 0; t < T; ++t) {
        j0[2 * t] = r.jinv[4 * t];
        j0[2 * t + 1] = r.jinv[4 * t + 1];
        j1[2 * t] = r.jinv[4 * t + 2];
        j1[2 * t + 1] = r.jinv[4 * t + 3];
    }
    h2d(s, s->jinv + 2 * e, j0.data(), j0.size());
    h2d(s, s->jinv + 2 * ((int64_t)s->ld + e), j1.data(), j1.size());
    h2d(s, reinterpret_cast<int32_t*>(s->tcode) + 4 * e, r.tiles.code.data(), r.tiles.code.size());
    std::vector<int32_t> cn(r.conn);
    for (int t = 0; t < T; ++t)
        for (int k = 0; k < 3; ++k)
            if (cn[4 * t + k] >= 0) cn[4 * t + k] += (int32_t)e;
    h2d(s, reinterpret_cast<int32_t*>(s->conn) + 4 * e, cn.data(), cn.size());
    if (r.limiter) upload_limiter(s->lim, s->ld, e, r.lim, T, kprec(s), s->stream);
    h2d(s, s->perm + e, r.perm.data(), r.perm.size());
    std::vector<int32_t> hl(r.tiles.halo);
    for (size_t i = 0; i < hl.size(); i += 2) hl[i] += (int32_t)e;
    h2d(s, reinterpret_cast<int32_t*>(s->halo) + 2 * r.h_off, hl.data(), hl.size());
    h2d(s, s->task + r.k_off, r.tiles.task.data(), r.tiles.task.size());
    // state (native basis, caller order) -> pool
    RKDG_CUDA_TRY(cudaMemcpyAsync(s->staging, r.U0.data(), sizeof(double) * r.U0.size(),
                                  cudaMemcpyHostToDevice, s->stream));
    launch_import(T, s->ld, s->staging, T, nullptr, s->perm + e, static_cast<char*>(s->U[0]) + 16 * e,
                  r.order, kprec(s), r.far, lo_row(s), s->stream);
    StepCtl c{};
    c.cfl = s->p.cfl;
    c.t_final = r.t_final > 0 ? r.t_final : 1e-300;
    h2d(s, s->ctl + r.slot, &c, 1);
    h2d(s, s->far + 4 * r.slot, r.far, 4);
    int flag = r.limiter ? 1 : 0;
    h2d(s, s->flags + r.slot, &flag, 1);
    RKDG_CUDA_TRY(cudaStreamSynchronize(s->stream));  // host buffers above are temporaries
    r.U0.clear();
    r.U0.shrink_to_fit();
}

// Relocated descriptors of one request's tiles, appended to d.
void relocate(const Request& r, std::vector<int32_t>& d) {
    const auto& td = r.tiles.desc;
    for (size_t i = 0; i < td.size(); i += 8) {
        d.push_back(td[i] + (int32_t)r.e_off);
        d.push_back(td[i + 1]);
        d.push_back(r.slot);
        d.push_back(td[i + 3]);
        d.push_back(td[i + 4] + (int32_t)r.h_off);
        d.push_back(td[i + 5]);
        d.push_back(td[i + 6] + (int32_t)r.k_off);
        d.push_back(td[i + 7]);
    }
}

// Rewrites the active tile lists (per flux and order) and measures the CFL
// wave speed of the newly admitted solves over their own tiles only, so the
// solves already in flight keep the value their last stage computed.
void rebuild_tiles(rkdg_server* s, const std::vector<std::shared_ptr<Request>>& fresh) {
    std::vector<int32_t> d[kLists], dn;
    for (auto& r : s->active)
        if (r) relocate(*r, d[list_of(r->flux, r->order)]);
    for (auto& r : fresh) relocate(*r, dn);
    for (int l = 0; l < kLists; ++l) {
        s->ntiles[l] = (int)(d[l].size() / 8);
        h2d(s, reinterpret_cast<int32_t*>(const_cast<int4*>(s->tiles[l].desc)), d[l].data(), d[l].size());
    }
    h2d(s, s->ntiles_dev, s->ntiles, kLists);
    if (!dn.empty()) {
        int4* scratch = s->desc + 2 * kLists * s->tcap;
        h2d(s, reinterpret_cast<int32_t*>(scratch), dn.data(), dn.size());
        TileArgs t = s->tiles[0];
        t.desc = scratch;
        t.ntiles = (int)(dn.size() / 8);
        t.ntiles_dev = nullptr;
        launch_wave(t, s->ld, s->U[0], kprec(s), s->jinv, s->p.gamma, s->ctl, 0, s->far, s->stream);
    }
    RKDG_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->tiles_dirty = false;
}

void retire(rkdg_server* s, Request& r, bool failed) {
    if (!failed) {
        r.result.assign((size_t)4 * r.nb * r.T, 0.0);
        launch_export(r.T, s->ld, static_cast<char*>(s->U[0]) + 16 * r.e_off, nullptr, s->perm + r.e_off,
                      s->staging, r.T, r.order, kprec(s), 0, nullptr, r.far, lo_row(s), s->stream);
        RKDG_CUDA_TRY(cudaMemcpyAsync(r.result.data(), s->staging, sizeof(double) * r.result.size(),
                                      cudaMemcpyDeviceToHost, s->stream));
        RKDG_CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    // the slot stops doing work: done flag set, no tiles after the rebuild
    StepCtl c{};
    c.done = 1;
    h2d(s, s->ctl + r.slot, &c, 1);
    std::lock_guard<std::mutex> lk(s->mu);
    s->elems.release(r.e_off, elem_span(r.T));
    s->halos.release(r.h_off, (int64_t)r.tiles.halo.size() / 2);
    s->tasks.release(r.k_off, (int64_t)r.tiles.task.size());
    s->free_slots.push_back(r.slot);
    s->active[r.slot].reset();
    r.t_done = now_s();
    r.status = failed ? REQ_FAILED : REQ_DONE;
    if (failed) {
        try {
            throw_ctl_error(s->h_ctl[r.slot].error, "request " + std::to_string(r.id));
        } catch (const Error& e) {
            r.error = e.msg;
            r.error_code = e.code;
        }
    }
    r.tiles = TileTables();
    r.jinv.clear();
    r.lim.clear();
    r.conn.clear();
    if (!failed) ++s->completed;
    s->tiles_dirty = true;
    s->cv_done.notify_all();
}

// Moves queued requests that fit into the pool (skip-ahead: a large request
// at the head does not block smaller ones behind it).
std::vector<std::shared_ptr<Request>> admit(rkdg_server* s) {
    std::vector<std::shared_ptr<Request>> in;
    for (auto it = s->queue.begin(); it != s->queue.end();) {
        Request& r = **it;
        if (s->free_slots.empty()) break;
        const int64_t nh = (int64_t)r.tiles.halo.size() / 2, nk = (int64_t)r.tiles.task.size();
        int64_t e = s->elems.alloc(elem_span(r.T));
        if (e < 0) {
            ++it;
            continue;
        }
        int64_t h = s->halos.alloc(nh);
        if (h < 0) {
            s->elems.release(e, elem_span(r.T));
            ++it;
            continue;
        }
        int64_t k = s->tasks.alloc(nk);
        if (k < 0) {
            s->elems.release(e, elem_span(r.T));
            s->halos.release(h, nh);
            ++it;
            continue;
        }
        r.e_off = e;
        r.h_off = h;
        r.k_off = k;
        r.slot = s->free_slots.back();
        s->free_slots.pop_back();
        r.status = REQ_RUNNING;
        r.t_admit = now_s();
        s->active[r.slot] = *it;
        in.push_back(*it);
        it = s->queue.erase(it);
    }
    return in;
}

void engine_loop(rkdg_server* s) {
    try {
        RKDG_CUDA_TRY(cudaSetDevice(s->device));
        const int chunk = 4;
        while (true) {
            std::vector<std::shared_ptr<Request>> in;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                s->cv_work.wait(lk, [&] {
                    if (s->stop) return true;
                    bool any = false;
                    for (auto& r : s->active) any = any || (bool)r;
                    return any || !s->queue.empty();
                });
                if (s->stop) return;
                in = admit(s);
            }
            const double ta = now_s();
            for (auto& r : in) upload(s, *r);
            if (!in.empty() || s->tiles_dirty) rebuild_tiles(s, in);
            const double tb = now_s();
            int in_flight = 0;
            for (auto& r : s->active) in_flight += r ? 1 : 0;
            if (in_flight == 0) continue;
            s->peak = std::max(s->peak, in_flight);
            {
                std::lock_guard<std::mutex> lk(s->mu);
                if (s->fault_after == 0) throw Error{RKDG_ERR_CUDA, "engine stopped by rkdg_server_inject_fault"};
                if (s->fault_after > 0) --s->fault_after;
            }
            const double t0 = now_s();
            for (int i = 0; i < chunk; ++i) RKDG_CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
            RKDG_CUDA_TRY(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(StepCtl) * s->max_slots,
                                          cudaMemcpyDeviceToHost, s->stream));
            RKDG_CUDA_TRY(cudaStreamSynchronize(s->stream));
            const double t1 = now_s();
            std::vector<std::shared_ptr<Request>> done;
            {
                std::lock_guard<std::mutex> lk(s->mu);
                s->busy += t1 - t0;
                s->t_admit += tb - ta;
                ++s->chunks;
                for (auto& r : s->active) {
                    if (!r) continue;
                    const StepCtl& c = s->h_ctl[r->slot];
                    const int ns = c.step - r->step_seen;
                    r->step_seen = c.step;
                    r->steps = c.step;
                    s->dof_updates += (double)ns * s->p.rk * 4 * r->nb * r->T;
                    if (c.done || c.error) done.push_back(r);
                }
            }
            const double tr = now_s();
            for (auto& r : done) retire(s, *r, s->h_ctl[r->slot].error != 0);
            if (!done.empty()) {
                std::lock_guard<std::mutex> lk(s->mu);
                s->t_retire += now_s() - tr;
            }
        }
    } catch (const Error& e) {
        std::lock_guard<std::mutex> lk(s->mu);
        s->fatal = e.msg;
        s->fatal_code = e.code;
        for (auto& r : s->active)
            if (r) r->status = REQ_FAILED, r->error = e.msg, r->error_code = e.code;
        for (auto& r : s->queue) r->status = REQ_FAILED, r->error = e.msg, r->error_code = e.code;
        s->queue.clear();
        s->cv_done.notify_all();
    }
}

void destroy_server(rkdg_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->engine.joinable()) s->engine.join();
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    for (void* p : {s->U[0], s->U[1], s->U[2], (void*)s->jinv, (void*)s->tcode, (void*)s->conn, (void*)s->lim,
                    (void*)s->perm, (void*)s->halo, (void*)s->task, (void*)s->desc, (void*)s->ntiles_dev,
                    (void*)s->ctl, (void*)s->far, (void*)s->flags, (void*)s->tile_flags, (void*)s->tile_list,
                    (void*)s->staging})
        cudaFree(p);
    if (s->h_ctl) cudaFreeHost(s->h_ctl);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    for (int l = 0; l < kLists - 1; ++l) {
        if (s->ev_join[l]) cudaEventDestroy(s->ev_join[l]);
        if (s->side[l]) cudaStreamDestroy(s->side[l]);
    }
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

}  // namespace

extern "C" {

double rkdg_server_clock(void) { return now_s(); }

int rkdg_server_create(const rkdg_params* params, size_t budget, int32_t max_slots, rkdg_server** out) {
    rkdg_server* s = nullptr;
    int rc = guarded([&] {
        if (!params || !out || max_slots <= 0) throw Error{RKDG_ERR_INVALID, "rkdg_server_create: bad arguments"};
        *out = nullptr;
        const rkdg_params& p = *params;
        if (p.nq != 6) throw Error{RKDG_ERR_INVALID, "the server runs P2 tiles with nq 6"};
        if (p.rk != 2 && p.rk != 3) throw Error{RKDG_ERR_INVALID, "rk must be 2 or 3"};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error{RKDG_ERR_NODEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e)};
        }
        cudaDeviceProp prop;
        RKDG_CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
        if (prop.major < 10) throw Error{RKDG_ERR_NODEVICE, "this library is built for sm_100a"};
        s = new rkdg_server();
        s->p = p;
        s->device = dev;
        s->word = p.precision == RKDG_FP64 ? 8 : 4;
        s->max_slots = max_slots;
        // per element: 3 state buffers (P2 rows), J^-1, tile codes, connectivity,
        // limiter geometry, permutation, ~1 halo entry, 2 task entries, descriptors
        // bytes per pooled element: 3 state buffers (P2 rows), J^-1, tile
        // codes, connectivity, limiter geometry, permutation, one halo entry,
        // three flux tasks, tile descriptors, flags and lists (2 bytes: 192
        // per tile); plus the FP64 staging buffer of the largest admissible
        // request and a fixed reserve
        const size_t per_elem = (size_t)3 * 16 * state_rows(p.precision, 6) + 32 + 16 + 16 +
                                (kernel_prec(p.precision) == RKDG_FP64 ? 48 : 24) + 4 + 8 + 6 + 2;
        const size_t fixed = (size_t)64 << 20, stage_per_elem = 24 * sizeof(double);
        if (budget < fixed + 4096 * (per_elem + stage_per_elem))
            throw Error{RKDG_ERR_NOMEM, "HBM budget too small"};
        // the staging buffer holds a request as large as the pool, up to 2^21 triangles
        const size_t avail = budget - fixed;
        const int64_t kMaxRequest = (int64_t)1 << 21;
        int64_t cap = (int64_t)(avail / (per_elem + stage_per_elem));
        if (cap > kMaxRequest) cap = (int64_t)((avail - stage_per_elem * (size_t)kMaxRequest) / per_elem);
        s->cap = std::min<int64_t>(cap / 128 * 128, (int64_t)1 << 30);
        s->max_T = std::min(s->cap, kMaxRequest);
        s->ld = (int)s->cap;
        s->hcap = s->cap;
        s->kcap = 3 * s->cap;
        s->tcap = s->cap / 128 + 2 * (int64_t)max_slots + 16;
        RKDG_CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        RKDG_CUDA_TRY(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming));
        for (int l = 0; l < kLists - 1; ++l) {
            RKDG_CUDA_TRY(cudaStreamCreateWithFlags(&s->side[l], cudaStreamNonBlocking));
            RKDG_CUDA_TRY(cudaEventCreateWithFlags(&s->ev_join[l], cudaEventDisableTiming));
        }
        upload_tables(6, 3);
        upload_tables(3, 2);
        for (int k = 0; k < 3; ++k) {
            s->U[k] = salloc(s, state_bytes(s));
            RKDG_CUDA_TRY(cudaMemsetAsync(s->U[k], 0, state_bytes(s), s->stream));
        }
        s->jinv = (double*)salloc(s, sizeof(double) * 4 * (size_t)s->ld);
        RKDG_CUDA_TRY(cudaMemsetAsync(s->jinv, 0, sizeof(double) * 4 * (size_t)s->ld, s->stream));
        s->tcode = (int4*)salloc(s, sizeof(int4) * (size_t)s->cap);
        s->conn = (int4*)salloc(s, sizeof(int4) * (size_t)s->cap);
        s->lim = salloc(s, (size_t)3 * s->ld * (kernel_prec(p.precision) == RKDG_FP64 ? 16 : 8));
        s->perm = (int32_t*)salloc(s, sizeof(int32_t) * (size_t)s->cap);
        s->halo = (int2*)salloc(s, sizeof(int2) * (size_t)s->hcap + kTablePad);
        s->task = (uint16_t*)salloc(s, sizeof(uint16_t) * (size_t)s->kcap + kTablePad);
        // the lists' descriptors and the admission scratch, 2 int4 per tile each
        s->desc = (int4*)salloc(s, sizeof(int4) * 2 * (kLists + 1) * (size_t)s->tcap);
        s->ntiles_dev = (int*)salloc(s, kLists * sizeof(int));
        RKDG_CUDA_TRY(cudaMemsetAsync(s->ntiles_dev, 0, kLists * sizeof(int), s->stream));
        s->ctl = (StepCtl*)salloc(s, sizeof(StepCtl) * max_slots);
        std::vector<StepCtl> c(max_slots);
        for (auto& x : c) {
            std::memset(&x, 0, sizeof(x));
            x.done = 1;
            x.cfl = p.cfl;
        }
        h2d(s, s->ctl, c.data(), c.size());
        s->far = (double*)salloc(s, sizeof(double) * 4 * max_slots);
        std::vector<double> f(4 * (size_t)max_slots);
        for (int i = 0; i < max_slots; ++i)
            for (int v = 0; v < 4; ++v) f[4 * i + v] = p.farfield[v];
        h2d(s, s->far, f.data(), f.size());
        s->flags = (int*)salloc(s, sizeof(int) * max_slots);
        s->tile_flags = (int*)salloc(s, sizeof(int) * kLists * (size_t)s->tcap);
        s->tile_list = (int*)salloc(s, sizeof(int) * kLists * (kListHead + (size_t)s->tcap));
        RKDG_CUDA_TRY(cudaMemsetAsync(s->flags, 0, sizeof(int) * max_slots, s->stream));
        RKDG_CUDA_TRY(cudaMemsetAsync(s->tile_flags, 0, sizeof(int) * kLists * (size_t)s->tcap, s->stream));
        RKDG_CUDA_TRY(cudaMemsetAsync(s->tile_list, 0, sizeof(int) * kLists * (kListHead + (size_t)s->tcap),
                                      s->stream));
        s->staging = (double*)salloc(s, sizeof(double) * 24 * (size_t)s->max_T);
        RKDG_CUDA_TRY(cudaMallocHost(&s->h_ctl, sizeof(StepCtl) * max_slots));
        s->elems.reset(s->cap);
        s->halos.reset(s->hcap);
        s->tasks.reset(s->kcap);
        for (int i = max_slots - 1; i >= 0; --i) s->free_slots.push_back(i);
        s->active.assign(max_slots, nullptr);
        // persistent grid, and a graph of one step whose tile count is read on the device
        for (int l = 0; l < kLists; ++l) {
            const int per_sm = std::max(1, tiled_max_ctas_per_sm(kernel_prec(p.precision), list_order(l), p.nq,
                                                                 list_flux(l), kPoolHalo));
            s->ctas[l] = prop.multiProcessorCount * per_sm;
            TileArgs& t = s->tiles[l];
            t.code = s->tcode;
            t.desc = s->desc + 2 * l * s->tcap;
            t.halo = s->halo;
            t.task = s->task;
            t.max_halo = kPoolHalo;
            t.ntiles = (int)s->tcap;
            t.ntiles_dev = s->ntiles_dev + l;
        }
        RKDG_CUDA_TRY(cudaStreamSynchronize(s->stream));
        cudaGraph_t g;
        RKDG_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_step(s);
        } catch (...) {
            cudaStreamEndCapture(s->stream, &g);
            throw;
        }
        RKDG_CUDA_TRY(cudaStreamEndCapture(s->stream, &g));
        RKDG_CUDA_TRY(cudaGraphInstantiate(&s->graph, g, 0));
        cudaGraphDestroy(g);
        s->engine = std::thread(engine_loop, s);
        *out = s;
    });
    if (rc != RKDG_OK && s) destroy_server(s);
    return rc;
}

int rkdg_server_destroy(rkdg_server* s) {
    return guarded([&] { destroy_server(s); });
}

int rkdg_server_submit_method(rkdg_server* s, const rkdg_mesh_desc* mesh, int32_t order, const double* U0,
                              double t_final, const double* farfield, int32_t limiter, int32_t flux, int64_t* id) {
    return guarded([&] {
        if (!s || !mesh || !U0 || !id || (order != 1 && order != 2) ||
            (flux != RKDG_FLUX_LLF && flux != RKDG_FLUX_HLLC))
            throw Error{RKDG_ERR_INVALID, "rkdg_server_submit: bad arguments"};
        auto r = std::make_shared<Request>();
        r->t_submit = now_s();
        r->order = order;
        r->flux = flux;
        r->nb = order == 1 ? 3 : 6;
        r->limiter = limiter != 0;
        r->t_final = t_final;
        for (int v = 0; v < 4; ++v) r->far[v] = farfield ? farfield[v] : s->p.farfield[v];
        HostMesh m = build_mesh(*mesh);
        m = permute_mesh(m, morton_order(m));
        r->T = m.T;
        if (r->T > s->max_T)
            throw Error{RKDG_ERR_NOMEM, "request of " + std::to_string(r->T) +
                                            " triangles exceeds the pool (" + std::to_string(s->max_T) + ")"};
        HostGeometry g = build_geometry(m, order, false, r->limiter);
        r->jinv = std::move(g.jinv);
        r->lim = std::move(g.lim);
        r->conn.resize((size_t)4 * m.T);
        for (int t = 0; t < m.T; ++t) {
            for (int k = 0; k < 3; ++k) r->conn[4 * t + k] = m.nbr[3 * t + k];
            r->conn[4 * t + 3] = (int32_t)pack_info(&m.shared[3 * t], &m.bc[3 * t],
                                                    g.lim_pair.empty() ? 0u : g.lim_pair[t]);
        }
        r->perm = m.perm;
        r->tiles = build_tiles(m, 0, 0, order, 0, 0);
        if (r->tiles.max_halo > kPoolHalo)
            throw Error{RKDG_ERR_INVALID, "a tile of this mesh has " + std::to_string(r->tiles.max_halo) +
                                              " halo neighbours; the pool stages at most " +
                                              std::to_string(kPoolHalo)};
        if ((int64_t)r->tiles.halo.size() / 2 > s->hcap || (int64_t)r->tiles.task.size() > s->kcap)
            throw Error{RKDG_ERR_NOMEM, "request tables exceed the pool"};
        r->U0.assign(U0, U0 + (size_t)4 * r->nb * r->T);
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->fatal.empty()) throw Error{RKDG_ERR_CUDA, "server stopped: " + s->fatal};
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->queue.push_back(r);
        *id = r->id;
        s->cv_work.notify_all();
    });
}

int rkdg_server_submit(rkdg_server* s, const rkdg_mesh_desc* mesh, int32_t order, const double* U0,
                       double t_final, const double* farfield, int32_t limiter, int64_t* id) {
    if (!s) {
        set_error("rkdg_server_submit: null server");
        return RKDG_ERR_INVALID;
    }
    return rkdg_server_submit_method(s, mesh, order, U0, t_final, farfield, limiter, s->p.flux, id);
}

int rkdg_server_wait(rkdg_server* s, int64_t id, double timeout_s, int32_t* status, double* U,
                     double* times, int32_t* steps) {
    return guarded([&] {
        if (!s) throw Error{RKDG_ERR_INVALID, "null server"};
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) throw Error{RKDG_ERR_INVALID, "unknown request id"};
        std::shared_ptr<Request> r = it->second;
        auto ready = [&] { return r->status >= REQ_DONE; };
        if (timeout_s < 0) s->cv_done.wait(lk, ready);
        else s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready);
        if (status) *status = r->status;
        if (r->status == REQ_DONE || r->status == REQ_FAILED) {
            if (U && r->status == REQ_DONE) std::memcpy(U, r->result.data(), sizeof(double) * r->result.size());
            if (times) {
                times[0] = r->t_submit;
                times[1] = r->t_admit;
                times[2] = r->t_done;
            }
            if (steps) *steps = r->steps;
            const bool failed = r->status == REQ_FAILED;
            std::string err = r->error;
            const int code = r->error_code;
            s->reqs.erase(it);
            if (failed) throw Error{code, err.empty() ? "request failed" : err};
        }
    });
}

int rkdg_server_status(rkdg_server* s, int32_t* queued, int32_t* in_flight) {
    return guarded([&] {
        if (!s) throw Error{RKDG_ERR_INVALID, "null server"};
        std::lock_guard<std::mutex> lk(s->mu);
        int n = 0;
        for (auto& r : s->active) n += (r && r->status == REQ_RUNNING) ? 1 : 0;
        if (queued) *queued = s->fatal.empty() ? (int32_t)s->queue.size() : 0;
        if (in_flight) *in_flight = s->fatal.empty() ? n : 0;
        if (!s->fatal.empty()) throw Error{s->fatal_code, "server stopped: " + s->fatal};
    });
}

int rkdg_server_timing(rkdg_server* s, double* admit_s, double* retire_s, double* step_s, int64_t* chunks) {
    return guarded([&] {
        if (!s) throw Error{RKDG_ERR_INVALID, "null server"};
        std::lock_guard<std::mutex> lk(s->mu);
        if (admit_s) *admit_s = s->t_admit;
        if (retire_s) *retire_s = s->t_retire;
        if (step_s) *step_s = s->busy;
        if (chunks) *chunks = s->chunks;
    });
}

int rkdg_server_inject_fault(rkdg_server* s, int32_t after_chunks) {
    return guarded([&] {
        if (!s || after_chunks < 0) throw Error{RKDG_ERR_INVALID, "rkdg_server_inject_fault: bad arguments"};
        std::lock_guard<std::mutex> lk(s->mu);
        s->fault_after = after_chunks;
    });
}

int rkdg_server_stats(rkdg_server* s, double* dof, double* busy, int64_t* completed, int32_t* peak,
                      int64_t* capacity) {
    return guarded([&] {
        if (!s) throw Error{RKDG_ERR_INVALID, "null server"};
        std::lock_guard<std::mutex> lk(s->mu);
        if (dof) *dof = s->dof_updates;
        if (busy) *busy = s->busy;
        if (completed) *completed = s->completed;
        if (peak) *peak = s->peak;
        if (capacity) *capacity = s->cap;
    });
}

}  // extern "C"
