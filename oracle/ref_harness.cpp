/*
 * ref_harness.cpp -- single-process CPU driver for the REFERENCE's own RKDG code.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or loads this file.
 * It is built by oracle/Makefile together with the reference's unmodified
 * sources (read in place from the reference checkout) into
 * oracle/_ref/librkdg_ref.so, and is used only by tests/, by the fixture
 * generator under tests/golden/, and by bench.py's CPU-baseline leg.
 *
 * What it mirrors (paths relative to the reference's multi_gpuRkdg/):
 *   - mesh + geometry set-up: CCUDARkdgSolver::run / runNext
 *     (src/cudarkdgsolver.cu:158-230) with nprocs = 1, i.e.
 *     CUnstructuredGrid::initializeGrid / initializeGridNext,
 *     initializeTriangleInfos, markLocalBoundaryTriangles;
 *   - device arrays: CCUDAArrays::allocateMemory (src/cudaarrays.cpp:72-152),
 *     here host vectors with pitch = number of cells;
 *   - initial condition: CCUDARkdgSolver::initRKDG (src/cudarkdgsolver.cu:326-368);
 *   - launch wrappers: src/cudarkdgsolver.cu:370-611, each `<<<grid, block>>>`
 *     replaced by a loop over emulated blocks/threads that calls the
 *     reference kernel body (src/kernelfunctions.cu) compiled as C++;
 *   - the step: RkdgAdvance::advance (src/rkdgadvance.cpp:91-217) without
 *     MPI: dt, copy U -> U_old, 3 x [ConVars, BC, VolumeRHS, LFCoeff, EdgeFG,
 *     Flux x2, EdgeRHS, stage update], residual monitor.
 *
 * The two single-block reductions (kernel_getTimeStep, kernel_calculateResidual)
 * are run with blockDim = 1 and zeroed shared scratch: the one thread then
 * folds every element in its strided loop and the tree phase only compares
 * against zeros, so the unmodified kernel returns the exact maximum.
 *
 * Blocks of the per-element kernels may be spread over OpenMP threads
 * (rkdg_ref_set_threads); the emulated shared memory and thread indices are
 * thread_local (see ref_stub/cuda_runtime.h), so this is race-free.
 */
#include <unistd.h>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <stdexcept>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "unstructuredgrid.h"
#include "kernelfunctions.cuh"

thread_local rkdg_emu_dim3 threadIdx;
thread_local rkdg_emu_dim3 blockIdx;
thread_local rkdg_emu_dim3 blockDim;

// Backing store of the reference kernels' `extern __shared__` arrays.
static const int kMaxBlock = 1024;
thread_local double freedom[CONSERVATIVE_VARS * kMaxBlock];
thread_local double sw[TRIANGLE_EDGES * EDGE_GPOINTS * kMaxBlock];
thread_local double mx[kMaxBlock];
thread_local double res[RESIDUAL_VARS * kMaxBlock];

static int g_threads = 1;

namespace {

struct Rows {
    std::vector<double> v;
    void alloc(int rows, int pitch) { v.assign((size_t)rows * pitch, 0.0); }
    double* p() { return v.data(); }
};

struct RefCase {
    CUnstructuredGrid grid;
    int tnum = 0, num = 0, P = 0;
    int tpb = 512;
    double gamma = 1.4, alpha = 0, mach = 0.4, cfl = 0.18, rhoref = 1, pref = 1;
    // far-field state used by the boundary kernel (src/rkdgadvance.cpp:31-34)
    double bc_rho = 1, bc_rhou = 0, bc_rhov = 0, bc_rhoE = 0;

    std::vector<int> neighbour, sharedEdge, flag;
    Rows area, perimeter, normal, mass, vol_bf, vol_bdf, edge_bf, vol_w, edge_w;
    Rows U[4], Uold[4], cv_vol[4], cv_edge[4], rhs_vol[4], rhs_edge[4];
    Rows fe[4], ge[4], lf[4], lfcoeff;
    double ddt = 0, residual[RESIDUAL_VARS] = {0, 0};
};

template <class F>
void launch(int n, int tpb, F body) {
    int blocks = (n % tpb) ? n / tpb + 1 : n / tpb;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (int b = 0; b < blocks; ++b) {
        blockDim = {(unsigned)tpb, 1, 1};
        blockIdx = {(unsigned)b, 0, 0};
        for (int t = 0; t < tpb; ++t) {
            threadIdx = {(unsigned)t, 0, 0};
            body();
        }
    }
}

void single_thread_block() {
    blockDim = {1, 1, 1};
    blockIdx = {0, 0, 0};
    threadIdx = {0, 0, 0};
    std::memset(mx, 0, sizeof(mx));
    std::memset(res, 0, sizeof(res));
}

void time_step(RefCase& c) {
    single_thread_block();
    kernel_getTimeStep(c.tnum, c.gamma, c.cfl, &c.ddt, c.U[0].p(), c.U[1].p(), c.U[2].p(),
                       c.U[3].p(), c.perimeter.p(), c.area.p());
}

void residual_monitor(RefCase& c) {
    single_thread_block();
    kernel_calculateResidual(c.tnum, c.U[0].p(), c.U[3].p(), c.Uold[0].p(), c.Uold[3].p(),
                             c.residual);
}

// One evaluation of R(U) in the order of src/rkdgadvance.cpp:135-159.
void rhs(RefCase& c) {
    const int P = c.P, tnum = c.tnum, num = c.num, tpb = c.tpb;
    launch(tnum, tpb, [&] {
        kernel_calculateConVars(tnum, P, c.U[0].p(), c.U[1].p(), c.U[2].p(), c.U[3].p(),
                                c.cv_vol[0].p(), c.cv_vol[1].p(), c.cv_vol[2].p(), c.cv_vol[3].p(),
                                c.cv_edge[0].p(), c.cv_edge[1].p(), c.cv_edge[2].p(),
                                c.cv_edge[3].p(), c.vol_bf.p(), c.edge_bf.p());
    });
    if (num > tnum) {
        launch(num - tnum, 64, [&] {
            kernel_boundaryCondition(tnum, num, P, c.bc_rho, c.bc_rhou, c.bc_rhov, c.bc_rhoE,
                                     c.cv_edge[0].p(), c.cv_edge[1].p(), c.cv_edge[2].p(),
                                     c.cv_edge[3].p(), c.U[0].p(), c.U[1].p(), c.U[2].p(),
                                     c.U[3].p(), c.neighbour.data(), c.sharedEdge.data(),
                                     c.flag.data(), c.normal.p());
        });
    }
    launch(tnum, tpb, [&] {
        kernel_calculateVolumeRHS(tnum, P, c.gamma, c.cv_vol[0].p(), c.cv_vol[1].p(),
                                  c.cv_vol[2].p(), c.cv_vol[3].p(), c.rhs_vol[0].p(),
                                  c.rhs_vol[1].p(), c.rhs_vol[2].p(), c.rhs_vol[3].p(),
                                  c.vol_w.p(), c.vol_bdf.p());
    });
    launch(tnum, tpb, [&] {
        kernel_calculateLFCoeff(tnum, P, P, c.gamma, c.normal.p(), c.neighbour.data(), c.U[0].p(),
                                c.U[1].p(), c.U[2].p(), c.U[3].p(), c.lfcoeff.p());
    });
    launch(num, tpb, [&] {
        kernel_calculateEdgeFG(tnum, num, P, c.gamma, c.cv_edge[0].p(), c.cv_edge[1].p(),
                               c.cv_edge[2].p(), c.cv_edge[3].p(), c.fe[0].p(), c.fe[1].p(),
                               c.fe[2].p(), c.fe[3].p(), c.ge[0].p(), c.ge[1].p(), c.ge[2].p(),
                               c.ge[3].p());
    });
    launch(tnum, tpb, [&] {
        kernel_calculateFlux(tnum, P, P, c.neighbour.data(), c.sharedEdge.data(), c.cv_edge[0].p(),
                             c.cv_edge[1].p(), c.fe[0].p(), c.fe[1].p(), c.ge[0].p(), c.ge[1].p(),
                             c.normal.p(), c.lfcoeff.p(), c.lf[0].p(), c.lf[1].p());
    });
    launch(tnum, tpb, [&] {
        kernel_calculateFlux(tnum, P, P, c.neighbour.data(), c.sharedEdge.data(), c.cv_edge[2].p(),
                             c.cv_edge[3].p(), c.fe[2].p(), c.fe[3].p(), c.ge[2].p(), c.ge[3].p(),
                             c.normal.p(), c.lfcoeff.p(), c.lf[2].p(), c.lf[3].p());
    });
    launch(tnum, tpb, [&] {
        kernel_calculateEdgeRHS(tnum, P, c.edge_w.p(), c.edge_bf.p(), c.lf[0].p(), c.lf[1].p(),
                                c.lf[2].p(), c.lf[3].p(), c.rhs_edge[0].p(), c.rhs_edge[1].p(),
                                c.rhs_edge[2].p(), c.rhs_edge[3].p(), c.rhs_vol[0].p(),
                                c.rhs_vol[1].p(), c.rhs_vol[2].p(), c.rhs_vol[3].p());
    });
}

void stage_update(RefCase& c, int i, double dt) {
    const int P = c.P, tnum = c.tnum;
    launch(tnum, c.tpb, [&] {
        if (i == 0)
            kernel_rkdgStepOne(tnum, P, dt, c.mass.p(), c.U[0].p(), c.U[1].p(), c.U[2].p(),
                               c.U[3].p(), c.rhs_edge[0].p(), c.rhs_edge[1].p(),
                               c.rhs_edge[2].p(), c.rhs_edge[3].p());
        else if (i == 1)
            kernel_rkdgStepTwo(tnum, P, dt, c.mass.p(), c.U[0].p(), c.U[1].p(), c.U[2].p(),
                               c.U[3].p(), c.rhs_edge[0].p(), c.rhs_edge[1].p(),
                               c.rhs_edge[2].p(), c.rhs_edge[3].p(), c.Uold[0].p(),
                               c.Uold[1].p(), c.Uold[2].p(), c.Uold[3].p());
        else
            kernel_rkdgStepThree(tnum, P, dt, c.mass.p(), c.U[0].p(), c.U[1].p(), c.U[2].p(),
                                 c.U[3].p(), c.rhs_edge[0].p(), c.rhs_edge[1].p(),
                                 c.rhs_edge[2].p(), c.rhs_edge[3].p(), c.Uold[0].p(),
                                 c.Uold[1].p(), c.Uold[2].p(), c.Uold[3].p());
    });
}

void copy_rows(std::vector<double>& dst, const double* src, int rows, int n, int P) {
    for (int r = 0; r < rows; ++r)
        std::memcpy(dst.data() + (size_t)r * P, src + (size_t)r * n, sizeof(double) * n);
}

}  // namespace

extern "C" {

void rkdg_ref_set_threads(int n) { g_threads = n > 0 ? n : 1; }

/* params: gamma, alpha (degrees), mach, cfl, rhoref, pref.  Returns NULL and
 * fills err on failure.  workdir must hold input/ElemDepart.dat (the reader's
 * hard-coded path, src/unstructuredgrid.cpp:38) and the mesh files named in
 * the mesh configuration file meshconf (relative to workdir). */
void* rkdg_ref_open(const char* workdir, const char* meshconf, const double* params, int tpb,
                    char* err, int errlen) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) cwd[0] = 0;
    RefCase* c = nullptr;
    try {
        if (chdir(workdir) != 0) throw std::runtime_error(std::string("cannot chdir to ") + workdir);
        c = new RefCase();
        c->gamma = params[0];
        c->alpha = params[1] * std::atan(1.0) * 4 / 180;  // src/cudarkdgsolver.cu:116
        c->mach = params[2];
        c->cfl = params[3];
        c->rhoref = params[4];
        c->pref = params[5];
        c->tpb = tpb > 0 ? (tpb > kMaxBlock ? kMaxBlock : tpb) : 512;

        CUnstructuredGrid& g = c->grid;
        g.config_file = meshconf;
        g.initializeGrid(0, 1);
        g.initializeGridNext();
        g.testLocalTriangleAntiwise();
        g.triangle_infos.allocateMemory(g.getLocalCellNumber());
        g.initializeTriangleInfos();
        g.markLocalBoundaryTriangles();

        const int num = g.getLocalCellNumber();
        const int tnum = g.getLocalTriangleNumber();
        c->num = num;
        c->tnum = tnum;
        c->P = num;
        const int P = num;

        c->neighbour.assign(g.local_tri_neighbour, g.local_tri_neighbour + 3 * num);
        c->sharedEdge.assign(g.local_tri_sharedEdge, g.local_tri_sharedEdge + 3 * num);
        c->flag.assign(g.local_tri_flag, g.local_tri_flag + num);

        CTriangleInfo& ti = g.triangle_infos;
        c->area.alloc(1, P);
        c->perimeter.alloc(1, P);
        c->normal.alloc(6, P);
        c->mass.alloc(BASIS_FUNCTIONS, P);
        c->vol_bf.alloc(VOLUME_GPOINTS * BASIS_FUNCTIONS, P);
        c->vol_bdf.alloc(2 * VOLUME_GPOINTS * BASIS_FUNCTIONS, P);
        c->edge_bf.alloc(TRIANGLE_EDGES * EDGE_GPOINTS * BASIS_FUNCTIONS, P);
        c->vol_w.alloc(VOLUME_GPOINTS, P);
        c->edge_w.alloc(TRIANGLE_EDGES * EDGE_GPOINTS, P);
        copy_rows(c->area.v, ti.area, 1, num, P);
        copy_rows(c->perimeter.v, ti.perimeter, 1, num, P);
        copy_rows(c->normal.v, ti.outer_normal_vector, 6, num, P);
        copy_rows(c->mass.v, ti.mass_coeff, BASIS_FUNCTIONS, num, P);
        copy_rows(c->vol_bf.v, ti.vol_bf_value, VOLUME_GPOINTS * BASIS_FUNCTIONS, num, P);
        copy_rows(c->vol_bdf.v, ti.vol_bdf_value, 2 * VOLUME_GPOINTS * BASIS_FUNCTIONS, num, P);
        copy_rows(c->edge_bf.v, ti.edge_bf_value, TRIANGLE_EDGES * EDGE_GPOINTS * BASIS_FUNCTIONS,
                  num, P);
        copy_rows(c->vol_w.v, ti.vol_gauss_weight, VOLUME_GPOINTS, num, P);
        copy_rows(c->edge_w.v, ti.edge_gauss_weight, TRIANGLE_EDGES * EDGE_GPOINTS, num, P);

        for (int v = 0; v < 4; ++v) {
            c->U[v].alloc(BASIS_FUNCTIONS, P);
            c->Uold[v].alloc(BASIS_FUNCTIONS, P);
            c->cv_vol[v].alloc(VOLUME_GPOINTS, P);
            c->cv_edge[v].alloc(TRIANGLE_EDGES * EDGE_GPOINTS, P);
            c->rhs_vol[v].alloc(BASIS_FUNCTIONS, P);
            c->rhs_edge[v].alloc(BASIS_FUNCTIONS, P);
            c->fe[v].alloc(TRIANGLE_EDGES * EDGE_GPOINTS, P);
            c->ge[v].alloc(TRIANGLE_EDGES * EDGE_GPOINTS, P);
            c->lf[v].alloc(TRIANGLE_EDGES * EDGE_GPOINTS, P);
        }
        c->lfcoeff.alloc(TRIANGLE_EDGES, P);

        // far-field state of the boundary kernel (src/rkdgadvance.cpp:31-34)
        double ut = std::sqrt(c->gamma * c->pref / c->rhoref) * c->mach;
        c->bc_rho = c->rhoref;
        c->bc_rhou = c->rhoref * ut * std::cos(c->alpha);
        c->bc_rhov = c->rhoref * ut * std::sin(c->alpha);
        c->bc_rhoE = 0.5 * c->rhoref * (ut * ut) + c->pref / (c->gamma - 1);
    } catch (const std::exception& e) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
        delete c;
        c = nullptr;
    }
    if (cwd[0] && chdir(cwd) != 0) { /* best effort */ }
    return c;
}

void rkdg_ref_close(void* h) { delete static_cast<RefCase*>(h); }

void rkdg_ref_sizes(void* h, int* tnum, int* num) {
    RefCase* c = static_cast<RefCase*>(h);
    *tnum = c->tnum;
    *num = c->num;
}

/* Overrides the boundary kernel's far-field state (rho, rhou, rhov, rhoE). */
void rkdg_ref_set_farfield(void* h, const double* s) {
    RefCase* c = static_cast<RefCase*>(h);
    c->bc_rho = s[0];
    c->bc_rhou = s[1];
    c->bc_rhov = s[2];
    c->bc_rhoE = s[3];
}

/* Free-stream initial condition of CCUDARkdgSolver::initRKDG
 * (src/cudarkdgsolver.cu:326-368): row 0 of every cell, other rows zero. */
void rkdg_ref_init_freestream(void* h) {
    RefCase* c = static_cast<RefCase*>(h);
    double ut = std::sqrt(c->gamma * c->pref / c->rhoref) * c->mach;
    double u = ut * std::cos(c->alpha), v = ut * std::sin(c->alpha);
    for (int k = 0; k < 4; ++k) std::fill(c->U[k].v.begin(), c->U[k].v.end(), 0.0);
    for (int i = 0; i < c->num; ++i) {
        c->U[0].v[i] = c->rhoref;
        c->U[1].v[i] = c->rhoref * u;
        c->U[2].v[i] = c->rhoref * v;
        c->U[3].v[i] = c->rhoref * (ut * ut) / 2 + c->pref / (c->rhoref * (c->gamma - 1));
    }
}

/* geometry of every cell (owned then ghost), rows of length num:
 * area[num], perimeter[num], normal[6][num], mass[6][num], barycenter[2][num],
 * neighbour[3][num], sharedEdge[3][num], flag[num]. */
void rkdg_ref_get_geometry(void* h, double* area, double* perimeter, double* normal, double* mass,
                           double* bary, int* neighbour, int* shared, int* flag) {
    RefCase* c = static_cast<RefCase*>(h);
    const int n = c->num;
    std::memcpy(area, c->area.p(), sizeof(double) * n);
    std::memcpy(perimeter, c->perimeter.p(), sizeof(double) * n);
    std::memcpy(normal, c->normal.p(), sizeof(double) * 6 * n);
    std::memcpy(mass, c->mass.p(), sizeof(double) * BASIS_FUNCTIONS * n);
    for (int i = 0; i < n; ++i) {
        bary[i] = c->grid.triangle_infos.barycenter[i].getX();
        bary[n + i] = c->grid.triangle_infos.barycenter[i].getY();
    }
    std::memcpy(neighbour, c->neighbour.data(), sizeof(int) * 3 * n);
    std::memcpy(shared, c->sharedEdge.data(), sizeof(int) * 3 * n);
    std::memcpy(flag, c->flag.data(), sizeof(int) * n);
}

/* Per-cell basis tables: vol_bf[42][num], vol_bdf[84][num], edge_bf[54][num],
 * vol_w[7][num], edge_w[9][num], basis coefficients [num][36]. */
void rkdg_ref_get_tables(void* h, double* vol_bf, double* vol_bdf, double* edge_bf, double* vol_w,
                         double* edge_w, double* coeff) {
    RefCase* c = static_cast<RefCase*>(h);
    const int n = c->num;
    std::memcpy(vol_bf, c->vol_bf.p(), sizeof(double) * c->vol_bf.v.size());
    std::memcpy(vol_bdf, c->vol_bdf.p(), sizeof(double) * c->vol_bdf.v.size());
    std::memcpy(edge_bf, c->edge_bf.p(), sizeof(double) * c->edge_bf.v.size());
    std::memcpy(vol_w, c->vol_w.p(), sizeof(double) * c->vol_w.v.size());
    std::memcpy(edge_w, c->edge_w.p(), sizeof(double) * c->edge_w.v.size());
    const std::vector<double>& bc = c->grid.triangle_infos.basis_fun_coeff;
    size_t ncoeff = std::min(bc.size(), (size_t)n * 36);
    std::memcpy(coeff, bc.data(), sizeof(double) * ncoeff);
}

/* DOFs as [var][basis][num] (var = rho, rhou, rhov, rhoE). */
void rkdg_ref_set_dofs(void* h, const double* U) {
    RefCase* c = static_cast<RefCase*>(h);
    const size_t blk = (size_t)BASIS_FUNCTIONS * c->num;
    for (int v = 0; v < 4; ++v) std::memcpy(c->U[v].p(), U + v * blk, sizeof(double) * blk);
}

void rkdg_ref_get_dofs(void* h, double* U) {
    RefCase* c = static_cast<RefCase*>(h);
    const size_t blk = (size_t)BASIS_FUNCTIONS * c->num;
    for (int v = 0; v < 4; ++v) std::memcpy(U + v * blk, c->U[v].p(), sizeof(double) * blk);
}

double rkdg_ref_time_step(void* h) {
    RefCase* c = static_cast<RefCase*>(h);
    time_step(*c);
    return c->ddt;
}

/* One R(U) evaluation; R as [var][basis][num] (the reference's rhs_edge_*). */
void rkdg_ref_residual(void* h, double* R) {
    RefCase* c = static_cast<RefCase*>(h);
    rhs(*c);
    const size_t blk = (size_t)BASIS_FUNCTIONS * c->num;
    if (R)
        for (int v = 0; v < 4; ++v) std::memcpy(R + v * blk, c->rhs_edge[v].p(), sizeof(double) * blk);
}

/* U_old <- U (src/rkdgadvance.cpp:104-107) */
void rkdg_ref_save_old(void* h) {
    RefCase* c = static_cast<RefCase*>(h);
    for (int v = 0; v < 4; ++v) c->Uold[v].v = c->U[v].v;
}

/* R(U) followed by rkdgStep{One,Two,Three} (i = 0, 1, 2). */
void rkdg_ref_stage(void* h, int i, double dt) {
    RefCase* c = static_cast<RefCase*>(h);
    rhs(*c);
    stage_update(*c, i, dt);
}

/* nsteps full steps as RkdgAdvance::advance; per-step dt and the residual
 * monitor (max |d rho_mean|, max |d rhoE_mean|) are written when non-NULL. */
void rkdg_ref_advance(void* h, int nsteps, double* dts, double* resid) {
    RefCase* c = static_cast<RefCase*>(h);
    for (int s = 0; s < nsteps; ++s) {
        time_step(*c);
        double dt = c->ddt;
        for (int v = 0; v < 4; ++v) c->Uold[v].v = c->U[v].v;
        for (int i = 0; i < RUNGE_KUTTA_STEPS; ++i) {
            rhs(*c);
            stage_update(*c, i, dt);
        }
        residual_monitor(*c);
        if (dts) dts[s] = dt;
        if (resid) {
            resid[2 * s] = c->residual[0];
            resid[2 * s + 1] = c->residual[1];
        }
    }
}

}  // extern "C"
