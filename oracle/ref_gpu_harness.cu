// GPU driver for the reference's OWN CUDA code (measurement and test
// infrastructure only; the product library never links it).
//
// It builds a CCUDARkdgSolver (src/cudarkdgsolver.cu) on one device exactly
// as CCUDARkdgSolver::run + runNext do (src/cudarkdgsolver.cu:158-230, minus
// the log file and the configuration-file parser: the fields are set from
// the arguments), and advances it with the single-process body of
// RkdgAdvance::advance (src/rkdgadvance.cpp:91-243: dt kernel, U_old copy,
// per RK stage the seven kernels and the stage update, dt read back to the
// host every step, the residual kernel), without MPI, logging or printing.
// Built by oracle/Makefile (target libref_gpu) from the reference checkout.
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "cudarkdgsolver.h"

namespace {

struct RefGpu {
    CCUDARkdgSolver s;
    int tnum = 0, num = 0, blocks = 0;
    double bc[4] = {0, 0, 0, 0};
};

// R(U) as one RK stage of RkdgAdvance::advance forms it (src/rkdgadvance.cpp:135-189).
// The boundary kernel covers the ghost cells; a mesh without ghost cells
// (fully periodic) has none to fill, and its zero-size launch is skipped.
void residual(RefGpu* c, int pitch_num, int ipitch_num) {
    CCUDARkdgSolver& s = c->s;
    const int tnum = c->tnum, num = c->num, blocks = c->blocks;
    s.calculateConVars(tnum, pitch_num, blocks);
    if (num > tnum) s.boundaryCondition(tnum, num, pitch_num, c->bc[0], c->bc[1], c->bc[2], c->bc[3]);
    s.calculateVolumeRHS(tnum, pitch_num, blocks);
    s.calculateLFCoeff(tnum, ipitch_num, pitch_num, blocks);
    s.calculateEdgeFG(tnum, num, pitch_num, blocks);
    s.calculateFlux(tnum, ipitch_num, pitch_num, blocks);
    s.calculateEdgeRHS(tnum, pitch_num, blocks);
}

void check_cuda(const char* where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw std::runtime_error(std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

/* params: gamma, alpha (degrees), mach, cfl, rhoref, pref.  workdir holds the
 * mesh files (and input/ElemDepart.dat) named by meshconf. */
void* rkdg_refgpu_open(const char* workdir, const char* meshconf, const double* params, int tpb,
                       char* err, int errlen) {
    char cwd[4096];
    if (!getcwd(cwd, sizeof(cwd))) cwd[0] = 0;
    RefGpu* c = nullptr;
    try {
        if (chdir(workdir) != 0) throw std::runtime_error(std::string("cannot chdir to ") + workdir);
        c = new RefGpu();
        CCUDARkdgSolver& s = c->s;
        s.myid = 0;
        s.nprocs = 1;
        s.log_history = 'N';
        s.gamma = params[0];
        s.alpha = params[1] * std::atan(1.0) * 4 / 180;  // src/cudarkdgsolver.cu:116
        s.mach = params[2];
        s.cfl = params[3];
        s.rhoref = params[4];
        s.pref = params[5];
        s.threads_per_block = tpb > 0 ? tpb : 512;
        s.reduction_threads = 512;
        s.grid.config_file = meshconf;
        s.grid.initializeGrid(0, 1);
        s.runNext();
        check_cuda("set-up");
        c->tnum = s.grid.getLocalTriangleNumber();
        c->num = s.grid.getLocalCellNumber();
        c->blocks = (c->tnum + s.threads_per_block - 1) / s.threads_per_block;
        const double ut = std::sqrt(s.gamma * s.pref / s.rhoref) * s.mach;  // src/rkdgadvance.cpp:31-34
        c->bc[0] = s.rhoref;
        c->bc[1] = s.rhoref * ut * std::cos(s.alpha);
        c->bc[2] = s.rhoref * ut * std::sin(s.alpha);
        c->bc[3] = 0.5 * s.rhoref * (ut * ut) + s.pref / (s.gamma - 1);
        cudaDeviceSynchronize();
        check_cuda("set-up");
    } catch (const std::exception& e) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
        delete c;
        c = nullptr;
    }
    if (cwd[0] && chdir(cwd) != 0) { /* best effort */ }
    return c;
}

void rkdg_refgpu_close(void* h) {
    delete static_cast<RefGpu*>(h);
    cudaDeviceSynchronize();
}

void rkdg_refgpu_sizes(void* h, int* tnum, int* num) {
    RefGpu* c = static_cast<RefGpu*>(h);
    *tnum = c->tnum;
    *num = c->num;
}

/* U: [4][BASIS_FUNCTIONS][num] (rho, rhou, rhov, rhoE). */
int rkdg_refgpu_set_dofs(void* h, const double* U) {
    RefGpu* c = static_cast<RefGpu*>(h);
    CCUDAArrays& a = c->s._cuarrays;
    const size_t pitch = a.getDoublePitch(), row = sizeof(double) * c->num;
    double* dst[4] = {a.freedom_rho, a.freedom_rhou, a.freedom_rhov, a.freedom_rhoE};
    for (int v = 0; v < 4; ++v)
        cudaMemcpy2D(dst[v], pitch, U + (size_t)v * BASIS_FUNCTIONS * c->num, row, row, BASIS_FUNCTIONS,
                     cudaMemcpyHostToDevice);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int rkdg_refgpu_get_dofs(void* h, double* U) {
    RefGpu* c = static_cast<RefGpu*>(h);
    CCUDAArrays& a = c->s._cuarrays;
    const size_t pitch = a.getDoublePitch(), row = sizeof(double) * c->num;
    double* src[4] = {a.freedom_rho, a.freedom_rhou, a.freedom_rhov, a.freedom_rhoE};
    for (int v = 0; v < 4; ++v)
        cudaMemcpy2D(U + (size_t)v * BASIS_FUNCTIONS * c->num, row, src[v], pitch, row, BASIS_FUNCTIONS,
                     cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

/* R(U) of the current state into R: [4][BASIS_FUNCTIONS][num], the edge
 * right-hand side before the mass division (rhs_edge_*). */
int rkdg_refgpu_residual(void* h, double* R) {
    RefGpu* c = static_cast<RefGpu*>(h);
    CCUDAArrays& a = c->s._cuarrays;
    const size_t pitch = a.getDoublePitch(), row = sizeof(double) * c->num;
    residual(c, (int)(pitch / sizeof(double)), (int)(a.getIntPitch() / sizeof(int)));
    double* src[4] = {a.rhs_edge_rho, a.rhs_edge_rhou, a.rhs_edge_rhov, a.rhs_edge_rhoE};
    for (int v = 0; v < 4; ++v)
        cudaMemcpy2D(R + (size_t)v * BASIS_FUNCTIONS * c->num, row, src[v], pitch, row, BASIS_FUNCTIONS,
                     cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

/* The reference's own Tecplot writer, CCUDARkdgSolver::outputSolution
 * (src/cudarkdgsolver.cu:860-1001), on the opened mesh with the given cell
 * means M [4][tnum] (rho, rhou, rhov, rhoE) as its single rank's results.
 * It prints its progress lines to stdout, as the reference does. */
int rkdg_refgpu_write_solution(void* h, const double* M, const char* path) {
    RefGpu* c = static_cast<RefGpu*>(h);
    CCUDARkdgSolver& s = c->s;
    const size_t T = (size_t)c->tnum;
    std::vector<double> r(M, M + 4 * T);
    int data_size[1] = {c->tnum};
    s.solution_file = path;
    s.outputSolution(data_size, r.data(), r.data() + T, r.data() + 2 * T, r.data() + 3 * T);
    return 0;
}

/* n steps; *ms = device milliseconds between events recorded before the
 * first and after the last step (the per-step host read of dt included, as
 * in the reference's loop).  *dt_last = the last step's dt.  0 on success. */
int rkdg_refgpu_steps(void* h, int n, double* ms, double* dt_last) {
    RefGpu* c = static_cast<RefGpu*>(h);
    CCUDARkdgSolver& s = c->s;
    CCUDAArrays& a = s._cuarrays;
    const size_t pitch = a.getDoublePitch();
    const int pitch_num = (int)(pitch / sizeof(double));
    const int ipitch_num = (int)(a.getIntPitch() / sizeof(int));
    const int tnum = c->tnum, blocks = c->blocks;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int step = 0; step < n; ++step) {
        s.getTimeStep(tnum);
        cudaMemcpy2DAsync(a.freedom_rho_old, pitch, a.freedom_rho, pitch, pitch, BASIS_FUNCTIONS, cudaMemcpyDeviceToDevice);
        cudaMemcpy2DAsync(a.freedom_rhou_old, pitch, a.freedom_rhou, pitch, pitch, BASIS_FUNCTIONS, cudaMemcpyDeviceToDevice);
        cudaMemcpy2DAsync(a.freedom_rhov_old, pitch, a.freedom_rhov, pitch, pitch, BASIS_FUNCTIONS, cudaMemcpyDeviceToDevice);
        cudaMemcpy2DAsync(a.freedom_rhoE_old, pitch, a.freedom_rhoE, pitch, pitch, BASIS_FUNCTIONS, cudaMemcpyDeviceToDevice);
        for (int i = 0; i < RUNGE_KUTTA_STEPS; ++i) {
            residual(c, pitch_num, ipitch_num);
            if (i == 0) {
                cudaMemcpy(s._dt, a.ddt, sizeof(double), cudaMemcpyDeviceToHost);
                s.rkdgStepOne(s._dt[0], tnum, pitch_num, blocks);
            } else if (i == 1) {
                s.rkdgStepTwo(s._dt[0], tnum, pitch_num, blocks);
            } else {
                s.rkdgStepThree(s._dt[0], tnum, pitch_num, blocks);
            }
        }
        s.calculateResidual(tnum);
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float t = 0;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms) *ms = t;
    if (dt_last) *dt_last = s._dt[0];
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // extern "C"
