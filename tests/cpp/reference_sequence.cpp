// The reference's C++ call sequence (multi_gpuRkdg/src/main.cpp:56-149:
// CCUDARkdgSolver::run -> runNext -> initRKDG -> RkdgAdvance::advance ->
// runAfter -> outputSolution) rewired onto librkdg.so's C ABI, as a
// maintainer of the reference would bind it.  Built and run by
// tests/test_gpu_integration.py:
//
//   g++ -std=c++17 reference_sequence.cpp -I include -L <pkg> -lrkdg -Wl,-rpath,<pkg>
//   ./a.out NSTEPS            (in a directory holding input/mesh.conf and the mesh files)
//
// Writes output/solution.plt and output/residual.dat as the reference does,
// plus the final state for the test: output/state_reference.bin and
// output/state_native.bin ([4][nbasis][ntri] doubles, reference and native
// basis) and output/summary.txt (ntri, nbasis, steps, time, totals).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "rkdg.h"

static int fail(const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, rkdg_last_error());
    return 1;
}

int main(int argc, char** argv) {
    const int nsteps = argc > 1 ? std::atoi(argv[1]) : 10;

    // CUnstructuredGrid::initializeGrid + readers (src/unstructuredgrid.cpp:14-60)
    rkdg_mesh_desc mesh;
    if (rkdg_read_mesh(".", "input/mesh.conf", &mesh) != RKDG_OK) return fail("rkdg_read_mesh");

    // runNext: grid, triangle infos, boundary marks, device arrays
    // (src/cudarkdgsolver.cu:192-224); bc = NULL applies the reference's
    // |x|,|y| > 15 far-field rule
    rkdg_params p;
    rkdg_default_params(&p);  // P2, 7/3-point rules, LLF, SSP-RK3, FP64, cfl 0.18, M 0.4, 5 deg
    rkdg_ctx* ctx = nullptr;
    if (rkdg_create(&mesh, &p, &ctx) != RKDG_OK) return fail("rkdg_create");

    // initRKDG (src/cudarkdgsolver.cu:326-368)
    if (rkdg_init_freestream(ctx) != RKDG_OK) return fail("rkdg_init_freestream");

    // RkdgAdvance::advance with its residual file (src/rkdgadvance.cpp:10-17, 91-243)
    if (rkdg_set_residual_log(ctx, "output/residual.dat") != RKDG_OK) return fail("rkdg_set_residual_log");
    double t = 0.0;
    int32_t steps = 0;
    if (rkdg_advance(ctx, nsteps, 0.0, &t, &steps) != RKDG_OK) return fail("rkdg_advance");
    rkdg_set_residual_log(ctx, nullptr);

    // runAfter -> copyFreedomToHost (src/cudarkdgsolver.cu:232-264)
    int32_t ntri = 0, nb = 0;
    rkdg_get_sizes(ctx, &ntri, &nb, nullptr);
    std::vector<double> U((size_t)4 * nb * ntri);
    for (int basis : {RKDG_BASIS_REFERENCE, RKDG_BASIS_NATIVE}) {
        if (rkdg_get_state(ctx, U.data(), ntri, basis) != RKDG_OK) return fail("rkdg_get_state");
        FILE* f = std::fopen(basis == RKDG_BASIS_REFERENCE ? "output/state_reference.bin"
                                                           : "output/state_native.bin", "wb");
        if (!f || std::fwrite(U.data(), sizeof(double), U.size(), f) != U.size()) return 1;
        std::fclose(f);
    }

    // outputSolution (src/cudarkdgsolver.cu:860-1001)
    if (rkdg_write_solution(ctx, "output/solution.plt") != RKDG_OK) return fail("rkdg_write_solution");

    double tot[4];
    if (rkdg_conservation_totals(ctx, tot) != RKDG_OK) return fail("rkdg_conservation_totals");
    FILE* s = std::fopen("output/summary.txt", "w");
    if (!s) return 1;
    std::fprintf(s, "%d %d %d %.17g %.17g %.17g %.17g %.17g\n", ntri, nb, steps, t, tot[0], tot[1], tot[2], tot[3]);
    std::fclose(s);

    // ~CCUDARkdgSolver
    rkdg_destroy(ctx);
    rkdg_free_mesh(&mesh);
    std::printf("ok: %d triangles, %d steps, t = %.6g\n", ntri, steps, t);
    return 0;
}
