// ref_shim.cu -- TEST INFRASTRUCTURE ONLY.
// C entry points around the reference CUDA prototype, compiled together
// with the prototype's own sources (gpu/src/*.cu, *.cpp) by build_ref.sh
// into oracle/_ref/libref_brdc_gpu.so.  They call the reference's solve
// entry evd::internal::tridiag_solver_run_from_device_tridiagonal
// (gpu/src/tridiag_solver.cu:2541) with the bench's values-only settings
// (gpu/bench/tridiag_dc_bench.cu:937-979: backend GPU, eigenvectors off)
// and copy its per-level diagnostics (gpu/src/handle_impl.hpp:16-77) out.
// The prototype's CPU fallback links LAPACK dstedc_; dstedc_ here forwards
// to scipy's OpenBLAS, whose path the caller passes to ref_init().
#include <dlfcn.h>

#include <cstdint>
#include <cstring>

#include "handle_impl.hpp"
#include "syev2stage_pipeline.hpp"

namespace {
void *g_lapack = nullptr;
typedef void (*dstedc_fn)(const char *, const int *, double *, double *, double *,
                          const int *, double *, const int *, int *, const int *,
                          int *, size_t);
dstedc_fn g_dstedc = nullptr;

evd_syev2stage_config make_config(int64_t n, int diagnostics) {
    evd_syev2stage_config c{};
    c.n = n;
    c.band_size = 0;
    c.bulge_block_size = 0;
    c.uplo = EVD_FILL_MODE_LOWER;
    c.compute_eigenvectors = 0;
    c.enable_timing = 0;
    c.tridiag_solver_backend = EVD_TRIG_SOLVER_BACKEND_GPU;
    c.tridiag_sort_backend = EVD_TRIDIAG_SORT_BACKEND_CUB;
    c.enable_tridiag_diagnostics = diagnostics;
    return c;
}
} // namespace

extern "C" void dstedc_(const char *compz, const int *n, double *d, double *e,
                        double *z, const int *ldz, double *work, const int *lwork,
                        int *iwork, const int *liwork, int *info) {
    if (g_dstedc == nullptr) {
        *info = -100;
        return;
    }
    g_dstedc(compz, n, d, e, z, ldz, work, lwork, iwork, liwork, info, 1);
}

extern "C" int ref_init(const char *lapack_path) {
    if (lapack_path != nullptr && g_lapack == nullptr) {
        g_lapack = dlopen(lapack_path, RTLD_NOW | RTLD_LOCAL);
        if (g_lapack != nullptr) {
            g_dstedc = (dstedc_fn)dlsym(g_lapack, "scipy_dstedc_");
        }
    }
    return 0;
}

extern "C" int ref_create(void **handle) {
    evd_handle h = nullptr;
    const evd_status st = evd_create_handle(&h);
    *handle = h;
    return (int)st;
}

extern "C" int ref_destroy(void *handle) {
    return (int)evd_destroy_handle(static_cast<evd_handle>(handle));
}

extern "C" void *ref_stream(void *handle) {
    return static_cast<evd_handle>(handle)->stream;
}

extern "C" int ref_workspace_size(int64_t n, size_t *bytes) {
    const evd_syev2stage_config c = make_config(n, 0);
    return (int)evd::internal::tridiag_solver_workspace_size(c, bytes);
}

extern "C" int ref_solve(void *handle, int64_t n, const double *dD,
                         const double *dE, double *dW, void *ws, size_t bytes,
                         int diagnostics) {
    const evd_syev2stage_config c = make_config(n, diagnostics);
    return (int)evd::internal::tridiag_solver_run_from_device_tridiagonal(
        static_cast<evd_handle>(handle), c, dD, dE, dW, ws, bytes);
}

// Per-level counters of the last diagnostic solve: for level k,
// out[8*k + 0..7] = merge_count, size_sum, dd_before_sum, dd_after_sum,
// dd_after_max, secular_iter_sum, secular_iter_max, secular_iter_failed.
// Returns the number of levels.
extern "C" int ref_level_diagnostics(void *handle, int *out, int max_levels) {
    evd_handle h = static_cast<evd_handle>(handle);
    const auto &lv = h->last_tridiag_diagnostics.levels;
    int k = 0;
    for (; k < (int)lv.size() && k < max_levels; ++k) {
        out[8 * k + 0] = lv[k].merge_count;
        out[8 * k + 1] = lv[k].size_sum;
        out[8 * k + 2] = lv[k].dd_before_sum;
        out[8 * k + 3] = lv[k].dd_after_sum;
        out[8 * k + 4] = lv[k].dd_after_max;
        out[8 * k + 5] = lv[k].secular_iter_sum;
        out[8 * k + 6] = lv[k].secular_iter_max;
        out[8 * k + 7] = lv[k].secular_iter_failed;
    }
    return k;
}
