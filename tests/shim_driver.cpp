// shim_driver.cpp -- test support: plain C entry points that call the
// evd::internal forwarding shim (ppopp27-brdc-ae_b200/shim/
// evd_tridiag_shim.cpp) the way the reference's bench does
// (gpu/bench/tridiag_dc_bench.cu:953, 1222-1261), with an evd handle that
// carries only a stream.  Built with the shim by tests/build_shim_check.sh
// into tests/libshim_check.so.
#include <cstdint>

#include "handle_impl.hpp"
#include "syev2stage_pipeline.hpp"

namespace {
evd_syev2stage_config config(int64_t n, int uplo, int backend, int vectors) {
    evd_syev2stage_config c{};
    c.n = n;
    c.uplo = static_cast<evd_fill_mode>(uplo);
    c.compute_eigenvectors = vectors;
    c.tridiag_solver_backend = static_cast<evd_tridiag_solver_backend>(backend);
    c.tridiag_sort_backend = EVD_TRIDIAG_SORT_BACKEND_CUB;
    return c;
}
} // namespace

extern "C" int shim_workspace_size(int64_t n, size_t *bytes) {
    return evd::internal::tridiag_solver_workspace_size(config(n, 0, 2, 0), bytes);
}

extern "C" int shim_solve(int64_t n, int uplo, int backend, int vectors, const double *dD,
                          const double *dE, double *dW, void *ws, size_t bytes, void *stream) {
    evd_handle_struct h{};
    h.stream = static_cast<cudaStream_t>(stream);
    return evd::internal::tridiag_solver_run_from_device_tridiagonal(
        &h, config(n, uplo, backend, vectors), dD, dE, dW, ws, bytes);
}
