// evd_tridiag_shim.cpp -- drop-in for the reference CUDA prototype's solve
// entry points, forwarding to this library's C ABI (include/brdc.h).
//
// A maintainer of the reference builds this file in place of the
// definitions in gpu/src/tridiag_solver.cu:2373-2388 and :2541-2583, with
// the reference's own headers on the include path (gpu/include, gpu/src),
// and links -lbrdc_b200.  The two functions keep the reference's names,
// namespace and signatures (declared in gpu/src/syev2stage_pipeline.hpp:
// 70-77), so its callers (gpu/bench/tridiag_dc_bench.cu:953, 1222-1261)
// compile and link unchanged.  The argument checks are the reference's, in
// its order (tridiag_solver.cu:2545-2557): handle, pointers, then n, uplo
// and the backend rule of use_gpu_tridiag_solver
// (gpu/src/tridiag_solver_dc.cuh:41-50: CPU backend, or AUTO with n < 17,
// is rejected).  The solve runs on the evd handle's stream; a CUDA failure
// is recorded in the evd handle's last-error fields as the reference's
// EVD_RETURN_IF_CUDA_ERROR does (gpu/src/handle_impl.hpp:170-192).
//
// compute_eigenvectors = 1 returns EVD_STATUS_NOT_IMPLEMENTED: the
// reference keeps those eigenvectors inside its own workspace layout for
// its back-transform stage; this library returns them in a caller array
// (brdc_dstebr_vectors), which a caller reaches directly.
#include <cstddef>
#include <cstdint>

#include "../../include/brdc.h"
#include "handle_impl.hpp"
#include "syev2stage_pipeline.hpp"

namespace evd::internal {
namespace {

constexpr int64_t kMinDcSize = 17; // gpu/src/tridiag_solver_dc.cuh:23

bool gpu_backend(const evd_syev2stage_config &config) {
    if (config.tridiag_solver_backend == EVD_TRIG_SOLVER_BACKEND_CPU) {
        return false;
    }
    if (config.tridiag_solver_backend == EVD_TRIG_SOLVER_BACKEND_GPU) {
        return true;
    }
    return config.n >= kMinDcSize;
}

// One library handle per host thread (a brdc handle is not thread safe);
// it runs on whatever stream the evd handle carries at each call.
brdc_handle thread_handle() {
    static thread_local brdc_handle h = [] {
        brdc_handle x = nullptr;
        return brdc_create(&x) == BRDC_STATUS_SUCCESS ? x : nullptr;
    }();
    return h;
}

} // namespace

evd_status tridiag_solver_workspace_size(const evd_syev2stage_config &config, size_t *bytes) {
    if (bytes == nullptr) {
        return EVD_STATUS_INVALID_POINTER;
    }
    return static_cast<evd_status>(brdc_dstebr_workspace_size(config.n, 0, bytes));
}

evd_status tridiag_solver_run_from_device_tridiagonal(evd_handle handle,
                                                      const evd_syev2stage_config &config,
                                                      const double *d_diag,
                                                      const double *d_subdiag, double *d_W,
                                                      void *workspace, size_t workspace_size) {
    if (handle == nullptr) {
        return EVD_STATUS_INVALID_HANDLE;
    }
    if (d_diag == nullptr || d_W == nullptr || (config.n > 1 && d_subdiag == nullptr)) {
        return EVD_STATUS_INVALID_POINTER;
    }
    if (config.n <= 0 || config.uplo != EVD_FILL_MODE_LOWER || !gpu_backend(config)) {
        return EVD_STATUS_INVALID_VALUE;
    }
    if (config.compute_eigenvectors != 0) {
        return EVD_STATUS_NOT_IMPLEMENTED;
    }
    brdc_handle bh = thread_handle();
    if (bh == nullptr) {
        return EVD_STATUS_CUDA_ERROR;
    }
    brdc_status st = brdc_set_stream(bh, reinterpret_cast<brdc_stream_t>(handle->stream));
    if (st == BRDC_STATUS_SUCCESS) {
        st = brdc_dstebr(bh, config.n, d_diag, d_subdiag, d_W, workspace, workspace_size);
    }
    if (st == BRDC_STATUS_CUDA_ERROR) {
        int code = 0;
        brdc_error_source src = BRDC_ERROR_SRC_NONE;
        const char *site = nullptr;
        brdc_get_last_error(bh, &code, &src, &site);
        set_last_error(handle, code, EVD_ERROR_SRC_CUDA, site);
    }
    // codes 0-8 are the same numbers in both enums
    return static_cast<evd_status>(st);
}

} // namespace evd::internal
