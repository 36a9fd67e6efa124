// ref_merge.cu -- TEST INFRASTRUCTURE ONLY.
// Runs the reference CUDA prototype's own deflation kernels
// (gpu/src/tridiag_solver_merge_kernels.cuh, compiled here from the
// reference's header as it lies) on merge inputs the caller supplies, so a
// test can hand them exactly the inputs this build's merges saw and compare
// the decisions one by one.  One call processes one merge level:
//   stedc_merge_prepare_deflatezero_boundary_kernel<256>  z, rho, tol, small-z mask
//                                                        (merge_kernels.cuh:1040-1102)
//   stedc_merge_sortd_kernel                             active-first rank sort (:143-182)
//   stedc_merge_setcandflags_kernel                      close-pole candidates (:184-212)
//   stedc_merge_deflatecount_kernel                      Givens chains (:214-252)
//   stedc_merge_deflateapply_kernel                      rotations of z (:254-290)
// with the split arrays of that level filled as the reference's
// stedc_update_splits_* kernels fill them (node sizes and starts per merge
// and per row).  Built by build_ref.sh into oracle/_ref/libref_merge.so.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "tridiag_solver_merge_kernels.cuh"

using namespace evd::internal;

// Inputs (host): n rows of one level, `merges` merges of sizes
// child_sizes[2m] + child_sizes[2m+1] laid out back to back; D[n] the
// children's eigenvalues by row (left child's rows, then right child's);
// E[n] with the merge's coupling |E| at its split - 1; first_rows[n] and
// last_rows[n] the children's boundary rows by row.
// Outputs (host, n each): mask0 (small-z survivors, by row), mask (after
// the close-pole rotations, by row), map (sorted position -> row), md
// (sorted position -> d), ndd (sorted position -> survivors of its node),
// dcount (sorted position -> members rotated into the base there), z, cc,
// ss (by row, after the rotations), tol and rho (by row).
// Returns 0 or a CUDA error code.
extern "C" int ref_merge_level(int n, int merges, const int *child_sizes, const double *D,
                               const double *E, const double *first_rows,
                               const double *last_rows, int *mask0, int *mask, int *map,
                               double *md, int *ndd, int *dcount, double *z, double *cc,
                               double *ss, double *tol, double *rho) {
    std::vector<int> splits(get_splits_size(n), 0);
    int *bsz = ptr_bsz(n, splits.data());
    int *bps = ptr_bps(n, splits.data());
    int *em = ptr_em(n, splits.data());
    int *nsz = ptr_nsz(n, splits.data());
    int *nps = ptr_nps(n, splits.data());
    int *hmask = ptr_mask(n, splits.data());
    int *hmap = ptr_map(n, splits.data());
    int start = 0;
    for (int m = 0; m < merges; ++m) {
        const int sl = child_sizes[2 * m], sr = child_sizes[2 * m + 1];
        bsz[2 * m] = sl;
        bsz[2 * m + 1] = sr;
        bps[2 * m] = start;
        bps[2 * m + 1] = start + sl;
        for (int i = start; i < start + sl + sr; ++i) {
            em[i] = m;
            nsz[i] = sl + sr;
            nps[i] = start;
            hmask[i] = 1;
            hmap[i] = i;
        }
        start += sl + sr;
    }
    if (start != n) {
        return -1;
    }
    int *dsplits = nullptr;
    double *dtmpz = nullptr, *dD = nullptr, *dE = nullptr, *dbr = nullptr;
    cudaError_t e = cudaSuccess;
    auto chk = [&](cudaError_t x) {
        if (e == cudaSuccess) {
            e = x;
        }
    };
    chk(cudaMalloc(&dsplits, sizeof(int) * get_splits_size(n)));
    chk(cudaMalloc(&dtmpz, sizeof(double) * get_tmpz_size(n)));
    chk(cudaMalloc(&dD, sizeof(double) * n));
    chk(cudaMalloc(&dE, sizeof(double) * n));
    chk(cudaMalloc(&dbr, sizeof(double) * get_boundary_rows_size(n)));
    if (e == cudaSuccess) {
        chk(cudaMemcpy(dsplits, splits.data(), sizeof(int) * splits.size(), cudaMemcpyHostToDevice));
        chk(cudaMemset(dtmpz, 0, sizeof(double) * get_tmpz_size(n)));
        chk(cudaMemcpy(dD, D, sizeof(double) * n, cudaMemcpyHostToDevice));
        chk(cudaMemcpy(dE, E, sizeof(double) * n, cudaMemcpyHostToDevice));
        chk(cudaMemcpy(ptr_first_rows(n, dbr), first_rows, sizeof(double) * n,
                       cudaMemcpyHostToDevice));
        chk(cudaMemcpy(ptr_last_rows(n, dbr), last_rows, sizeof(double) * n,
                       cudaMemcpyHostToDevice));
    }
    const int threads = 256;
    const int blocks = (n + threads - 1) / threads;
    const double eps = std::numeric_limits<double>::epsilon();
    if (e == cudaSuccess) {
        stedc_merge_prepare_deflatezero_boundary_kernel<256>
            <<<merges, 256>>>(merges, n, dD, dE, dbr, dtmpz, dsplits, eps);
        chk(cudaGetLastError());
        chk(cudaMemcpy(mask0, ptr_mask(n, dsplits), sizeof(int) * n, cudaMemcpyDeviceToHost));
        stedc_merge_sortd_kernel<<<blocks, threads>>>(n, dD, dtmpz, dsplits);
        chk(cudaGetLastError());
        chk(cudaMemcpy(map, ptr_map(n, dsplits), sizeof(int) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(md, ptr_md(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(ndd, ptr_ndd(n, dsplits), sizeof(int) * n, cudaMemcpyDeviceToHost));
        stedc_merge_setcandflags_kernel<<<blocks, threads>>>(n, dtmpz, dsplits);
        chk(cudaGetLastError());
        stedc_merge_deflatecount_kernel<<<blocks, threads>>>(n, dtmpz, dsplits);
        chk(cudaGetLastError());
        stedc_merge_deflateapply_kernel<<<blocks, threads>>>(n, dtmpz, dsplits);
        chk(cudaGetLastError());
        chk(cudaMemcpy(mask, ptr_mask(n, dsplits), sizeof(int) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(dcount, ptr_dcount(n, dsplits), sizeof(int) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(z, ptr_z(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(cc, ptr_cc(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(ss, ptr_ss(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(tol, ptr_tolsD(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
        chk(cudaMemcpy(rho, ptr_r1p(n, dtmpz), sizeof(double) * n, cudaMemcpyDeviceToHost));
    }
    cudaFree(dsplits);
    cudaFree(dtmpz);
    cudaFree(dD);
    cudaFree(dE);
    cudaFree(dbr);
    return (int)e;
}
