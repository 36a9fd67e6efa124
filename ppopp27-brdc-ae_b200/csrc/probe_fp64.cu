// probe_fp64.cu -- FP64 FMA throughput probe for the roofline denominator.
// The pool's measured-peaks file carries HBM and bf16 figures only, so the
// benchmark measures the B200's non-tensor FP64 rate itself: every thread
// runs 8 independent DFMA chains.  Built as a separate library; the solver
// does not link it.
#include <cuda_runtime.h>

__global__ void k_dfma(int iters, double *out) {
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        a[q] = 1.0 + 1e-9 * (threadIdx.x + q);
    }
    const double m = 0.999999999, c = 1e-12;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            a[q] = fma(a[q], m, c);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        s += a[q];
    }
    if (s == 12345.0) {
        out[0] = s; // keeps the chains alive
    }
}

// Returns the achieved FP64 rate in GFLOP/s (2 flops per FMA), or a
// negative CUDA error code.
extern "C" double brdc_probe_dfma_gflops(int blocks, int threads, int iters) {
    double *out = nullptr;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) {
        return -1.0;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_dfma<<<blocks, threads>>>(iters / 10, out); // warm-up
    cudaEventRecord(e0);
    k_dfma<<<blocks, threads>>>(iters, out);
    cudaEventRecord(e1);
    const cudaError_t st = cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (st != cudaSuccess || ms <= 0.0f) {
        return -(double)st;
    }
    const double flops = 2.0 * 8.0 * (double)blocks * threads * (double)iters;
    return flops / (ms * 1e-3) / 1e9;
}

// ------------------------------------------------------------------
// Accuracy of the solver's pair-loop reciprocal (brdc_rcp) against IEEE
// division: for each x, out[i] = |brdc_rcp(x) - 1/x| / ulp(1/x).
#include "brdc_secular.cuh"

__global__ void k_rcp_ulps(const double *x, double *out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double ref = 1.0 / x[i];
        const double got = brdc::brdc_rcp(x[i]);
        const double a = fabs(ref);
        const double ulp = __longlong_as_double(__double_as_longlong(a) + 1) - a;
        out[i] = fabs(got - ref) / ulp;
    }
}

// Host arrays in and out; returns 0 or a CUDA error code.
extern "C" int brdc_probe_rcp_ulps(const double *x, double *out, int n) {
    double *dx = nullptr, *dout = nullptr;
    if (n <= 0) {
        return 0;
    }
    if (cudaMalloc(&dx, sizeof(double) * n) != cudaSuccess) {
        return 2;
    }
    if (cudaMalloc(&dout, sizeof(double) * n) != cudaSuccess) {
        cudaFree(dx);
        return 2;
    }
    cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    k_rcp_ulps<<<(n + 255) / 256, 256>>>(dx, dout, n);
    const cudaError_t st = cudaMemcpy(out, dout, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dout);
    return (int)st;
}
