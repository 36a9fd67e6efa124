// rcp_ulps.cu -- test support: accuracy of the solver's pair-loop
// reciprocal (brdc_rcp, ppopp27-brdc-ae_b200/csrc/brdc_secular.cuh) against
// IEEE division on the device: for each x, out[i] = |brdc_rcp(x) - 1/x| /
// ulp(1/x).  Built into tests/librcp_ulps.so by tests/test_rcp_gpu.py.
#include <cuda_runtime.h>

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
