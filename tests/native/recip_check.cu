// Test-only CUDA build: the mixed form's Newton-refined reciprocal and
// reciprocal square root (emergence_b200/csrc/physics.cuh: rcp_nr, rsqrt_nr)
// and the fast FP64 form's one-ulp versions (rcp_f, rsqrt_f, sqrt_f) next to
// CUDA's correctly rounded division and square root, on the same inputs, so
// their relative error can be measured on the GPU.
#include "../../emergence_b200/csrc/physics.cuh"

#include <cuda_runtime.h>
#include <stddef.h>

namespace {

// out: [0] rcp_nr(y)   [1] 1/y
//      [2] rsqrt_nr(x) [3] 1/sqrt(x)   [4] x·rsqrt_nr(x)   [5] sqrt(x)   (x = |y|)
__global__ void recip_kernel(const double* y, double* out, size_t n) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = y[i];
    const double x = fabs(v);
    const double r = emg::rsqrt_nr(x);
    out[0 * n + i] = emg::rcp_nr(v);
    out[1 * n + i] = 1.0 / v;
    out[2 * n + i] = r;
    out[3 * n + i] = 1.0 / sqrt(x);
    out[4 * n + i] = x * r;
    out[5 * n + i] = sqrt(x);
}

// the fast FP64 form's one-ulp versions: [0] rcp_f(y) [1] 1/y [2] rsqrt_f(x)
// [3] 1/sqrt(x) [4] sqrt_f(x) [5] sqrt(x)
__global__ void recip_fast_kernel(const double* y, double* out, size_t n) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = y[i];
    const double x = fabs(v);
    out[0 * n + i] = emg::rcp_f(v);
    out[1 * n + i] = 1.0 / v;
    out[2 * n + i] = emg::rsqrt_f(x);
    out[3 * n + i] = 1.0 / sqrt(x);
    out[4 * n + i] = emg::sqrt_f(x);
    out[5 * n + i] = sqrt(x);
}

}  // namespace

// fast != 0: the fast FP64 form's versions (recip_fast_kernel)
extern "C" int recip_check(const double* y_host, double* out_host, size_t n, int fast) {
    double *y = nullptr, *out = nullptr;
    if (cudaMalloc(&y, n * sizeof(double)) != cudaSuccess) return 1;
    if (cudaMalloc(&out, 6 * n * sizeof(double)) != cudaSuccess) {
        cudaFree(y);
        return 1;
    }
    int rc = 0;
    if (cudaMemcpy(y, y_host, n * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) rc = 1;
    if (!rc) {
        if (fast)
            recip_fast_kernel<<<(unsigned)((n + 255) / 256), 256>>>(y, out, n);
        else
            recip_kernel<<<(unsigned)((n + 255) / 256), 256>>>(y, out, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 1;
    }
    if (!rc && cudaMemcpy(out_host, out, 6 * n * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) rc = 1;
    cudaFree(y);
    cudaFree(out);
    return rc;
}
