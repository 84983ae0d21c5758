// Device evaluation of the solve's scalar helpers for tests: the FP64 link
// reciprocal rcp64 (kappa_ops.cuh) next to the IEEE division it replaces.
#include <cuda_runtime.h>

#include "kappa_ops.cuh"
#include "pfsf/pfsf_b200.h"

namespace pfsf_b200 {
namespace {

__global__ void k_rcp64_eval(const double* __restrict__ s, double* __restrict__ approx, double* __restrict__ ieee,
                             int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double v = s[i];
    approx[i] = kappa::rcp64(v);
    ieee[i] = 1.0 / v;
}

}  // namespace
}  // namespace pfsf_b200

extern "C" PFSF_API pfsf_result pfsf_debug_rcp64(const double* in, double* out_rcp64, double* out_ieee, int64_t n) {
    if (n < 0 || (n > 0 && (!in || !out_rcp64 || !out_ieee))) return PFSF_ERROR_INVALID_ARG;
    if (n == 0) return PFSF_OK;
    if (n > (int64_t)1 << 26) return PFSF_ERROR_INVALID_ARG;
    double* d = nullptr;
    if (cudaMalloc(&d, (size_t)n * 24) != cudaSuccess) {
        cudaGetLastError();
        return PFSF_ERROR_OUT_OF_VRAM;
    }
    bool ok = cudaMemcpy(d, in, (size_t)n * 8, cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) {
        const int threads = 256;
        pfsf_b200::k_rcp64_eval<<<(unsigned)((n + threads - 1) / threads), threads>>>(d, d + n, d + 2 * n, n);
        ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cudaMemcpy(out_rcp64, d + n, (size_t)n * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
    ok = ok && cudaMemcpy(out_ieee, d + 2 * n, (size_t)n * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
    cudaFree(d);
    return ok ? PFSF_OK : PFSF_ERROR_VULKAN;
}
