// Shared device helpers and constants for the PFSF B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pfsf_b200 {

// Stencil constants (SH/stencil_constants.glsl:9-10, PFSFStencil.java).
constexpr float kEdgeP = 0.5f;
constexpr float kCornerP = 0.1666667f;
constexpr int kMacroBlock = 8;
constexpr uint32_t kMacroSeedBits = 0x38D1B717u;  // 1e-4f
constexpr float kPhiOrphan = 1e6f;

enum : uint8_t { kAir = 0, kSolid = 1, kAnchor = 2 };

// 26-neighbour offsets: 6 faces (-X,+X,-Y,+Y,-Z,+Z), 12 edges in the shader
// order (XY --,++,-+,+-; XZ; YZ), 8 corners (bit0 x, bit1 y, bit2 z; set = +1).
__host__ __device__ constexpr int kOfs(int k, int axis) {
    constexpr signed char t[26][3] = {
        {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1},
        {-1, -1, 0}, {1, 1, 0}, {-1, 1, 0}, {1, -1, 0},
        {-1, 0, -1}, {1, 0, 1}, {-1, 0, 1}, {1, 0, -1},
        {0, -1, -1}, {0, 1, 1}, {0, -1, 1}, {0, 1, -1},
        {-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
        {-1, -1, 1}, {1, -1, 1}, {-1, 1, 1}, {1, 1, 1}};
    return t[k][axis];
}
// face directions (a, b) of edge e
__host__ __device__ constexpr int kEdgeDir(int e, int j) {
    constexpr signed char t[12][2] = {{0, 2}, {1, 3}, {0, 3}, {1, 2}, {0, 4}, {1, 5},
                                      {0, 5}, {1, 4}, {2, 4}, {3, 5}, {2, 5}, {3, 4}};
    return t[e][j];
}

__device__ __forceinline__ bool finite_f(float v) { return !isnan(v) && !isinf(v); }
__device__ __forceinline__ float clamp_f(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

__device__ __forceinline__ float edge_weight(const float s6[6], int e) {
    return sqrtf(fmaxf(s6[kEdgeDir(e, 0)] * s6[kEdgeDir(e, 1)], 0.0f)) * kEdgeP;
}
__device__ __forceinline__ float corner_weight(const float s6[6], int ci) {
    const float sx = (ci & 1) ? s6[1] : s6[0];
    const float sy = (ci & 2) ? s6[3] : s6[2];
    const float sz = (ci & 4) ? s6[5] : s6[4];
    return cbrtf(fmaxf(sx * sy * sz, 0.0f)) * kCornerP;
}

__host__ __device__ __forceinline__ int64_t ceil_div64(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace pfsf_b200
