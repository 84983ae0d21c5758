// Island labelling: 26-connected components of the non-air voxels of a box.
//
// The reference labels on the GPU by label propagation -- every solid or
// anchor voxel starts with label i + 1, alternating "hook to the smallest
// neighbour label" and "jump to the parent's label" passes with atomicMin
// until nothing changes (SH/label_prop_init.comp.glsl, label_prop_iterate.
// comp.glsl), then one slot per root with block count, anchored flag and
// bounding box (label_prop_summarise_alloc / _aggregate.comp.glsl).  Its
// fixed point labels every voxel of a component with 1 + the smallest flat
// index in the component; that value is what is bit-exact here.
//
// B200 form: a union-find instead of iterating to the fixed point.  One pass
// unites every voxel with its 13 already-visited neighbours, always linking
// the larger root under the smaller (lock-free compare-and-swap, path
// halving); parents only ever point to smaller indices, so the surviving
// root of a component is its smallest index and the labels equal the
// reference's fixed point.  Three full passes (unite, flatten, aggregate)
// replace O(diameter) propagation passes.  Component slots are assigned in
// ascending root order by a prefix sum, so the component table is
// deterministic (the reference hands slots out by atomicAdd order).
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "labels.h"

namespace pfsf_b200 {
namespace labels {
namespace {

constexpr uint32_t kNoIsland = 0xFFFFFFFFu;
constexpr int kUniteRetryLimit = 1 << 20;

// Representative of x with path halving; parents only decrease, so the walk
// ends.  Stale reads are harmless: every stored value is an ancestor.
__device__ __forceinline__ uint32_t rep(uint32_t* par, uint32_t x) {
    uint32_t cur = par[x];
    if (cur != x) {
        uint32_t prev = x, next;
        while (cur > (next = par[cur])) {
            par[prev] = next;
            prev = cur;
            cur = next;
        }
    }
    return cur;
}

__device__ void unite(uint32_t* par, uint32_t a, uint32_t b, int* err) {
    uint32_t ra = rep(par, a), rb = rep(par, b);
    for (int tries = 0; ra != rb; tries++) {
        if (tries > kUniteRetryLimit) {  // cannot happen with a correct forest; bounded anyway
            atomicExch(err, 1);
            return;
        }
        if (ra < rb) {
            const uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        const uint32_t old = atomicCAS(&par[ra], ra, rb);
        if (old == ra) return;
        ra = rep(par, old);
        rb = rep(par, rb);
    }
}

__global__ void k_init(const uint8_t* __restrict__ type, uint32_t* __restrict__ par, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) par[i] = type[i] != kAir ? (uint32_t)i : kNoIsland;
}

__global__ void k_unite(const uint8_t* __restrict__ type, uint32_t* par, int lx, int ly, int lz, int* err) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        if (type[i] == kAir) continue;
        const int x = (int)(i % lx), y = (int)((i / lx) % ly), z = (int)(i / ((int64_t)lx * ly));
        // the 13 neighbours that precede i in flat order
        for (int dz = -1; dz <= 0; dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
                    const int nx = x + dx, ny = y + dy, nz = z + dz;
                    if (nx < 0 || nx >= lx || ny < 0 || ny >= ly || nz < 0) continue;
                    const int64_t j = nx + (int64_t)lx * (ny + (int64_t)ly * nz);
                    if (type[j] != kAir) unite(par, (uint32_t)i, (uint32_t)j, err);
                }
    }
}

// root[i] = the smallest index of i's component (kNoIsland on air); root flags
// for the slot scan
__global__ void k_flatten(uint32_t* par, uint32_t* __restrict__ root, uint32_t* __restrict__ flag, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (par[i] == kNoIsland) {
        root[i] = kNoIsland;
        flag[i] = 0;
        return;
    }
    const uint32_t r = rep(par, (uint32_t)i);
    root[i] = r;
    flag[i] = r == (uint32_t)i ? 1u : 0u;
}

// label = root + 1 (the reference's convention), kNoIsland on air
__global__ void k_labels(const uint32_t* __restrict__ root, uint32_t* __restrict__ lab, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lab[i] = root[i] == kNoIsland ? kNoIsland : root[i] + 1u;
}

__global__ void k_slots_init(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ slot, int64_t n,
                             int32_t cap, pfsf_label_component* comps) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !flag[i]) return;
    const uint32_t s = slot[i];
    if (s >= (uint32_t)cap) return;
    pfsf_label_component& c = comps[s];
    c.root_label = (uint32_t)i + 1u;
    c.block_count = 0;
    c.anchored = 0;
    c._pad0 = 0;
    c.aabb_min[0] = c.aabb_min[1] = c.aabb_min[2] = 0xFFFFFFFFu;
    c._pad1 = 0;
    c.aabb_max[0] = c.aabb_max[1] = c.aabb_max[2] = 0u;
    c._pad2 = 0;
}

__global__ void k_aggregate(const uint8_t* __restrict__ type, const uint32_t* __restrict__ root,
                            const uint32_t* __restrict__ slot, int lx, int ly, int lz, int32_t cap,
                            pfsf_label_component* comps) {
    const int64_t n = (int64_t)lx * ly * lz;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r = root[i];
    if (r == kNoIsland) return;
    const uint32_t s = slot[r];
    if (s >= (uint32_t)cap) return;
    pfsf_label_component& c = comps[s];
    const uint32_t x = (uint32_t)(i % lx), y = (uint32_t)((i / lx) % ly), z = (uint32_t)(i / ((int64_t)lx * ly));
    atomicAdd(&c.block_count, 1u);
    if (type[i] == kAnchor) atomicOr(&c.anchored, 1u);
    atomicMin(&c.aabb_min[0], x);
    atomicMin(&c.aabb_min[1], y);
    atomicMin(&c.aabb_min[2], z);
    atomicMax(&c.aabb_max[0], x);
    atomicMax(&c.aabb_max[1], y);
    atomicMax(&c.aabb_max[2], z);
}

#define LB_OK(expr) (cudaSuccess == (expr))

}  // namespace

pfsf_result label_components(cudaStream_t s, int num_sms, const uint8_t* host_type, int32_t lx, int32_t ly, int32_t lz,
                             uint32_t* host_labels, pfsf_label_component* host_comps, int32_t capacity,
                             int32_t* out_count, int32_t* out_overflow) {
    if (!host_type || lx <= 0 || ly <= 0 || lz <= 0 || capacity < 0 || (capacity > 0 && !host_comps) || !out_count)
        return PFSF_ERROR_INVALID_ARG;
    const int64_t n = (int64_t)lx * ly * lz;
    if (n >= (int64_t)kNoIsland) return PFSF_ERROR_INVALID_ARG;  // labels are 32-bit
    uint8_t* type = nullptr;
    uint32_t *par = nullptr, *root = nullptr, *flag = nullptr, *slot = nullptr;
    pfsf_label_component* comps = nullptr;
    int* err = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flag, slot, (int64_t)n, s);
    const size_t cbytes = sizeof(pfsf_label_component) * (size_t)std::max(capacity, 1);
    bool ok = LB_OK(cudaMalloc(&type, (size_t)n)) && LB_OK(cudaMalloc(&par, (size_t)n * 4)) &&
              LB_OK(cudaMalloc(&root, (size_t)n * 4)) && LB_OK(cudaMalloc(&flag, (size_t)n * 4)) &&
              LB_OK(cudaMalloc(&slot, (size_t)n * 4)) && LB_OK(cudaMalloc(&comps, cbytes)) &&
              LB_OK(cudaMalloc(&err, sizeof(int))) && LB_OK(cudaMalloc(&tmp, std::max<size_t>(tmp_bytes, 16)));
    pfsf_result rc = PFSF_OK;
    int32_t herr = 0;
    uint32_t tail_slot = 0, tail_flag = 0;
    if (!ok) {
        cudaGetLastError();
        rc = PFSF_ERROR_OUT_OF_VRAM;
    } else {
        const unsigned b = 256, g = (unsigned)ceil_div64(n, b);
        const unsigned gu = (unsigned)std::min<int64_t>(g, (int64_t)num_sms * 16);
        ok &= LB_OK(cudaMemcpyAsync(type, host_type, (size_t)n, cudaMemcpyHostToDevice, s));
        ok &= LB_OK(cudaMemsetAsync(err, 0, sizeof(int), s));
        ok &= LB_OK(cudaMemsetAsync(comps, 0, cbytes, s));
        k_init<<<g, b, 0, s>>>(type, par, n);
        k_unite<<<gu, b, 0, s>>>(type, par, lx, ly, lz, err);
        k_flatten<<<g, b, 0, s>>>(par, root, flag, n);
        ok &= LB_OK(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, flag, slot, (int64_t)n, s));
        k_slots_init<<<g, b, 0, s>>>(flag, slot, n, capacity, comps);
        k_aggregate<<<g, b, 0, s>>>(type, root, slot, lx, ly, lz, capacity, comps);
        if (host_labels) {
            k_labels<<<g, b, 0, s>>>(root, par, n);
            ok &= LB_OK(cudaMemcpyAsync(host_labels, par, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
        }
        ok &= LB_OK(cudaMemcpyAsync(&tail_slot, slot + n - 1, 4, cudaMemcpyDeviceToHost, s));
        ok &= LB_OK(cudaMemcpyAsync(&tail_flag, flag + n - 1, 4, cudaMemcpyDeviceToHost, s));
        ok &= LB_OK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        if (capacity > 0) ok &= LB_OK(cudaMemcpyAsync(host_comps, comps, cbytes, cudaMemcpyDeviceToHost, s));
        ok &= LB_OK(cudaStreamSynchronize(s));
        if (!ok || herr) rc = PFSF_ERROR_VULKAN;
    }
    if (rc == PFSF_OK) {
        const uint32_t total = tail_slot + tail_flag;  // roots = exclusive prefix at the end + last flag
        *out_count = (int32_t)std::min<uint32_t>(total, (uint32_t)capacity);
        if (out_overflow) *out_overflow = total > (uint32_t)capacity ? 1 : 0;
    }
    cudaFree(type);
    cudaFree(par);
    cudaFree(root);
    cudaFree(flag);
    cudaFree(slot);
    cudaFree(comps);
    cudaFree(err);
    cudaFree(tmp);
    return rc;
}

}  // namespace labels
}  // namespace pfsf_b200
