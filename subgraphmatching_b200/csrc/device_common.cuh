// Device helpers shared by the filter and enumeration kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Kernel launches and shared-memory declarations go through these macros so
// the same kernel sources also build for the CPU warp emulator that the test
// suite uses (tests/emu, -DSMX_EMU); the CUDA build expands them to plain CUDA.
namespace smx {
void note_launch();  // counts launches for smx_launch_count()
}
#ifndef SMX_EMU
#define SMX_LAUNCH(kernel, grid, block, smem, stream, ...) \
    (::smx::note_launch(), kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__))
#define SMX_EXTERN_SMEM(name) extern __shared__ __align__(16) unsigned char name[]
#define SMX_SHARED_ARRAY(type, name, count) __shared__ type name[count]
#endif

namespace smx {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
#ifdef SMX_EMU
    return (1u << lane_id()) - 1u;
#else
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
#endif
}

__device__ __forceinline__ uint64_t warp_or64(uint64_t x) {
    uint32_t lo = __reduce_or_sync(kFull, (uint32_t)x);
    uint32_t hi = __reduce_or_sync(kFull, (uint32_t)(x >> 32));
    return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ uint64_t shfl64(uint64_t x, int src) {
    uint32_t lo = __shfl_sync(kFull, (uint32_t)x, src);
    uint32_t hi = __shfl_sync(kFull, (uint32_t)(x >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}

// Rank of data vertex w in the sorted candidate list of query vertex u, using
// the per-32-vertex directory {bits, prefix} laid out [w / 32][qn].
__device__ __forceinline__ uint32_t cand_rank(const uint2* __restrict__ rank, uint32_t qn, uint32_t u, uint32_t w) {
    uint2 r = __ldg(rank + (size_t)(w >> 5) * qn + u);
    return r.y + __popc(r.x & ((1u << (w & 31u)) - 1u));
}

// Branch-free search: true iff x occurs in the sorted array a[0, n).  Plain
// (coherent) loads: the array may be a list this kernel wrote earlier.
__device__ __forceinline__ bool bsearch_global(const uint32_t* a, uint32_t n, uint32_t x) {
    if (n == 0) return false;
    uint32_t base = 0;
    while (n > 1) {
        uint32_t half = n >> 1;
        base = (a[base + half] <= x) ? base + half : base;
        n -= half;
    }
    return a[base] == x;
}

__device__ __forceinline__ bool bsearch_shared(const uint32_t* a, uint32_t n, uint32_t x) {
    if (n == 0) return false;
    uint32_t base = 0;
    while (n > 1) {
        uint32_t half = n >> 1;
        base = (a[base + half] <= x) ? base + half : base;
        n -= half;
    }
    return a[base] == x;
}

// Branch-free search in read-only memory (data graph rows, tables).
__device__ __forceinline__ bool bsearch_ldg(const uint32_t* a, uint32_t n, uint32_t x) {
    if (n == 0) return false;
    uint32_t base = 0;
    while (n > 1) {
        uint32_t half = n >> 1;
        base = (__ldg(a + base + half) <= x) ? base + half : base;
        n -= half;
    }
    return __ldg(a + base) == x;
}

// Number of elements <= x in sorted a[0, n) (global memory, coherent loads).
__device__ __forceinline__ uint32_t upper_bound_global(const uint32_t* a, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
#ifdef SMX_EMU
    return emu_timer_ns();
#else
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
#endif
}

}  // namespace smx
