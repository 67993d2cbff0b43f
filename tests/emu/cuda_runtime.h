// CPU stand-in for the CUDA runtime and device intrinsics used by libsmx.
//
// TEST INFRASTRUCTURE ONLY.  tests/emu/Makefile compiles the product sources
// (subgraphmatching_b200/csrc/*.cu, *.cpp) with g++ -DSMX_EMU against this
// header into tests/emu/libsmx_emu.so, so the kernels' warp-level logic can be
// checked against the oracle on machines without a GPU.  Every GPU thread runs
// as a fiber (its own stack, switched cooperatively on one host thread; with
// -DEMU_THREADS as a host thread instead, which AddressSanitizer builds use);
// shuffles, ballots and reductions meet at a per-warp barrier, __syncthreads
// at a per-block barrier, and a fiber waiting at a barrier yields to the
// others.  "Device" memory is host memory.  The product package never loads
// this library.
#pragma once

#include <algorithm>
#include <atomic>
#include <barrier>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <tuple>
#include <type_traits>
#include <vector>

#ifndef SMX_EMU
#define SMX_EMU 1
#endif

// ------------------------------------------------------------------ keywords
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#define __launch_bounds__(...)
#define __restrict__ __restrict
#define __align__(n) __attribute__((aligned(n)))

struct dim3 {
    unsigned x, y, z;
    constexpr dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct uint2 {
    unsigned x, y;
};

namespace emu {

#ifdef EMU_THREADS
using Bar = std::barrier<>;
#else
void fiber_yield();
// Barrier among the fibers of one host thread: waiting fibers yield until the
// last arrival opens the next generation.
struct Bar {
    explicit Bar(unsigned n) : expected(n) {}
    unsigned expected;
    unsigned count = 0;
    uint64_t gen = 0;
    void arrive_and_wait() {
        const uint64_t g = gen;
        if (++count >= expected) {
            count = 0;
            ++gen;
            return;
        }
        while (gen == g) fiber_yield();
    }
    void arrive_and_drop() {
        --expected;
        if (expected > 0 && count >= expected) {
            count = 0;
            ++gen;
        }
    }
};
void run_fibers(unsigned n, const std::function<void(unsigned)>& body);
#endif

struct Block {
    std::unique_ptr<Bar> bar;
    std::vector<std::unique_ptr<Bar>> warp_bar;
    std::vector<std::vector<uint64_t>> warp_slot;
    std::vector<unsigned char> dyn;
    std::mutex mu;
    std::map<int, std::vector<unsigned char>> statics;
};

struct Ctx {
    dim3 tid, bid, bdim, gdim;
    Block* blk = nullptr;
    unsigned warp = 0, lane = 0;
};

extern thread_local Ctx ctx;

inline uint64_t* slots() { return ctx.blk->warp_slot[ctx.warp].data(); }
inline void wsync() { ctx.blk->warp_bar[ctx.warp]->arrive_and_wait(); }

template <class T>
inline uint64_t pack(T v) {
    static_assert(sizeof(T) <= 8, "shuffle of a type wider than 8 bytes");
    uint64_t x = 0;
    std::memcpy(&x, &v, sizeof(T));
    return x;
}
template <class T>
inline T unpack(uint64_t x) {
    T v;
    std::memcpy(&v, &x, sizeof(T));
    return v;
}

template <class T>
T* shared_static(int key, size_t count) {
    std::lock_guard<std::mutex> lk(ctx.blk->mu);
    auto& v = ctx.blk->statics[key];
    if (v.empty()) v.assign(count * sizeof(T) + 16, 0);
    return reinterpret_cast<T*>(v.data());
}

uint64_t timer_ns();

// ------------------------------------------------------------------ stream capture
struct Capture {
    bool on = false;
    std::vector<std::function<void()>> ops;
};
Capture& capture();

template <class... P>
void launch_now(void (*k)(P...), dim3 grid, dim3 block, size_t smem, std::tuple<std::decay_t<P>...> params) {
    const unsigned nthreads = block.x * block.y * block.z;
    if (nthreads == 0 || nthreads % 32 != 0) std::abort();
    for (unsigned by = 0; by < grid.y; ++by)
        for (unsigned bx = 0; bx < grid.x; ++bx) {
            Block B;
            B.bar = std::make_unique<Bar>(nthreads);
            const unsigned nw = nthreads / 32;
            for (unsigned w = 0; w < nw; ++w) {
                B.warp_bar.push_back(std::make_unique<Bar>(32));
                B.warp_slot.emplace_back(32, 0);
            }
            B.dyn.assign(smem + 64, 0);
            auto body = [&](unsigned t) {
                ctx.tid = dim3(t, 0, 0);
                ctx.bid = dim3(bx, by, 0);
                ctx.bdim = block;
                ctx.gdim = grid;
                ctx.blk = &B;
                ctx.warp = t / 32;
                ctx.lane = t % 32;
                std::tuple<std::decay_t<P>...> mine = params;
                std::apply(k, mine);
                B.warp_bar[ctx.warp]->arrive_and_drop();
                B.bar->arrive_and_drop();
            };
#ifdef EMU_THREADS
            std::vector<std::thread> th;
            th.reserve(nthreads);
            for (unsigned t = 0; t < nthreads; ++t) th.emplace_back(body, t);
            for (auto& x : th) x.join();
#else
            run_fibers(nthreads, body);
#endif
        }
}

template <class... P, class... A>
void launch(void (*k)(P...), dim3 grid, dim3 block, size_t smem, A&&... args) {
    std::tuple<std::decay_t<P>...> params(static_cast<std::decay_t<P>>(args)...);
    if (capture().on) {
        capture().ops.push_back([=]() { launch_now<P...>(k, grid, block, smem, params); });
        return;
    }
    launch_now<P...>(k, grid, block, smem, params);
}

}  // namespace emu

#define threadIdx (::emu::ctx.tid)
#define blockIdx (::emu::ctx.bid)
#define blockDim (::emu::ctx.bdim)
#define gridDim (::emu::ctx.gdim)

namespace smx {
void note_launch();
}
#define SMX_LAUNCH(kernel, grid, block, smem, stream, ...) \
    (::smx::note_launch(), ::emu::launch(kernel, dim3(grid), dim3(block), (size_t)(smem), __VA_ARGS__))
#define SMX_EXTERN_SMEM(name) unsigned char* name = ::emu::ctx.blk->dyn.data()
#define SMX_SHARED_ARRAY(type, name, count) type* name = ::emu::shared_static<type>(__LINE__, (count))

// ------------------------------------------------------------------ intrinsics
inline void __syncwarp(unsigned = 0xffffffffu) { emu::wsync(); }
inline void __syncthreads() { emu::ctx.blk->bar->arrive_and_wait(); }

template <class T>
inline T __shfl_sync(unsigned, T v, int src) {
    emu::slots()[emu::ctx.lane] = emu::pack(v);
    emu::wsync();
    uint64_t y = emu::slots()[src & 31];
    emu::wsync();
    return emu::unpack<T>(y);
}
template <class T>
inline T __shfl_up_sync(unsigned, T v, unsigned d) {
    emu::slots()[emu::ctx.lane] = emu::pack(v);
    emu::wsync();
    uint64_t y = emu::ctx.lane >= d ? emu::slots()[emu::ctx.lane - d] : emu::pack(v);
    emu::wsync();
    return emu::unpack<T>(y);
}
template <class T>
inline T __shfl_down_sync(unsigned, T v, unsigned d) {
    emu::slots()[emu::ctx.lane] = emu::pack(v);
    emu::wsync();
    uint64_t y = emu::ctx.lane + d < 32 ? emu::slots()[emu::ctx.lane + d] : emu::pack(v);
    emu::wsync();
    return emu::unpack<T>(y);
}
template <class T>
inline T __shfl_xor_sync(unsigned, T v, int m) {
    emu::slots()[emu::ctx.lane] = emu::pack(v);
    emu::wsync();
    uint64_t y = emu::slots()[(emu::ctx.lane ^ (unsigned)m) & 31];
    emu::wsync();
    return emu::unpack<T>(y);
}
inline unsigned __ballot_sync(unsigned, int p) {
    emu::slots()[emu::ctx.lane] = p ? 1 : 0;
    emu::wsync();
    unsigned m = 0;
    for (unsigned i = 0; i < 32; ++i) m |= (unsigned)(emu::slots()[i] & 1) << i;
    emu::wsync();
    return m;
}
inline int __any_sync(unsigned mask, int p) { return __ballot_sync(mask, p) != 0; }
inline int __all_sync(unsigned mask, int p) { return __ballot_sync(mask, p) == 0xffffffffu; }
inline unsigned __reduce_or_sync(unsigned, unsigned v) {
    emu::slots()[emu::ctx.lane] = v;
    emu::wsync();
    unsigned r = 0;
    for (unsigned i = 0; i < 32; ++i) r |= (unsigned)emu::slots()[i];
    emu::wsync();
    return r;
}
inline unsigned __reduce_add_sync(unsigned, unsigned v) {
    emu::slots()[emu::ctx.lane] = v;
    emu::wsync();
    unsigned r = 0;
    for (unsigned i = 0; i < 32; ++i) r += (unsigned)emu::slots()[i];
    emu::wsync();
    return r;
}
inline unsigned __reduce_min_sync(unsigned, unsigned v) {
    emu::slots()[emu::ctx.lane] = v;
    emu::wsync();
    unsigned r = 0xffffffffu;
    for (unsigned i = 0; i < 32; ++i) r = std::min(r, (unsigned)emu::slots()[i]);
    emu::wsync();
    return r;
}

inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline int __popcll(unsigned long long x) { return __builtin_popcountll(x); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
inline int __ffsll(long long x) { return __builtin_ffsll(x); }
template <class T>
inline T __ldg(const T* p) { return *p; }
inline size_t __cvta_generic_to_shared(const void* p) { return (size_t)p; }

template <class A, class B>
inline std::common_type_t<A, B> min(A a, B b) {
    using C = std::common_type_t<A, B>;
    return (C)a < (C)b ? (C)a : (C)b;
}
template <class A, class B>
inline std::common_type_t<A, B> max(A a, B b) {
    using C = std::common_type_t<A, B>;
    return (C)a > (C)b ? (C)a : (C)b;
}

inline unsigned long long atomicAdd(unsigned long long* p, unsigned long long v) {
    return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned atomicAdd(unsigned* p, unsigned v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline int atomicCAS(int* p, int cmp, int v) {
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
inline unsigned atomicCAS(unsigned* p, unsigned cmp, unsigned v) {
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
inline unsigned long long atomicCAS(unsigned long long* p, unsigned long long cmp, unsigned long long v) {
    __atomic_compare_exchange_n(p, &cmp, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST);
    return cmp;
}
inline unsigned atomicExch(unsigned* p, unsigned v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicAnd(unsigned* p, unsigned v) { return __atomic_fetch_and(p, v, __ATOMIC_SEQ_CST); }
inline unsigned atomicOr(unsigned* p, unsigned v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
inline unsigned __ldcg(const unsigned* p) { return __atomic_load_n(p, __ATOMIC_SEQ_CST); }
inline int __clz(unsigned x) { return x ? __builtin_clz(x) : 32; }
inline unsigned long long atomicAnd(unsigned long long* p, unsigned long long v) {
    return __atomic_fetch_and(p, v, __ATOMIC_SEQ_CST);
}
inline unsigned long long atomicMax(unsigned long long* p, unsigned long long v) {
    unsigned long long cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return cur;
}
inline unsigned atomicMax(unsigned* p, unsigned v) {
    unsigned cur = __atomic_load_n(p, __ATOMIC_SEQ_CST);
    while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_SEQ_CST, __ATOMIC_SEQ_CST)) {
    }
    return cur;
}

inline uint64_t emu_timer_ns() { return emu::timer_ns(); }

// ------------------------------------------------------------------ runtime API
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorMemoryAllocation = 2 };
typedef void* cudaStream_t;
typedef struct EmuEvent* cudaEvent_t;
typedef struct EmuGraph* cudaGraph_t;
typedef struct EmuGraph* cudaGraphExec_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
};
enum cudaDeviceAttr { cudaDevAttrMultiProcessorCount = 16 };
enum cudaFuncAttribute { cudaFuncAttributeMaxDynamicSharedMemorySize = 8 };
enum cudaStreamCaptureMode { cudaStreamCaptureModeGlobal = 0, cudaStreamCaptureModeThreadLocal = 1 };
#define cudaStreamNonBlocking 1

cudaError_t cudaGetDeviceCount(int* n);
cudaError_t cudaSetDevice(int d);
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int d);
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned flags);
cudaError_t cudaStreamDestroy(cudaStream_t s);
cudaError_t cudaStreamSynchronize(cudaStream_t s);
cudaError_t cudaMalloc(void** p, size_t n);
cudaError_t cudaMallocAsync(void** p, size_t n, cudaStream_t s);
cudaError_t cudaFree(void* p);
cudaError_t cudaMemGetInfo(size_t* free_bytes, size_t* total_bytes);
typedef struct EmuPool* cudaMemPool_t;
enum cudaMemPoolAttr { cudaMemPoolAttrReleaseThreshold = 4 };
inline cudaError_t cudaDeviceGetDefaultMemPool(cudaMemPool_t* p, int) {
    *p = nullptr;
    return 0;
}
inline cudaError_t cudaMemPoolSetAttribute(cudaMemPool_t, cudaMemPoolAttr, void*) { return 0; }
cudaError_t cudaFreeAsync(void* p, cudaStream_t s);
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind k);
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind k, cudaStream_t st);
cudaError_t cudaMemset(void* p, int v, size_t n);
cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t st);
cudaError_t cudaEventCreate(cudaEvent_t* e);
cudaError_t cudaEventDestroy(cudaEvent_t e);
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t s);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b);
cudaError_t cudaGetLastError();
const char* cudaGetErrorString(cudaError_t e);
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned flags);
#define cudaHostAllocMapped 2
#define cudaHostAllocPortable 1
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned flags);
cudaError_t cudaFreeHost(void* p);
cudaError_t cudaStreamBeginCapture(cudaStream_t s, cudaStreamCaptureMode m);
cudaError_t cudaStreamEndCapture(cudaStream_t s, cudaGraph_t* g);
cudaError_t cudaGraphInstantiate(cudaGraphExec_t* e, cudaGraph_t g, unsigned long long flags);
cudaError_t cudaGraphLaunch(cudaGraphExec_t e, cudaStream_t s);
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t e);
cudaError_t cudaGraphDestroy(cudaGraph_t g);

template <class F>
cudaError_t cudaFuncSetAttribute(F, cudaFuncAttribute, int) {
    return cudaSuccess;
}
template <class F>
cudaError_t cudaOccupancyMaxActiveBlocksPerMultiprocessor(int* n, F, int, size_t) {
    *n = 1;
    return cudaSuccess;
}
template <class T>
cudaError_t cudaGetSymbolAddress(void** p, const T& symbol) {
    *p = (void*)&symbol;  // "device" variables are host variables here
    return cudaSuccess;
}
// typed overloads, as the CUDA runtime header provides for C++
template <class T>
cudaError_t cudaMalloc(T** p, size_t n) {
    return cudaMalloc(reinterpret_cast<void**>(p), n);
}
template <class T>
cudaError_t cudaMallocAsync(T** p, size_t n, cudaStream_t s) {
    return cudaMallocAsync(reinterpret_cast<void**>(p), n, s);
}
