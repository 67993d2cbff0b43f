// Runtime half of the CPU stand-in (see cuda_runtime.h).  TEST INFRASTRUCTURE ONLY.
#include "cuda_runtime.h"

namespace emu {
thread_local Ctx ctx;

#ifndef EMU_THREADS
// ------------------------------------------------------------------ fibers
// x86-64 System V context switch: saves the callee-saved registers and the
// stack pointer of the running context into *save, resumes the one at `to`.
extern "C" void emu_fiber_switch(void** save, void* to);
asm(R"(
    .text
    .globl emu_fiber_switch
    .type emu_fiber_switch,@function
emu_fiber_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size emu_fiber_switch,.-emu_fiber_switch
)");

namespace {
constexpr size_t kFiberStack = 256 * 1024;
struct Fiber {
    void* sp = nullptr;
    Ctx ctx;
    bool done = false;
};
struct Sched {
    void* main_sp = nullptr;
    std::vector<Fiber> fibers;
    size_t cur = 0;
    const std::function<void(unsigned)>* body = nullptr;
};
thread_local Sched* g_sched = nullptr;
}  // namespace

extern "C" void emu_fiber_entry() {
    Sched* S = g_sched;
    const size_t me = S->cur;
    (*S->body)((unsigned)me);
    S->fibers[me].done = true;
    S->fibers[me].ctx = ctx;
    emu_fiber_switch(&S->fibers[me].sp, S->main_sp);
    std::abort();  // a finished fiber is never resumed
}

void fiber_yield() {
    Sched* S = g_sched;
    Fiber& f = S->fibers[S->cur];
    f.ctx = ctx;
    emu_fiber_switch(&f.sp, S->main_sp);
    ctx = S->fibers[S->cur].ctx;
}

void run_fibers(unsigned n, const std::function<void(unsigned)>& body) {
    Sched S;
    S.body = &body;
    S.fibers.resize(n);
    std::vector<char*> stacks(n);
    for (unsigned i = 0; i < n; ++i) {
        stacks[i] = static_cast<char*>(std::malloc(kFiberStack));
        if (!stacks[i]) std::abort();
        uintptr_t top = (reinterpret_cast<uintptr_t>(stacks[i]) + kFiberStack) & ~(uintptr_t)15;
        void** sp = reinterpret_cast<void**>(top);
        *--sp = nullptr;                                         // alignment pad
        *--sp = reinterpret_cast<void*>(&emu_fiber_entry);       // popped by ret
        for (int r = 0; r < 6; ++r) *--sp = nullptr;             // rbp rbx r12-r15
        S.fibers[i].sp = sp;
    }
    Sched* saved = g_sched;
    const Ctx saved_ctx = ctx;
    g_sched = &S;
    unsigned alive = n;
    while (alive) {
        for (unsigned i = 0; i < n; ++i) {
            if (S.fibers[i].done) continue;
            S.cur = i;
            ctx = S.fibers[i].ctx;
            emu_fiber_switch(&S.main_sp, S.fibers[i].sp);
            if (S.fibers[i].done) --alive;
        }
    }
    g_sched = saved;
    ctx = saved_ctx;
    for (char* p : stacks) std::free(p);
}
#endif

Capture& capture() {
    static thread_local Capture c;
    return c;
}

uint64_t timer_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}
}  // namespace emu

struct EmuEvent {
    uint64_t t = 0;
};
struct EmuGraph {
    std::vector<std::function<void()>> ops;
};

cudaError_t cudaGetDeviceCount(int* n) {
    *n = 1;
    return cudaSuccess;
}
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr, int) {
    *v = 1;  // one "SM": launches shrink to a handful of blocks
    return cudaSuccess;
}
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* s, unsigned) {
    *s = reinterpret_cast<cudaStream_t>(0x1);
    return cudaSuccess;
}
cudaError_t cudaStreamDestroy(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
static void* poisoned_alloc(size_t n) {
    const size_t sz = ((n ? n : 1) + 255) & ~(size_t)255;
    void* p = std::aligned_alloc(256, sz);
    if (p) std::memset(p, 0xCD, sz);  // poison: no zeroed memory may be assumed
    return p;
}
cudaError_t cudaMalloc(void** p, size_t n) {
    *p = poisoned_alloc(n);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaMallocAsync(void** p, size_t n, cudaStream_t) {
    *p = poisoned_alloc(n);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaMemGetInfo(size_t* free_bytes, size_t* total_bytes) {
    // host memory stands in for the device: report a generous fixed size
    *free_bytes = (size_t)16 << 30;
    *total_bytes = (size_t)16 << 30;
    return cudaSuccess;
}

cudaError_t cudaFree(void* p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaFreeAsync(void* p, cudaStream_t) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) {
    std::memmove(d, s, n);
    return cudaSuccess;
}
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) {
    std::memmove(d, s, n);
    return cudaSuccess;
}
cudaError_t cudaMemset(void* p, int v, size_t n) {
    std::memset(p, v, n);
    return cudaSuccess;
}
cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t) {
    if (emu::capture().on) {
        emu::capture().ops.push_back([=]() { std::memset(p, v, n); });
        return cudaSuccess;
    }
    std::memset(p, v, n);
    return cudaSuccess;
}
cudaError_t cudaEventCreate(cudaEvent_t* e) {
    *e = new EmuEvent();
    return cudaSuccess;
}
cudaError_t cudaEventDestroy(cudaEvent_t e) {
    delete e;
    return cudaSuccess;
}
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t) {
    e->t = emu::timer_ns();
    return cudaSuccess;
}
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = (float)((double)(b->t - a->t) / 1e6);
    return cudaSuccess;
}
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "emulated error"; }
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned) {
    *d = h;
    return cudaSuccess;
}
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned) {
    *p = poisoned_alloc(n);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFreeHost(void* p) {
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaStreamBeginCapture(cudaStream_t, cudaStreamCaptureMode) {
    emu::capture().on = true;
    emu::capture().ops.clear();
    return cudaSuccess;
}
cudaError_t cudaStreamEndCapture(cudaStream_t, cudaGraph_t* g) {
    auto* gr = new EmuGraph();
    gr->ops.swap(emu::capture().ops);
    emu::capture().on = false;
    *g = gr;
    return cudaSuccess;
}
cudaError_t cudaGraphInstantiate(cudaGraphExec_t* e, cudaGraph_t g, unsigned long long) {
    *e = new EmuGraph(*g);
    return cudaSuccess;
}
cudaError_t cudaGraphLaunch(cudaGraphExec_t e, cudaStream_t) {
    for (auto& op : e->ops) op();
    return cudaSuccess;
}
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t e) {
    delete e;
    return cudaSuccess;
}
cudaError_t cudaGraphDestroy(cudaGraph_t g) {
    delete g;
    return cudaSuccess;
}
