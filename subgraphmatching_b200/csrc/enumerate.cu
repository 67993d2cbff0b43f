// Device enumeration: one persistent, work-stealing kernel that counts
// embeddings for one or many queries.
//
// Execution model.  Every warp is an independent depth-first searcher.  Work
// items ("tasks") are prefixes of the search tree: for the candidate-table
// mode the entries of E[order0][order1] (a root and one depth-1 extension),
// for the cache mode the roots C(order0).  Tasks of all queries of a batch
// form one index space; warps claim `grab` consecutive tasks with one atomic
// on a global counter, so hub-rooted subtrees do not strand the rest of the
// grid behind one warp.
//
// Warp state.  The search state of depth d lives in lane d % 32 (second
// register set for depths 32..63): chosen candidate index and vertex, the
// current list (pointer + length), the next batch position and the valid-mask
// of the current 32-candidate batch.  Injectivity is a ballot over the lanes
// holding the chosen vertices (explore.h:548's vis[] without a |V| array).
//
// Set intersection (common_ops.h:248-254 semantics: sorted uint32 lists, the
// result keeps the shorter list's order) is warp-cooperative:
//   * merge: the longer list is staged in shared memory, chunk by chunk, by a
//     cp.async.bulk copy (16-byte aligned window, mbarrier completion with a
//     bounded wait) or by plain loads; lanes binary-search the shorter list's
//     elements in the staged chunk;
//   * galloping: when the longer list exceeds a chunk and is more than
//     gallop_ratio times longer, lanes binary-search it directly in global
//     memory (L2-resident rows).
// The last depth is never materialised: its count is |intersection| minus the
// already-embedded vertices that fall in it (rank lookups + membership tests).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "smx_internal.h"

namespace smx {

namespace {

struct BnRef {
    const uint32_t* off;   // candidate-table mode: E[bn][u] offsets
    const uint32_t* edge;  // candidate-table mode: E[bn][u] candidate indices
    uint32_t depth;        // depth of the backward neighbour
    uint32_t max_deg;
};

struct DepthInfo {
    const uint32_t* cand;  // C(u) (vertex ids, ascending)
    uint32_t u;            // query vertex at this depth
    uint32_t nbn;          // backward neighbours (explore.h: prevNeb[u].size())
    uint32_t bn_begin;     // into QPlan::bn
    uint32_t list_off;     // candidate-table mode: buffer holding this depth's list (kInvalid: the row itself)
    uint64_t anc;          // DAF ancestor mask (prune.h:100-104)
    uint32_t nops;         // cache mode: ops computed at this depth
    uint32_t ops_begin;    // into QPlan::op
    uint32_t iter_op;      // cache mode: op holding this depth's candidates
    uint32_t part_begin;   // candidate-table mode: partial intersections computed at this depth
    uint32_t npart;
    uint32_t pad;
};

// Candidate-table mode keeps, for every depth t with backward neighbours
// p_1 < ... < p_k, the partial intersections P_t^j = row_{p_1} ∩ ... ∩ row_{p_j}
// (j >= 2) in the warp scratch.  P_t^j is computed at depth p_j, right after
// the candidate of p_j is chosen, from P_t^{j-1} (still valid: it depends only
// on depths <= p_{j-1}).  The list of depth t is P_t^k, so a deep depth costs
// one intersection of a short partial with one row instead of an
// intersection of all k rows, and an empty partial prunes the candidate at
// once.  Buffers: word 0 holds the length, the elements start at word 4.
struct PartRef {
    uint32_t bn_first;  // BnRef of p_1 (P_t^1 is its row)
    uint32_t bn_this;   // BnRef of p_j
    uint32_t prev_off;  // buffer of P_t^{j-1}; kInvalid when j == 2
    uint32_t out_off;   // buffer of P_t^j
    uint32_t target;    // t
};

struct OpInfo {
    uint32_t parent;   // op id or kInvalid
    uint32_t vdepth;   // conf_dep when this op comes out empty (explore.h:233)
    uint32_t scr_off;  // result buffer in the warp scratch (elements)
    uint32_t pad;
};

struct QPlan {
    uint32_t n;          // query vertices
    uint32_t qn;         // rank directory stride
    uint32_t mode;       // smx_explore_kind
    uint32_t nops;
    uint64_t ntasks;
    uint32_t nroot;      // |C(order0)|
    uint32_t lane_depth; // candidate-table mode: from this depth on each lane enumerates its own subtree
    const uint2* rank;
    const uint64_t* mask;
    const uint64_t* off;    // data CSR
    const uint32_t* adj;
    const BnRef* bn;
    const OpInfo* op;
    const PartRef* part;
    // candidate-table mode, last depth L = n-1: its list without the row of
    // depth n-2 (G) is a row (leaf_g_bn), a partial (leaf_g_off) or unconstrained
    uint32_t leaf_inb;     // n-2 is a backward neighbour of L
    uint32_t leaf_g_bn;    // kInvalid unless G is one row
    uint32_t leaf_g_off;   // kInvalid unless G is a partial buffer
    uint32_t leaf_gp_off;  // buffer for G without the embedded vertices
    uint32_t leaf_bm;      // 1: G may be marked in the warp's bitmap (indices into C(u_L))
    uint32_t leaf_gdepth;  // deepest depth G depends on when < n-3 (G may stay marked), else kInvalid
    uint32_t hub_words;    // words per row of the hub adjacency matrix (0: none)
    const uint32_t* hub_id;
    const uint32_t* hub_bits;
    // factored tail (candidate-table mode): the lists S of depth n-2 and G of
    // the last depth (without depth n-2's row) depend only on depths <=
    // tail_depth (kInvalid: not used); tail_rev = E[u_L][u_{n-2}]
    uint32_t tail_depth;
    uint32_t tail_bms;     // word offset of S's bitmap after G's in the warp bitmap
    BnRef tail_rev;
    DepthInfo dep[kMaxQ];
};

struct EnumArgs {
    const QPlan* plans;
    const uint64_t* task_prefix;    // nq + 1
    unsigned long long* next_task;  // work queue head
    unsigned long long* qcount;     // per query
    uint32_t* qstop;                // per query: limit reached
    const uint64_t* qlimit;         // per query, 0 = none
    uint32_t* scratch;              // per warp lists
    unsigned long long* stats;      // [0] intersections [1] nodes [2] bytes [3] tasks [4] pruned
    int* status;                    // 0 ok, SMX_TIMEOUT, SMX_STOPPED, SMX_CUDA_ERROR
    unsigned long long* qstart;     // per query: %globaltimer when its first task began (per-query budgets)
    const volatile uint32_t* host_stop;
    uint64_t scratch_stride;        // elements per warp
    uint32_t* bitmap;               // per warp membership bitmap of the last depth's G (or null)
    uint64_t bm_stride;             // bitmap words per warp
    uint64_t budget_ns;             // time budget per warp from its start, 0 = none
    uint32_t bitmap_min;            // |G| from which the bitmap is used
    uint32_t nq;
    uint32_t max_ops;               // op-state entries per warp (cache mode)
    uint32_t grab;
    uint32_t chunk;                 // staged elements per warp
    uint32_t gallop_ratio;
    uint32_t use_tma;
    uint32_t failing_sets;
    uint32_t per_query;             // 1: budget_ns applies to each query from its first task (qstop = 2 on expiry)
    uint32_t pad;
};

// ------------------------------------------------------------------ staging

struct Stage {
    uint32_t* buf;      // shared, 16-byte aligned, chunk + 8 elements
    uint64_t* mbar;     // shared mbarrier (one arrival + tx bytes)
    uint32_t phase;
    uint32_t chunk;
    bool tma;
    bool failed;
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Copies src[0, len) (len <= chunk) into the stage buffer; returns the index
// of src[0] inside the buffer.  The bulk copy moves the 16-byte aligned
// window that covers the row (at most 3 elements before and after it; every
// list lives in an allocation padded by >= 32 bytes).
__device__ uint32_t stage_load(Stage& s, const uint32_t* src, uint32_t len) {
    const uint32_t lane = lane_id();
    __syncwarp();
    if (!s.tma || len < 64) {
        for (uint32_t i = lane; i < len; i += 32) s.buf[i] = src[i];
        __syncwarp();
        return 0;
    }
#ifdef SMX_EMU
    return 0;  // unreachable: the emulator runs with use_tma = 0
#else
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uintptr_t a0 = a & ~(uintptr_t)15;
    const uint32_t head = (uint32_t)((a - a0) >> 2);
    const uint32_t bytes = (uint32_t)(((a + (uintptr_t)len * 4 - a0) + 15) & ~(uintptr_t)15);
    const uint32_t mb = smem_addr(s.mbar);
    if (lane == 0) {
        // order the warp's earlier generic-proxy accesses (reads of the stage
        // buffer, writes of scratch lists that may be the source) before the
        // async-proxy copy
        asm volatile("fence.proxy.async;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb), "r"(bytes) : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(s.buf)),
            "l"(a0), "r"(bytes), "r"(mb)
            : "memory");
    }
    // bounded wait on the phase
    uint32_t done = 0;
    for (uint32_t it = 0; it < (1u << 24); ++it) {
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(mb), "r"(s.phase)
            : "memory");
        if (done) break;
    }
    if (!__all_sync(kFull, done)) s.failed = true;
    s.phase ^= 1u;
    __syncwarp();
    return head;
#endif
}

// ------------------------------------------------------------------ intersection
// Intersect sorted S[0, s) with sorted G[0, g), s <= g.  Writes the common
// elements (in S order) to out unless COUNT_ONLY; returns the count.  out may
// alias S (outputs never overtake the reads of the same batch).
template <bool COUNT_ONLY>
__device__ uint32_t isect(Stage& st, uint32_t gallop_ratio, const uint32_t* S, uint32_t s, const uint32_t* G,
                          uint32_t g, uint32_t* out) {
    const uint32_t lane = lane_id();
    uint32_t cnt = 0;
    if (s == 0 || g == 0) return 0;
    if (g > st.chunk && (uint64_t)s * gallop_ratio < g) {
        for (uint32_t base = 0; base < s; base += 32) {
            const uint32_t i = base + lane;
            bool f = false;
            uint32_t x = 0;
            if (i < s) {
                x = S[i];
                f = bsearch_global(G, g, x);
            }
            const uint32_t b = __ballot_sync(kFull, f);
            if (!COUNT_ONLY && f) out[cnt + __popc(b & lanemask_lt())] = x;
            cnt += __popc(b);
        }
        // callers read the list right away from other lanes
        __syncwarp();
        return cnt;
    }
    uint32_t sp = 0;
    for (uint32_t cb = 0; cb < g && sp < s; cb += st.chunk) {
        const uint32_t cl = min(st.chunk, g - cb);
        const uint32_t glast = G[cb + cl - 1];
        if (S[sp] > glast) continue;
        const uint32_t head = stage_load(st, G + cb, cl);
        const uint32_t* sh = st.buf + head;
        const uint32_t se = (cb + cl >= g) ? s : sp + upper_bound_global(S + sp, s - sp, glast);
        for (uint32_t base = sp; base < se; base += 32) {
            const uint32_t i = base + lane;
            bool f = false;
            uint32_t x = 0;
            if (i < se) {
                x = S[i];
                f = bsearch_shared(sh, cl, x);
            }
            const uint32_t b = __ballot_sync(kFull, f);
            if (!COUNT_ONLY && f) out[cnt + __popc(b & lanemask_lt())] = x;
            cnt += __popc(b);
        }
        sp = se;
    }
    __syncwarp();
    return cnt;
}

// ------------------------------------------------------------------ lane-distributed slots
#define SLOT_GET(f, d) __shfl_sync(kFull, ((d) < 32) ? f##0 : f##1, (d)&31)
// The value is evaluated by every lane before the owning lane stores it, so
// an argument that itself shuffles (SLOT_GET) never runs in one lane only.
#define SLOT_SET(f, d, x)                                \
    do {                                                 \
        const auto slot_v_ = (x);                        \
        if (lane == ((d)&31u)) {                         \
            if ((d) < 32) f##0 = slot_v_; else f##1 = slot_v_; \
        }                                                \
    } while (0)

struct Counters {
    unsigned long long isect = 0, nodes = 0, bytes = 0, tasks = 0, pruned = 0;
};

// Flags that other warps (or the host) write are read by every lane; the
// warp acts on the vote, so all lanes take the same branch even when the
// write lands between the lanes' reads.
__device__ __forceinline__ bool poll_abort(const EnumArgs& A) {
    return __any_sync(kFull, *reinterpret_cast<volatile int*>(A.status) != 0);
}

__device__ __forceinline__ bool query_stopped(const EnumArgs& A, uint32_t q) {
    return __any_sync(kFull, *reinterpret_cast<volatile uint32_t*>(A.qstop + q) != 0);
}

// The caller's stop word ends the launch; a passed deadline ends the launch,
// or with per-query budgets only query q (qstop[q] = 2).
__device__ void check_global_stop(const EnumArgs& A, uint64_t deadline, uint32_t q = 0) {
    if (lane_id() == 0) {
        int code = 0;
        if (A.host_stop && *A.host_stop) code = SMX_STOPPED;
        else if (deadline && global_timer_ns() > deadline) code = SMX_TIMEOUT;
        if (code == SMX_TIMEOUT && A.per_query) atomicCAS(A.qstop + q, 0u, 2u);
        else if (code) atomicCAS(A.status, 0, code);
    }
    __syncwarp();
}

// Per-task accumulation: flushed to the query's counter at task end and
// whenever it grows large, so a limit stops long subtrees early.
struct Tally {
    unsigned long long local = 0;
    uint32_t q = 0;
    uint32_t polls = 0;
    uint64_t deadline = 0;
};

__device__ __forceinline__ void flush_tally(const EnumArgs& A, Tally& T) {
    if (lane_id() == 0 && T.local) {
        const unsigned long long tot = atomicAdd(A.qcount + T.q, T.local) + T.local;
        if (A.qlimit[T.q] && tot >= A.qlimit[T.q]) atomicExch(A.qstop + T.q, 1u);
    }
    T.local = 0;
    __syncwarp();
}

// Periodic in-task check: abort flag, the query's limit, large local tallies;
// every 64th call also the caller's stop word and the time budget, so a long
// subtree notices them too.
__device__ __forceinline__ bool task_should_stop(const EnumArgs& A, Tally& T) {
    if (T.local > (1ull << 22)) flush_tally(A, T);
    if ((++T.polls & 63u) == 0) check_global_stop(A, T.deadline, T.q);
    const bool a = poll_abort(A);
    const bool b = query_stopped(A, T.q);
    return a || b;
}

// ================================================================== candidate-table mode
struct Row {
    const uint32_t* p;
    uint32_t len;
};

__device__ __forceinline__ Row table_row(const BnRef& r, uint32_t idx) {
    const uint32_t s = __ldg(r.off + idx);
    return Row{r.edge + s, __ldg(r.off + idx + 1) - s};
}

// Data vertices v (hub id hv, or kInvalid) and w adjacent?  Two hubs: one
// bit of the hub matrix; otherwise a binary search of the shorter row.
__device__ __forceinline__ bool adjacent(const QPlan& P, uint32_t v, uint32_t hv, uint32_t w, uint32_t hw) {
    if (hv != kInvalid && hw != kInvalid)
        return (__ldg(P.hub_bits + (size_t)hv * P.hub_words + (hw >> 5)) >> (hw & 31)) & 1u;
    const uint64_t ov = __ldg(P.off + v), ow = __ldg(P.off + w);
    const uint32_t dv = (uint32_t)(__ldg(P.off + v + 1) - ov), dw = (uint32_t)(__ldg(P.off + w + 1) - ow);
    return dv <= dw ? bsearch_ldg(P.adj + ov, dv, w) : bsearch_ldg(P.adj + ow, dw, v);
}

// Candidate list of depth D (CandidatesBuffer::getNextCandidatesImpl,
// explore.h:284-354): with one backward neighbour the table row itself (no
// copy), otherwise the intersection of all rows, shortest first, in the
// depth's scratch buffer.  For the last depth (COUNT_ONLY) returns
// |intersection| and leaves the two lists that define it in r0 / r1 for the
// conflict test.  Rows of the backward neighbour at skip_depth are left out;
// with no row left the result is "unconstrained" (returns kInvalid).
template <bool COUNT_ONLY>
__device__ uint32_t build_rows(const QPlan& P, const DepthInfo& D, uint32_t* scr, Stage& st, uint32_t gallop_ratio,
                               Counters& C, Row& r0, Row& r1, const uint32_t (&slot_idx)[2],
                               uint32_t skip_depth = kInvalid) {
    const uint32_t lane = lane_id();
    const uint32_t nb = D.nbn;
    // lane i < min(nb, 32) holds row i
    Row mine{nullptr, 0xffffffffu};
    bool mine_ok = false;
    {
        uint32_t bd = 0;
        BnRef R{};
        if (lane < nb) {
            R = P.bn[D.bn_begin + lane];
            bd = R.depth;
        }
        const uint32_t id_lo = __shfl_sync(kFull, slot_idx[0], bd & 31);
        const uint32_t id_hi = __shfl_sync(kFull, slot_idx[1], bd & 31);
        if (lane < nb && bd != skip_depth) {
            mine = table_row(R, bd < 32 ? id_lo : id_hi);
            mine_ok = true;
        }
    }
    const uint32_t avail0 = __ballot_sync(kFull, mine_ok);
    uint32_t extra = 0;  // rows beyond the first 32 (queries with more than 33 vertices)
    for (uint32_t i = 32; i < nb; ++i) extra += (P.bn[D.bn_begin + i].depth != skip_depth);
    const uint32_t nrows = __popc(avail0);
    const uint32_t total = nrows + extra;
    r1 = Row{nullptr, 0};
    if (total == 0) {
        r0 = Row{nullptr, 0};
        return kInvalid;
    }
    // order rows by length: repeatedly take the shortest unused one
    uint32_t used = ~avail0;  // bit per lane
    auto take_shortest = [&](Row& out) {
        const bool avail = !((used >> lane) & 1u);
        const uint32_t key = avail ? mine.len : 0xffffffffu;
        const uint32_t mn = __reduce_min_sync(kFull, key);
        const uint32_t who = __ffs(__ballot_sync(kFull, avail && key == mn)) - 1;
        used |= 1u << who;
        out.p = reinterpret_cast<const uint32_t*>(shfl64(reinterpret_cast<uint64_t>(mine.p), who));
        out.len = __shfl_sync(kFull, mine.len, who);
    };
    Row a, b;
    take_shortest(a);
    if (total == 1) {
        r0 = a;
        return a.len;
    }
    take_shortest(b);
    C.isect++;
    C.bytes += 4ull * (a.len + b.len);
    if (total == 2) {
        if (COUNT_ONLY) {
            r0 = a;
            r1 = b;
            return isect<true>(st, gallop_ratio, a.p, a.len, b.p, b.len, nullptr);
        }
        const uint32_t k = isect<false>(st, gallop_ratio, a.p, a.len, b.p, b.len, scr);
        r0 = Row{scr, k};
        return k;
    }
    // three or more rows: materialise all but the longest, then count with it
    uint32_t k = isect<false>(st, gallop_ratio, a.p, a.len, b.p, b.len, scr);
    for (uint32_t t = 2; t < nrows; ++t) {
        Row c;
        take_shortest(c);
        if (k == 0) {
            r0 = Row{scr, 0};
            return 0;
        }
        C.isect++;
        C.bytes += 4ull * (k + c.len);
        const bool last = (t + 1 == nrows) && extra == 0;
        if (last && COUNT_ONLY) {
            r0 = Row{scr, k};
            r1 = c;
            return isect<true>(st, gallop_ratio, scr, k, c.p, c.len, nullptr);
        }
        // k <= every row taken so far <= c.len: scr stays the shorter side (in place is safe)
        k = isect<false>(st, gallop_ratio, scr, k, c.p, c.len, scr);
    }
    // backward neighbours beyond 32 (queries with more than 33 vertices): in input order
    for (uint32_t i = 32; i < nb; ++i) {
        const BnRef R = P.bn[D.bn_begin + i];
        if (R.depth == skip_depth) continue;
        const uint32_t id = __shfl_sync(kFull, R.depth < 32 ? slot_idx[0] : slot_idx[1], R.depth & 31);
        const Row c = table_row(R, id);
        if (k == 0) break;
        C.isect++;
        C.bytes += 4ull * (k + c.len);
        if (k <= c.len) {
            k = isect<false>(st, gallop_ratio, scr, k, c.p, c.len, scr);
        } else {
            // the row is the shorter side: the output would overtake reads of scr,
            // so write it past scr's current contents first, then move it down
            const uint32_t k2 = isect<false>(st, gallop_ratio, c.p, c.len, scr, k, scr + k);
            for (uint32_t j = lane; j < k2; j += 32) scr[j] = scr[k + j];
            __syncwarp();
            k = k2;
        }
    }
    r0 = Row{scr, k};
    return k;
}

// Per-lane |row ∩ G|: row is a table row (read-only), G a sorted list in
// shared or global memory written by this warp (plain loads).  The shorter
// list is walked; the longer one is searched.  Searches in a long row run
// four at a time (independent branch-free searches) so four loads are in
// flight per step instead of one.
__device__ __forceinline__ uint32_t lane_count_common(const uint32_t* row, uint32_t nr, const uint32_t* G,
                                                      uint32_t ng) {
    if (nr == 0 || ng == 0) return 0;
    uint32_t cnt = 0;
    if (nr <= ng) {
        uint32_t lo = 0;
        for (uint32_t i = 0; i < nr; ++i) {
            const uint32_t x = __ldg(row + i);
            uint32_t l = lo, h = ng;
            while (l < h) {
                const uint32_t m = (l + h) >> 1;
                if (G[m] < x) l = m + 1; else h = m;
            }
            lo = l;
            if (lo == ng) break;
            cnt += G[lo] == x;
        }
        return cnt;
    }
    uint32_t lo = 0;  // every later element lies at or after row[lo]
    for (uint32_t i = 0; i < ng; i += 4) {
        const uint32_t x0 = G[i];
        const uint32_t x1 = i + 1 < ng ? G[i + 1] : x0;
        const uint32_t x2 = i + 2 < ng ? G[i + 2] : x0;
        const uint32_t x3 = i + 3 < ng ? G[i + 3] : x0;
        uint32_t b0 = lo, b1 = lo, b2 = lo, b3 = lo, n = nr - lo;
        while (n > 1) {
            const uint32_t h = n >> 1;
            b0 = __ldg(row + b0 + h) <= x0 ? b0 + h : b0;
            b1 = __ldg(row + b1 + h) <= x1 ? b1 + h : b1;
            b2 = __ldg(row + b2 + h) <= x2 ? b2 + h : b2;
            b3 = __ldg(row + b3 + h) <= x3 ? b3 + h : b3;
            n -= h;
        }
        cnt += __ldg(row + b0) == x0;
        if (i + 1 < ng) cnt += __ldg(row + b1) == x1;
        if (i + 2 < ng) cnt += __ldg(row + b2) == x2;
        if (i + 3 < ng) cnt += __ldg(row + b3) == x3;
        lo = i + 3 < ng ? b3 : lo;
    }
    return cnt;
}

__device__ __forceinline__ Row part_list(const uint32_t* scr, uint32_t off) {
    return Row{scr + off + 4, scr[off]};
}

__device__ __forceinline__ uint32_t slot_get(const uint32_t (&a)[2], uint32_t d) {
    return __shfl_sync(kFull, d < 32 ? a[0] : a[1], d & 31);
}

// Slot value of depth d for every lane, each lane naming its own d.
__device__ __forceinline__ uint32_t slot_get_any(const uint32_t (&a)[2], uint32_t d) {
    const uint32_t lo = __shfl_sync(kFull, a[0], d & 31);
    const uint32_t hi = __shfl_sync(kFull, a[1], d & 31);
    return d < 32 ? lo : hi;
}

// Computes the partial intersections that end at depth d (its candidate just
// chosen).  Returns false as soon as one is empty: no embedding extends the
// candidate.  Lane p describes part p.  Parts whose lists are both long go
// through the staged merge one at a time; the galloping ones (short list
// against a long row) run together, one lane per element of their short
// lists, so their binary searches overlap instead of following each other.
__device__ bool compute_parts(const QPlan& P, uint32_t d, uint32_t* scr, Stage& st, uint32_t gallop_ratio,
                              Counters& C, const uint32_t (&slot_idx)[2], const uint32_t (&slot_vid)[2]) {
    const DepthInfo& D = P.dep[d];
    const uint32_t lane = lane_id();
    // the vertex just chosen at depth d: galloping against its rows can test
    // adjacency directly (hub matrix) instead of searching the row
    const uint32_t vd = slot_get_any(slot_vid, d);
    const uint32_t hvd = (D.npart && P.hub_words) ? __ldg(P.hub_id + vd) : kInvalid;
    for (uint32_t base = 0; base < D.npart; base += 32) {
        const bool has = lane < D.npart - base;
        PartRef R{0, 0, kInvalid, 0};
        BnRef Bf{}, Bt{};
        if (has) {
            R = P.part[D.part_begin + base + lane];
            Bt = P.bn[R.bn_this];
            if (R.prev_off == kInvalid) Bf = P.bn[R.bn_first];
        }
        const uint32_t i_this = slot_get_any(slot_idx, has ? Bt.depth : 0);
        const uint32_t i_first = slot_get_any(slot_idx, has && R.prev_off == kInvalid ? Bf.depth : 0);
        Row a{nullptr, 0}, b{nullptr, 0};
        uint32_t* out = nullptr;
        const uint32_t* tcand = nullptr;  // C(u_t) when b is depth d's row (adjacency test possible)
        if (has) {
            a = R.prev_off == kInvalid ? table_row(Bf, i_first) : part_list(scr, R.prev_off);
            b = table_row(Bt, i_this);
            if (a.len > b.len) {
                const Row t = a;
                a = b;
                b = t;
            } else if (hvd != kInvalid) {
                tcand = P.dep[R.target].cand;
            }
            out = scr + R.out_off;
        }
        if (__any_sync(kFull, has && a.len == 0)) return false;
        C.isect += __popc(__ballot_sync(kFull, has));
        C.bytes += __reduce_add_sync(kFull, has ? 4u * (a.len + b.len) + 8u : 0u);
        const bool gal = has && (uint64_t)a.len * gallop_ratio < b.len;
        // long against long: staged merge, one part at a time
        uint32_t mm = __ballot_sync(kFull, has && !gal);
        while (mm) {
            const int p = __ffs(mm) - 1;
            mm &= mm - 1;
            const uint32_t* pa = reinterpret_cast<const uint32_t*>(shfl64(reinterpret_cast<uint64_t>(a.p), p));
            const uint32_t* pb = reinterpret_cast<const uint32_t*>(shfl64(reinterpret_cast<uint64_t>(b.p), p));
            uint32_t* po = reinterpret_cast<uint32_t*>(shfl64(reinterpret_cast<uint64_t>(out), p));
            const uint32_t la = __shfl_sync(kFull, a.len, p), lb = __shfl_sync(kFull, b.len, p);
            const uint32_t k = isect<false>(st, gallop_ratio, pa, la, pb, lb, po + 4);
            __syncwarp();
            if (lane == 0) po[0] = k;
            __syncwarp();
            if (k == 0) return false;
        }
        // short against long: all galloping parts in one pass
        const uint32_t gm = __ballot_sync(kFull, gal);
        if (!gm) continue;
        const uint32_t len_g = gal ? a.len : 0;
        uint32_t incl = len_g;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(kFull, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t excl = incl - len_g;
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        uint32_t found = 0;  // lane p: elements of part p kept so far
        for (uint32_t g0 = 0; g0 < total; g0 += 32) {
            const uint32_t gi = g0 + lane;
            uint32_t mp = 32, off = 0, mbl = 0;
            const uint32_t* ma = nullptr;
            const uint32_t* mb = nullptr;
            const uint32_t* mc = nullptr;
            for (uint32_t m = gm; m; m &= m - 1) {
                const int q = __ffs(m) - 1;
                const uint32_t ex = __shfl_sync(kFull, excl, q), ln = __shfl_sync(kFull, len_g, q);
                const uint64_t ap = shfl64(reinterpret_cast<uint64_t>(a.p), q);
                const uint64_t bp = shfl64(reinterpret_cast<uint64_t>(b.p), q);
                const uint64_t cp = shfl64(reinterpret_cast<uint64_t>(tcand), q);
                const uint32_t bl = __shfl_sync(kFull, b.len, q);
                if (gi < total && gi >= ex && gi < ex + ln) {
                    mp = (uint32_t)q;
                    off = gi - ex;
                    ma = reinterpret_cast<const uint32_t*>(ap);
                    mb = reinterpret_cast<const uint32_t*>(bp);
                    mc = reinterpret_cast<const uint32_t*>(cp);
                    mbl = bl;
                }
            }
            uint32_t x = 0;
            bool hit = false;
            if (mp < 32) {
                x = ma[off];
                if (mc) {
                    // x in row(v_d) <=> C(u_t)[x] adjacent to v_d
                    const uint32_t w = __ldg(mc + x);
                    hit = adjacent(P, vd, hvd, w, __ldg(P.hub_id + w));
                } else {
                    hit = bsearch_global(mb, mbl, x);
                }
            }
            for (uint32_t m = gm; m; m &= m - 1) {
                const int q = __ffs(m) - 1;
                const uint32_t hm = __ballot_sync(kFull, hit && mp == (uint32_t)q);
                if (!hm) continue;
                const uint32_t before = __shfl_sync(kFull, found, q);
                uint32_t* oq = reinterpret_cast<uint32_t*>(shfl64(reinterpret_cast<uint64_t>(out), q));
                if (hit && mp == (uint32_t)q) oq[4 + before + __popc(hm & lanemask_lt())] = x;
                if (lane == (uint32_t)q) found += __popc(hm);
            }
        }
        __syncwarp();
        if (gal) out[0] = found;
        __syncwarp();
        if (__any_sync(kFull, gal && found == 0)) return false;
    }
    return true;
}

// The part of the last depth L = n-1 that does not depend on the candidate
// chosen at depth n-2, set up once when depth n-2 is opened:
//   G      the last depth's list without the row of depth n-2 (a cached
//          partial, one row, or unconstrained when n-2 is L's only backward
//          neighbour); when n-2 is a backward neighbour, the embedded vertices
//          of depths 0 .. n-3 are taken out and the rest is staged in shared
//          memory when it fits;
//   prank  per lane j < n-2: the index in C(u_L) of the embedded vertex of
//          depth j if it is a candidate of u_L inside G, else kInvalid (still
//          needed only where G is unconstrained);
//   K0     |G| - #valid pranks (the count when n-2 is not a backward neighbour).
// Then every candidate of depth n-2 is counted by its own lane (leaf_batch).
// G longer than this stays marked across depth-(n-2) lists when it can
#ifndef SMX_LEAF_PERSIST_MIN
#define SMX_LEAF_PERSIST_MIN 256
#endif
struct LeafState {
    uint64_t gptr;
    uint32_t glen;
    uint32_t gany;
    uint32_t inb;      // n-2 is a backward neighbour of L
    uint32_t k0;
    BnRef row;         // E[u_{n-2}][u_L] when inb
    uint32_t prank0, prank1;
    uint64_t pmask;    // depths with a valid prank
    uint32_t* bm;      // the warp bitmap while G is marked in it, else null
    uint32_t persist;  // 1: G (with the embedded vertices) stays marked beyond this depth-(n-2) list
    uint32_t hub;      // 1: G's vertex ids and hub ids are staged after G (shared memory, words 256 / 512)
};

// Per-lane |row ∩ G| by probing G's membership bitmap: one independent load
// per row element (L2, where the warp's atomics set the bits).
__device__ __forceinline__ uint32_t lane_count_bitmap(const uint32_t* row, uint32_t n, const uint32_t* bm) {
    uint32_t cnt = 0, i = 0;
    for (; i + 4 <= n; i += 4) {
        const uint32_t x0 = __ldg(row + i), x1 = __ldg(row + i + 1), x2 = __ldg(row + i + 2), x3 = __ldg(row + i + 3);
        const uint32_t w0 = __ldcg(bm + (x0 >> 5)), w1 = __ldcg(bm + (x1 >> 5));
        const uint32_t w2 = __ldcg(bm + (x2 >> 5)), w3 = __ldcg(bm + (x3 >> 5));
        cnt += ((w0 >> (x0 & 31)) & 1u) + ((w1 >> (x1 & 31)) & 1u) + ((w2 >> (x2 & 31)) & 1u) + ((w3 >> (x3 & 31)) & 1u);
    }
    for (; i < n; ++i) {
        const uint32_t x = __ldg(row + i);
        cnt += (__ldcg(bm + (x >> 5)) >> (x & 31)) & 1u;
    }
    return cnt;
}

// Unmarks G in the warp bitmap (G is still where leaf_prepare put it: nothing
// else runs at depth n-2).
__device__ void leaf_clear(LeafState& S) {
    if (!S.bm) return;
    if (S.persist) {  // unmarked when its prefix changes
        S.bm = nullptr;
        return;
    }
    const uint32_t* g = reinterpret_cast<const uint32_t*>(S.gptr);
    __syncwarp();
    for (uint32_t i = lane_id(); i < S.glen; i += 32) atomicAnd(S.bm + (g[i] >> 5), ~(1u << (g[i] & 31)));
    __syncwarp();
    S.bm = nullptr;
}

__device__ void leaf_prepare(const QPlan& P, uint32_t* scr, Stage& st, const uint32_t (&slot_idx)[2],
                             const uint32_t (&slot_vid)[2], LeafState& S, uint32_t* bm, uint32_t bitmap_min,
                             bool& g_live) {
    const uint32_t lane = lane_id();
    const uint32_t L = P.n - 1;
    const DepthInfo& D = P.dep[L];
    Row G{nullptr, 0};
    S.gany = 1;
    if (P.leaf_g_off != kInvalid) {
        G = part_list(scr, P.leaf_g_off);
    } else if (P.leaf_g_bn != kInvalid) {
        const BnRef R = P.bn[P.leaf_g_bn];
        G = table_row(R, slot_get(slot_idx, R.depth));
    } else {
        S.gany = 0;
    }
    S.gptr = reinterpret_cast<uint64_t>(G.p);
    S.glen = G.len;
    S.inb = P.leaf_inb;
    if (S.inb) S.row = P.bn[D.bn_begin + D.nbn - 1];  // depth n-2 is the last backward neighbour
    uint64_t pm = 0;
    for (uint32_t half = 0; half < 2; ++half) {
        const uint32_t j = half * 32 + lane;
        uint32_t pr = kInvalid;
        if (j + 1 < L) {  // depths 0 .. n-3
            const uint32_t w = half ? slot_vid[1] : slot_vid[0];
            if ((__ldg(P.mask + w) >> D.u) & 1ull) {
                const uint32_t r = cand_rank(P.rank, P.qn, D.u, w);
                if (!S.gany || bsearch_global(G.p, G.len, r)) pr = r;
            }
        }
        if (half) S.prank1 = pr; else S.prank0 = pr;
        pm |= (uint64_t)__ballot_sync(kFull, pr != kInvalid) << (32 * half);
        if (L <= 33) {
            if (!half) S.prank1 = kInvalid;
            break;
        }
    }
    S.pmask = pm;
    S.k0 = S.glen - __popcll(pm);
    S.hub = 0;
    S.persist = 0;
    if (S.inb && S.gany && bm && P.leaf_gdepth != kInvalid && G.len > SMX_LEAF_PERSIST_MIN) {
        // a long G that depends only on depths above n-3: it stays marked
        // while they keep their candidates, and the embedded vertices in it
        // (pmask) are subtracted per candidate instead of being removed
        if (!g_live) {
            __syncwarp();
            for (uint32_t i = lane; i < G.len; i += 32) atomicOr(bm + (G.p[i] >> 5), 1u << (G.p[i] & 31));
            __syncwarp();
            g_live = true;
        }
        S.bm = bm;
        S.persist = 1;
        return;
    }
    if (S.inb && S.gany) {
        // G minus the embedded vertices, into shared memory when it fits (the
        // stage buffer is idle until depth n-2 is left), else into its buffer;
        // the cached partial itself stays intact for other prefixes
        const bool in_smem = G.len <= st.chunk;
        uint32_t* dst = in_smem ? st.buf : scr + P.leaf_gp_off + 4;
        uint32_t k = 0;
        __syncwarp();
        for (uint32_t base = 0; base < G.len; base += 32) {
            const uint32_t i = base + lane;
            uint32_t x = 0;
            bool keep = false;
            if (i < G.len) {
                x = G.p[i];
                keep = true;
            }
            uint64_t m = pm;
            while (m) {
                const int j = __ffsll((long long)m) - 1;
                m &= m - 1;
                const uint32_t r = __shfl_sync(kFull, j < 32 ? S.prank0 : S.prank1, j & 31);
                keep &= x != r;
            }
            const uint32_t bal = __ballot_sync(kFull, keep);
            if (keep) dst[k + __popc(bal & lanemask_lt())] = x;
            k += __popc(bal);
        }
        __syncwarp();
        S.gptr = reinterpret_cast<uint64_t>(dst);
        S.glen = k;
        S.pmask = 0;
        S.k0 = k;
        S.hub = 0;
        if (in_smem && k <= 256 && st.chunk >= 768 && P.hub_words) {
            // G's data vertices and their hub ids, for adjacency tests per lane
            const uint32_t* candL = D.cand;
            for (uint32_t i = lane; i < k; i += 32) {
                const uint32_t w = __ldg(candL + dst[i]);
                st.buf[256 + i] = w;
                st.buf[512 + i] = __ldg(P.hub_id + w);
            }
            __syncwarp();
            S.hub = 1;
        }
        if (bm && P.leaf_bm && k >= bitmap_min) {
            for (uint32_t i = lane; i < k; i += 32) atomicOr(bm + (dst[i] >> 5), 1u << (dst[i] & 31));
            __syncwarp();
            S.bm = bm;
        }
    }
}

// Counts the last depth for every valid candidate of the current depth-(n-2)
// batch at once, one candidate per lane.  Adds the algorithmic bytes of the
// whole warp to C.bytes.
__device__ uint64_t leaf_batch(const QPlan& P, const LeafState& S, const uint32_t* lp, uint32_t base, uint32_t vm,
                               Counters& C, const uint32_t* st_buf) {
    const uint32_t lane = lane_id();
    const uint32_t L = P.n - 1;
    const uint32_t u = P.dep[L].u;
    const bool mine = (vm >> lane) & 1u;
    uint64_t cnt = 0;
    uint32_t row_len = 0, bytes = 0;
    const uint32_t* row = nullptr;
    if (mine) {
        const uint32_t c = lp[base + lane];
        if (!S.inb) {
            const uint32_t v = __ldg(P.dep[L - 1].cand + c);
            uint32_t hit = 0;
            if ((__ldg(P.mask + v) >> u) & 1ull)
                hit = bsearch_global(reinterpret_cast<const uint32_t*>(S.gptr), S.glen,
                                     cand_rank(P.rank, P.qn, u, v));
            cnt = S.k0 - hit;
            bytes = 16;
        } else {
            const Row r = table_row(S.row, c);
            row = r.p;
            row_len = r.len;
            uint32_t vc = 0, hc = kInvalid;
            if (S.hub) {
                vc = __ldg(P.dep[L - 1].cand + c);
                hc = __ldg(P.hub_id + vc);
            }
            if (hc != kInvalid && r.len > S.glen) {
                // a hub candidate: test each vertex of G against it (the hub
                // matrix for hub pairs, independent loads) instead of
                // searching its long row
                const uint32_t* gv = st_buf + 256;
                const uint32_t* gh = st_buf + 512;
                uint32_t k = 0;
                for (uint32_t i = 0; i < S.glen; ++i) k += adjacent(P, vc, hc, gv[i], gh[i]);
                cnt = k;
                bytes = 12 + 4 * S.glen;
            } else if (S.bm && r.len <= S.glen * (32u - __clz(r.len))) {
                // probes of the bitmap (independent loads) cost less than
                // |G| searches of the row (dependent loads)
                cnt = lane_count_bitmap(r.p, r.len, S.bm);
                bytes = 12 + 8 * r.len;
            } else {
                cnt = S.gany ? lane_count_common(r.p, r.len, reinterpret_cast<const uint32_t*>(S.gptr), S.glen)
                             : r.len;
                bytes = 12 + (S.gany ? 4 * (r.len + S.glen) : 0);
            }
        }
    }
    if (S.inb && S.pmask) {
        // unconstrained G: embedded vertices that lie in this lane's row
        uint64_t pm = S.pmask;
        while (pm) {
            const int j = __ffsll((long long)pm) - 1;
            pm &= pm - 1;
            const uint32_t r = __shfl_sync(kFull, j < 32 ? S.prank0 : S.prank1, j & 31);
            if (mine && bsearch_global(row, row_len, r)) --cnt;
        }
    }
    // warp sums
    uint32_t lo = (uint32_t)cnt, hi = (uint32_t)(cnt >> 32);
    for (int o = 16; o; o >>= 1) {
        const uint32_t l2 = __shfl_xor_sync(kFull, lo, o);
        const uint32_t h2 = __shfl_xor_sync(kFull, hi, o);
        const uint64_t s = ((uint64_t)hi << 32 | lo) + ((uint64_t)h2 << 32 | l2);
        lo = (uint32_t)s;
        hi = (uint32_t)(s >> 32);
        bytes += __shfl_xor_sync(kFull, bytes, o);
    }
    C.bytes += bytes;
    return (uint64_t)hi << 32 | lo;
}

// Full-warp count of the last depth L for the current prefix (depths < L set).
__device__ uint64_t last_depth_count(const QPlan& P, uint32_t L, uint32_t* scr_base, Stage& st,
                                     uint32_t gallop_ratio, Counters& C, const uint32_t (&slot_idx)[2],
                                     const uint32_t (&slot_vid)[2]) {
    const uint32_t lane = lane_id();
    const DepthInfo& D = P.dep[L];
    Row r0, r1;
    // at most two rows here (n == 3): counted without a buffer
    const uint32_t k = build_rows<true>(P, D, scr_base, st, gallop_ratio, C, r0, r1, slot_idx);
    if (k == 0) return 0;
    // embedded vertices that are candidates of u_L and lie in the result
    uint32_t conflicts = 0;
    for (uint32_t half = 0; half < 2; ++half) {
        const uint32_t j = half * 32 + lane;
        bool in = false;
        if (j < L) {
            const uint32_t v = half ? slot_vid[1] : slot_vid[0];
            if ((__ldg(P.mask + v) >> D.u) & 1ull) {
                const uint32_t r = cand_rank(P.rank, P.qn, D.u, v);
                in = bsearch_global(r0.p, r0.len, r) && (r1.p == nullptr || bsearch_global(r1.p, r1.len, r));
            }
        }
        conflicts += __popc(__ballot_sync(kFull, in));
        if (L <= 32) break;
    }
    return (uint64_t)(k - conflicts);
}

// ------------------------------------------------------------------ lane-level subtrees
// Below the plan's lane depth every list is an intersection of table rows and
// short, so a warp gains nothing from sharing one list: each lane takes one
// candidate of the batch and enumerates its subtree on its own (a plain
// depth-first search with no warp collectives).  A depth's candidates are
// produced by walking its shortest row and probing the others (binary
// search), so nothing is materialised.

__device__ __forceinline__ Row row_at(const BnRef& r, const uint32_t* idx) {
    const uint32_t i = idx[r.depth];
    const uint32_t s = __ldg(r.off + i);
    return Row{r.edge + s, __ldg(r.off + i + 1) - s};
}

__device__ __forceinline__ bool in_row(const uint32_t* p, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t m = (lo + hi) >> 1;
        if (__ldg(p + m) < x) lo = m + 1; else hi = m;
    }
    return lo < n && __ldg(p + lo) == x;
}

// x (an index into C(u_d)) lies in every row of depth d except row `skip`.
__device__ __forceinline__ bool in_other_rows(const QPlan& P, const DepthInfo& D, uint32_t skip, const uint32_t* idx,
                                              uint32_t x) {
    for (uint32_t i = 0; i < D.nbn; ++i) {
        if (i == skip) continue;
        const Row r = row_at(P.bn[D.bn_begin + i], idx);
        if (!in_row(r.p, r.len, x)) return false;
    }
    return true;
}

__device__ __forceinline__ uint32_t shortest_row(const QPlan& P, const DepthInfo& D, const uint32_t* idx, Row& best) {
    uint32_t bi = 0;
    best = row_at(P.bn[D.bn_begin], idx);
    for (uint32_t i = 1; i < D.nbn; ++i) {
        const Row r = row_at(P.bn[D.bn_begin + i], idx);
        if (r.len < best.len) {
            best = r;
            bi = i;
        }
    }
    return bi;
}

// Count of the last depth for the lane's prefix: |∩ rows| minus embedded
// vertices inside it (rl[j] = index of depth j's vertex in C(u_L) or kInvalid).
__device__ uint64_t lane_leaf(const QPlan& P, const uint32_t* idx, const uint32_t* rl, uint32_t L, uint32_t& work) {
    const DepthInfo& D = P.dep[L];
    Row drv;
    const uint32_t di = shortest_row(P, D, idx, drv);
    work += D.nbn == 1 ? 1 : drv.len;
    uint64_t k;
    if (D.nbn == 1) {
        k = drv.len;
    } else {
        k = 0;
        for (uint32_t i = 0; i < drv.len; ++i) k += in_other_rows(P, D, di, idx, __ldg(drv.p + i));
    }
    if (k == 0) return 0;
    for (uint32_t j = 0; j < L; ++j) {
        const uint32_t r = rl[j];
        if (r != kInvalid && in_row(drv.p, drv.len, r) && (D.nbn == 1 || in_other_rows(P, D, di, idx, r))) --k;
    }
    return k;
}

__device__ __forceinline__ uint32_t rank_in_last(const QPlan& P, uint32_t v) {
    const uint32_t u = P.dep[P.n - 1].u;
    return ((__ldg(P.mask + v) >> u) & 1ull) ? cand_rank(P.rank, P.qn, u, v) : kInvalid;
}

// Stop test for a lane running on its own: the warp-level checks cannot be
// used there, so the lane reads the flags itself.
__device__ bool lane_should_stop(const EnumArgs& A, uint32_t q, uint64_t deadline) {
    if (*reinterpret_cast<volatile int*>(A.status) != 0) return true;
    if (*reinterpret_cast<volatile uint32_t*>(A.qstop + q) != 0) return true;
    int code = 0;
    if (A.host_stop && *A.host_stop) code = SMX_STOPPED;
    else if (deadline && global_timer_ns() > deadline) code = SMX_TIMEOUT;
    if (code == SMX_TIMEOUT && A.per_query) {
        atomicCAS(A.qstop + q, 0u, 2u);
        return true;
    }
    if (code) {
        atomicCAS(A.status, 0, code);
        return true;
    }
    return false;
}

struct LaneWork {
    unsigned long long nodes = 0, bytes = 0;
};

// Enumerates depths d0+1 .. n-1 below the lane's candidate at depth d0 (idx,
// vid, rl hold depths 0 .. d0).  Embeddings found are added to the query's
// counter in chunks (so a count limit stops other warps early) and the rest
// is returned.
__device__ uint64_t lane_subtree(const EnumArgs& A, const QPlan& P, uint32_t d0, uint32_t* idx, uint32_t* vid,
                                 uint32_t* rl, const Tally& T, LaneWork& W) {
    const uint32_t L = P.n - 1;
    uint32_t dl[kMaxQ], dp[kMaxQ], db[kMaxQ];
    const uint32_t* de[kMaxQ];
    uint64_t cnt = 0;
    uint32_t d = d0 + 1;
    auto open = [&](uint32_t dd) {
        Row r;
        db[dd] = shortest_row(P, P.dep[dd], idx, r);
        de[dd] = r.p;
        dl[dd] = r.len;
        dp[dd] = 0;
    };
    open(d);
    // work since the last stop test: row elements walked plus leaf counts
    uint32_t work = 0;
    for (;;) {
        if (++work >= 1024u) {
            work = 0;
            if (lane_should_stop(A, T.q, T.deadline)) break;
            if (cnt >= (1u << 20)) {
                const unsigned long long tot = atomicAdd(A.qcount + T.q, cnt) + cnt;
                if (A.qlimit[T.q] && tot >= A.qlimit[T.q]) atomicExch(A.qstop + T.q, 1u);
                cnt = 0;
            }
        }
        const DepthInfo& D = P.dep[d];
        bool found = false;
        uint32_t x = 0, v = 0;
        while (dp[d] < dl[d]) {
            x = __ldg(de[d] + dp[d]++);
            W.bytes += 4;
            ++work;
            if (D.nbn > 1 && !in_other_rows(P, D, db[d], idx, x)) continue;
            v = __ldg(D.cand + x);
            W.bytes += 4;
            bool clash = false;
            for (uint32_t j = 0; j < d && !clash; ++j) clash = (vid[j] == v);
            if (clash) continue;
            found = true;
            break;
        }
        if (!found) {
            if (d == d0 + 1) break;
            --d;
            continue;
        }
        idx[d] = x;
        vid[d] = v;
        rl[d] = rank_in_last(P, v);
        W.nodes++;
        if (d + 1 == L) {
            cnt += lane_leaf(P, idx, rl, L, work);
            continue;
        }
        ++d;
        open(d);
    }
    return cnt;
}

// ------------------------------------------------------------------ factored tail
// When S (the list of depth n-2) and G (the last depth's list without the
// row of depth n-2) depend only on depths <= a < n-3, the count below a
// depth-(n-3) node is
//   sum over c in S \ E, g in G \ E of [c ~ g]
// with E the vertices embedded at depths 0 .. n-3.  By inclusion-exclusion
//   = B - sum_{e in E ∩ S} |N(e) ∩ G| - sum_{e in E ∩ G} |N(e) ∩ S|
//       + #{(e, f) in (E ∩ S) x (E ∩ G) : e ~ f}
// where B = sum_{c in S} |N(c) ∩ G| is computed once per depth-a node.  S and
// G stay marked in the warp's bitmaps (over C(u_{n-2}) and C(u_L) indices)
// while they are valid.

__device__ __forceinline__ Row tail_list(const QPlan& P, uint32_t* scr, uint32_t off, uint32_t bn,
                                         const uint32_t (&slot_idx)[2]) {
    if (off != kInvalid) return part_list(scr, off);
    const BnRef R = P.bn[bn];
    return table_row(R, slot_get(slot_idx, R.depth));
}

__device__ void tail_mark(Row X, uint32_t* bmx, bool set) {
    __syncwarp();
    for (uint32_t i = lane_id(); i < X.len; i += 32) {
        const uint32_t x = X.p[i];
        if (set) atomicOr(bmx + (x >> 5), 1u << (x & 31));
        else atomicAnd(bmx + (x >> 5), ~(1u << (x & 31)));
    }
    __syncwarp();
}

__device__ __forceinline__ bool bm_test(const uint32_t* bmx, uint32_t x) {
    return (__ldcg(bmx + (x >> 5)) >> (x & 31)) & 1u;
}

// B = sum over c in S of |row_{n-2 -> L}(c) ∩ G| (G marked in bmG)
__device__ uint64_t tail_base(Row S, const BnRef& rowSL, const uint32_t* bmG, Counters& C) {
    uint64_t sum = 0;
    uint32_t bytes = 0;
    for (uint32_t base = 0; base < S.len; base += 32) {
        const uint32_t i = base + lane_id();
        if (i < S.len) {
            const Row r = table_row(rowSL, S.p[i]);
            sum += lane_count_bitmap(r.p, r.len, bmG);
            bytes += 8 * r.len;
        }
    }
    for (int o = 16; o; o >>= 1) {
        sum += __shfl_xor_sync(kFull, sum, o);
        bytes += __shfl_xor_sync(kFull, bytes, o);
    }
    C.bytes += bytes;
    return sum;
}

// B - the corrections for E = the vertices at depths 0 .. n-3
__device__ uint64_t tail_count(const QPlan& P, uint64_t base, const uint32_t (&slot_vid)[2], const BnRef& rowSL,
                               const uint32_t* bmS, const uint32_t* bmG) {
    const uint32_t lane = lane_id();
    const uint32_t nE = P.n - 2;
    const uint32_t uS = P.dep[P.n - 2].u, uL = P.dep[P.n - 1].u;
    uint32_t e[2], he[2];
    bool inS[2], inG[2];
    uint64_t t12 = 0;
    for (uint32_t h = 0; h < 2; ++h) {
        const uint32_t j = h * 32 + lane;
        e[h] = kInvalid;
        he[h] = kInvalid;
        inS[h] = inG[h] = false;
        if (j < nE) {
            e[h] = slot_vid[h];
            const uint64_t m = __ldg(P.mask + e[h]);
            if ((m >> uS) & 1ull) {
                const uint32_t rS = cand_rank(P.rank, P.qn, uS, e[h]);
                if (bm_test(bmS, rS)) {
                    inS[h] = true;
                    const Row r = table_row(rowSL, rS);
                    t12 += lane_count_bitmap(r.p, r.len, bmG);
                }
            }
            if ((m >> uL) & 1ull) {
                const uint32_t rG = cand_rank(P.rank, P.qn, uL, e[h]);
                if (bm_test(bmG, rG)) {
                    inG[h] = true;
                    const Row r = table_row(P.tail_rev, rG);
                    t12 += lane_count_bitmap(r.p, r.len, bmS);
                }
            }
            if (P.hub_words) he[h] = __ldg(P.hub_id + e[h]);
        }
    }
    // pairs (e in S, f in G) of embedded vertices that are adjacent
    uint64_t t3 = 0;
    for (uint32_t hf = 0; hf < 2; ++hf) {
        for (uint32_t gm = __ballot_sync(kFull, inG[hf]); gm; gm &= gm - 1) {
            const int q = __ffs(gm) - 1;
            const uint32_t f = __shfl_sync(kFull, e[hf], q), hfid = __shfl_sync(kFull, he[hf], q);
            for (uint32_t h = 0; h < 2; ++h)
                if (inS[h] && e[h] != f) t3 += adjacent(P, e[h], he[h], f, hfid);
        }
    }
    for (int o = 16; o; o >>= 1) {
        t12 += __shfl_xor_sync(kFull, t12, o);
        t3 += __shfl_xor_sync(kFull, t3, o);
    }
    return base - t12 + t3;
}

// One task: root r = row of entry t in E[o0][o1], depth-1 candidate edge[t].
__device__ void run_table_task(const EnumArgs& A, const QPlan& P, uint64_t t, uint32_t* scr, uint32_t* bm, Stage& st,
                               Counters& C, Tally& T) {
    unsigned long long& local = T.local;
    const uint32_t lane = lane_id();
    const uint32_t n = P.n;
    const DepthInfo& D0 = P.dep[0];
    const DepthInfo& D1 = P.dep[1];
    const BnRef R01 = P.bn[D1.bn_begin];
    // root index: last r with off[r] <= t (off has |C(o0)| + 1 entries)
    uint32_t lo = 0, hi = P.nroot;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((uint64_t)__ldg(R01.off + mid) <= t) lo = mid; else hi = mid;
    }
    const uint32_t r = lo;
    const uint32_t c1 = __ldg(R01.edge + t);
    const uint32_t v0 = __ldg(D0.cand + r);
    const uint32_t v1 = __ldg(D1.cand + c1);
    C.tasks++;
    C.bytes += 8;
    if (v0 == v1) return;
    if (n == 2) {
        local += 1;
        return;
    }
    uint32_t slot_idx[2] = {0, 0}, slot_vid[2] = {kInvalid, kInvalid};
    uint32_t pos0 = 0, pos1 = 0, len0 = 0, len1 = 0, vm0 = 0, vm1 = 0;
    uint64_t ptr0 = 0, ptr1 = 0;
    if (lane == 0) { slot_idx[0] = r; slot_vid[0] = v0; }
    if (lane == 1) { slot_idx[0] = c1; slot_vid[0] = v1; }
    C.nodes += 2;
    if (n == 3) {
        local += last_depth_count(P, 2, scr, st, A.gallop_ratio, C, slot_idx, slot_vid);
        return;
    }
    // aliases used by SLOT_GET / SLOT_SET
#define idx0 slot_idx[0]
#define idx1 slot_idx[1]
#define vid0 slot_vid[0]
#define vid1 slot_vid[1]
    // partials ending at depth 1 (depth 0 is every target's first backward neighbour)
    if (!compute_parts(P, 1, scr, st, A.gallop_ratio, C, slot_idx, slot_vid)) return;
    uint32_t d = 2;
    LeafState leaf;
    leaf.bm = nullptr;
    leaf.persist = 0;
    // a long G kept marked across depth-(n-2) lists (see leaf_prepare)
    bool g_live = false;
    auto g_drop = [&]() {
        if (!g_live) return;
        const Row G = tail_list(P, scr, P.leaf_g_off, P.leaf_g_bn, slot_idx);
        __syncwarp();
        for (uint32_t i = lane; i < G.len; i += 32) atomicAnd(bm + (G.p[i] >> 5), ~(1u << (G.p[i] & 31)));
        __syncwarp();
        g_live = false;
    };
    // factored tail: S and G marked in the bitmaps and B valid for the current prefix
    const bool tail = P.tail_depth != kInvalid && bm != nullptr;
    bool tail_live = false;
    uint64_t tail_b = 0;
    const DepthInfo& DL = P.dep[n - 1];
    const BnRef rowSL = P.bn[DL.bn_begin + DL.nbn - 1];
    uint32_t* bmG = bm;
    uint32_t* bmS = bm ? bm + P.tail_bms : nullptr;
    auto tail_lists = [&](Row& S, Row& G) {
        S = tail_list(P, scr, P.dep[n - 2].list_off, P.dep[n - 2].bn_begin, slot_idx);
        G = tail_list(P, scr, P.leaf_g_off, P.leaf_g_bn, slot_idx);
    };
    auto tail_drop = [&]() {
        if (!tail_live) return;
        Row S, G;
        tail_lists(S, G);
        tail_mark(S, bmS, false);
        tail_mark(G, bmG, false);
        tail_live = false;
    };
    auto open_depth = [&](uint32_t dd) {
        const DepthInfo& D = P.dep[dd];
        Row r;
        if (D.list_off != kInvalid) {
            r = part_list(scr, D.list_off);
        } else {
            const BnRef R = P.bn[D.bn_begin];
            r = table_row(R, SLOT_GET(idx, R.depth));
        }
        SLOT_SET(ptr, dd, reinterpret_cast<uint64_t>(r.p));
        SLOT_SET(len, dd, r.len);
        SLOT_SET(pos, dd, 0u);
        SLOT_SET(vm, dd, 0u);
        if (tail && dd + 2 == n) {
            // the whole subtree below this depth-(n-3) node, counted at once
            if (!tail_live) {
                Row S, G;
                tail_lists(S, G);
                tail_mark(S, bmS, true);
                tail_mark(G, bmG, true);
                tail_b = tail_base(S, rowSL, bmG, C);
                tail_live = true;
            }
            local += tail_count(P, tail_b, slot_vid, rowSL, bmS, bmG);
            C.nodes += r.len;
            SLOT_SET(len, dd, 0u);
            return;
        }
        if (dd + 2 == n && r.len) leaf_prepare(P, scr, st, slot_idx, slot_vid, leaf, bm, A.bitmap_min, g_live);
    };
    open_depth(2);
    uint32_t iter = 0;
    for (;;) {
        if ((++iter & 255u) == 0 && task_should_stop(A, T)) break;
        uint32_t vm = SLOT_GET(vm, d);
        if (vm == 0) {
            const uint32_t pos = SLOT_GET(pos, d);
            const uint32_t len = SLOT_GET(len, d);
            if (pos >= len) {
                if (d + 2 == n) leaf_clear(leaf);
                if (d == 2) break;
                --d;
                continue;
            }
            const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
            const DepthInfo& D = P.dep[d];
            const uint32_t i = pos + lane;
            uint32_t v = kInvalid;
            if (i < len) v = __ldg(D.cand + lp[i]);
            bool clash = false;
            for (uint32_t j = 0; j < d; ++j) clash |= (SLOT_GET(vid, j) == v);
            vm = __ballot_sync(kFull, i < len && !clash);
            C.bytes += 8ull * min(32u, len - pos);
            SLOT_SET(pos, d, pos + 32);
            SLOT_SET(vm, d, vm);
            continue;
        }
        if (d >= P.lane_depth && d + 2 < n) {
            // each lane enumerates the subtree of one candidate of the batch
            const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
            const uint32_t base = SLOT_GET(pos, d) - 32;
            uint32_t lidx[kMaxQ], lvid[kMaxQ], lrl[kMaxQ];
            const uint32_t my_rl_lo = lane < d ? rank_in_last(P, vid0) : kInvalid;
            const uint32_t my_rl_hi = lane + 32 < d ? rank_in_last(P, vid1) : kInvalid;
            for (uint32_t j = 0; j < d; ++j) {
                lidx[j] = SLOT_GET(idx, j);
                lvid[j] = SLOT_GET(vid, j);
                lrl[j] = __shfl_sync(kFull, j < 32 ? my_rl_lo : my_rl_hi, j & 31);
            }
            uint64_t mine = 0;
            LaneWork W;
            if ((vm >> lane) & 1u) {
                const uint32_t c = lp[base + lane];
                lidx[d] = c;
                lvid[d] = __ldg(P.dep[d].cand + c);
                lrl[d] = rank_in_last(P, lvid[d]);
                mine = lane_subtree(A, P, d, lidx, lvid, lrl, T, W);
            }
            __syncwarp();
            for (int o = 16; o; o >>= 1) {
                mine += __shfl_xor_sync(kFull, mine, o);
                W.nodes += __shfl_xor_sync(kFull, W.nodes, o);
                W.bytes += __shfl_xor_sync(kFull, W.bytes, o);
            }
            local += mine;
            C.nodes += __popc(vm) + W.nodes;
            C.bytes += W.bytes;
            SLOT_SET(vm, d, 0u);
            continue;
        }
        if (d + 2 == n) {
            // all valid candidates of this batch at once, one per lane
            const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
            const uint32_t base = SLOT_GET(pos, d) - 32;
            local += leaf_batch(P, leaf, lp, base, vm, C, st.buf);
            C.nodes += __popc(vm);
            SLOT_SET(vm, d, 0u);
            continue;
        }
        const uint32_t b = __ffs(vm) - 1;
        SLOT_SET(vm, d, vm & (vm - 1));
        const uint32_t pos = SLOT_GET(pos, d) - 32 + b;
        const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
        const uint32_t c = lp[pos];
        const uint32_t v = __ldg(P.dep[d].cand + c);
        if (tail && d <= P.tail_depth) tail_drop();  // S and G change with this depth
        if (d <= P.leaf_gdepth) g_drop();             // as does a persistent G
        SLOT_SET(idx, d, c);
        SLOT_SET(vid, d, v);
        C.nodes++;
        if (!compute_parts(P, d, scr, st, A.gallop_ratio, C, slot_idx, slot_vid)) continue;
        ++d;
        open_depth(d);
    }
    leaf_clear(leaf);  // a stop can leave depth n-2 early
    tail_drop();
    g_drop();
#undef idx0
#undef idx1
#undef vid0
#undef vid1
}

// ================================================================== cache + failing-set mode
// explore_Intersection_Cache_DAF_Filter (explore.h:968-1129) with
// CacheBuffer::getNextCandidatesImpl (explore.h:200-243) and DAFFailingPrune
// (prune.h:82-171).  Op results are data-vertex lists: ops without a parent
// alias the adjacency row of the vertex just chosen; the others are
// parent ∩ N(v) in the op's scratch buffer.  Candidates are filtered by the
// candidate mask (candidates_exsist, explore.h:998).

struct OpState {  // per warp, in shared memory
    const uint32_t* p;
    uint32_t len;
    uint32_t pad;
};

// Computes the ops of depth dd for vertex v.  Returns kInvalid on success,
// else the vdepth of the first empty op (conf_dep).
__device__ uint32_t compute_ops(const QPlan& P, uint32_t dd, uint32_t v, uint32_t* scr, OpState* ops, Stage& st,
                                uint32_t gallop_ratio, Counters& C) {
    const DepthInfo& D = P.dep[dd];
    const uint64_t o0 = __ldg(P.off + v);
    const uint32_t dv = (uint32_t)(__ldg(P.off + v + 1) - o0);
    const uint32_t* nv = P.adj + o0;
    // v a hub: a short parent list is tested against v by adjacency (hub
    // matrix or the shorter row) instead of searching v's long row
    const uint32_t hv = (D.nops && P.hub_words) ? __ldg(P.hub_id + v) : kInvalid;
    for (uint32_t k = 0; k < D.nops; ++k) {
        const uint32_t id = D.ops_begin + k;
        const OpInfo O = P.op[id];
        uint32_t len;
        const uint32_t* p;
        if (O.parent == kInvalid) {
            p = nv;
            len = dv;
        } else {
            const OpState par = ops[O.parent];
            uint32_t* out = scr + O.scr_off;
            C.isect++;
            C.bytes += 4ull * (par.len + dv);
            if (hv != kInvalid && (uint64_t)par.len * gallop_ratio < dv) {
                len = 0;
                for (uint32_t base = 0; base < par.len; base += 32) {
                    const uint32_t i = base + lane_id();
                    uint32_t x = 0;
                    bool hit = false;
                    if (i < par.len) {
                        x = par.p[i];
                        hit = adjacent(P, v, hv, x, __ldg(P.hub_id + x));
                    }
                    const uint32_t b = __ballot_sync(kFull, hit);
                    if (hit) out[len + __popc(b & lanemask_lt())] = x;
                    len += __popc(b);
                }
                __syncwarp();
            } else if (par.len <= dv) {
                len = isect<false>(st, gallop_ratio, par.p, par.len, nv, dv, out);
            } else {
                len = isect<false>(st, gallop_ratio, nv, dv, par.p, par.len, out);
            }
            p = out;
        }
        __syncwarp();
        if (lane_id() == 0) {
            ops[id].p = p;
            ops[id].len = len;
        }
        __syncwarp();
        if (len == 0) return O.vdepth;
    }
    return kInvalid;
}

// Last depth: count list members that are candidates of u_L and not embedded.
// Returns the count; conf gets the depths of embedded vertices found.
__device__ uint64_t cache_last_count(const QPlan& P, uint32_t L, const uint32_t* lp, uint32_t len,
                                     const uint32_t (&slot_vid)[2], uint64_t& conf, Counters& C) {
    const uint32_t lane = lane_id();
    const uint32_t u = P.dep[L].u;
    uint32_t cnt = 0;
    for (uint32_t base = 0; base < len; base += 32) {
        const uint32_t i = base + lane;
        bool ok = false;
        if (i < len) ok = (__ldg(P.mask + lp[i]) >> u) & 1ull;
        cnt += __popc(__ballot_sync(kFull, ok));
    }
    C.bytes += 12ull * len;
    // embedded vertices among them: lane j tests the vertex of depth j
    conf = 0;
    for (uint32_t half = 0; half < 2; ++half) {
        const uint32_t j = half * 32 + lane;
        bool in = false;
        if (j < L) {
            const uint32_t v = half ? slot_vid[1] : slot_vid[0];
            if ((__ldg(P.mask + v) >> u) & 1ull) in = bsearch_global(lp, len, v);
        }
        const uint32_t b = __ballot_sync(kFull, in);
        conf |= (uint64_t)b << (32 * half);
        if (L <= 32) break;
    }
    return (uint64_t)(cnt - __popcll(conf));
}

__device__ void run_cache_task(const EnumArgs& A, const QPlan& P, uint64_t t, uint32_t* scr, OpState* ops, Stage& st,
                               Counters& C, Tally& T) {
    unsigned long long& local = T.local;
    const uint32_t lane = lane_id();
    const uint32_t n = P.n;
    const uint64_t ALL = ~0ull;
    const bool fs = A.failing_sets != 0;
    C.tasks++;
    // root (explore.h:1100-1122): v0 = candidates[u0][t]
    const uint32_t v0 = __ldg(P.dep[0].cand + t);
    C.bytes += 4;
    uint32_t slot_vid[2] = {kInvalid, kInvalid};
    uint32_t pos0 = 0, pos1 = 0, vm0 = 0, vm1 = 0, tot0 = 0, tot1 = 0, skip0 = 0, skip1 = 0;
    uint64_t fail0 = 0, fail1 = 0, ptr0 = 0, ptr1 = 0;
    if (lane == 0) slot_vid[0] = v0;
    C.nodes++;
#define vid0 slot_vid[0]
#define vid1 slot_vid[1]
    // ops of depth 0; an empty op means no extension of this root
    uint32_t conf = compute_ops(P, 0, v0, scr, ops, st, A.gallop_ratio, C);
    if (conf != kInvalid) return;
    auto enter = [&](uint32_t dd) {
        // candidates of depth dd come from its iteration op (already computed)
        const OpState it = ops[P.dep[dd].iter_op];
        SLOT_SET(ptr, dd, reinterpret_cast<uint64_t>(it.p));
        SLOT_SET(tot, dd, it.len);
        SLOT_SET(pos, dd, 0u);
        SLOT_SET(vm, dd, 0u);
        SLOT_SET(skip, dd, 0u);
    };
    auto fail_get = [&](uint32_t dd) -> uint64_t { return shfl64(dd < 32 ? fail0 : fail1, dd & 31); };
    auto fail_set = [&](uint32_t dd, uint64_t x) { SLOT_SET(fail, dd, x); };
    // PruneCheck(dd) (prune.h:119-141) with fail[dd] = f just set
    auto prune_check = [&](uint32_t dd, uint64_t f) {
        if (!((f >> dd) & 1ull)) {
            fail_set(dd - 1, f);
            SLOT_SET(pos, dd, SLOT_GET(tot, dd));
            SLOT_SET(vm, dd, 0u);
            C.pruned++;
        } else {
            fail_set(dd - 1, fail_get(dd - 1) | f);
        }
    };
    if (fs) fail_set(0, 0ull);
    uint32_t d = 1;
    if (n == 2) {
        uint64_t cf;
        const OpState it = ops[P.dep[1].iter_op];
        local += cache_last_count(P, 1, it.p, it.len, slot_vid, cf, C);
        return;
    }
    enter(1);
    uint32_t iter = 0;
    for (;;) {
        if ((++iter & 255u) == 0 && task_should_stop(A, T)) break;
        uint32_t vm = SLOT_GET(vm, d);
        if (vm == 0) {
            const uint32_t pos = SLOT_GET(pos, d);
            const uint32_t tot = SLOT_GET(tot, d);
            if (pos >= tot) {
                // end of depth d: all skipped -> fail[d-1] = anc[d] (explore.h:1068-1070)
                if (fs && SLOT_GET(skip, d) == tot) fail_set(d - 1, P.dep[d].anc);
                if (d == 1) break;
                --d;
                // PruneCheck(d) after returning from the child (explore.h:1063-1065)
                if (fs) prune_check(d, fail_get(d));
                continue;
            }
            // next batch: candidates of u_d (mask test); injectivity is checked per pick
            const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
            const uint32_t u = P.dep[d].u;
            const uint32_t i = pos + lane;
            bool isc = false;
            if (i < tot) isc = (__ldg(P.mask + lp[i]) >> u) & 1ull;
            const uint32_t cm = __ballot_sync(kFull, isc);
            const uint32_t nb = min(32u, tot - pos);
            C.bytes += 12ull * nb;
            SLOT_SET(skip, d, SLOT_GET(skip, d) + (nb - __popc(cm)));
            SLOT_SET(pos, d, pos + 32);
            SLOT_SET(vm, d, cm);
            continue;
        }
        const uint32_t b = __ffs(vm) - 1;
        SLOT_SET(vm, d, vm & (vm - 1));
        const uint32_t pos = SLOT_GET(pos, d) - 32 + b;
        const uint32_t* lp = reinterpret_cast<const uint32_t*>(shfl64(d < 32 ? ptr0 : ptr1, d & 31));
        const uint32_t v = lp[pos];
        // injectivity with the conflicting depth (explore.h:1014-1022)
        uint32_t cdep = kInvalid;
        for (uint32_t half = 0; half < 2; ++half) {
            const uint32_t bm = __ballot_sync(kFull, (half * 32 + lane) < d && (half ? vid1 : vid0) == v);
            if (bm && cdep == kInvalid) cdep = half * 32 + __ffs(bm) - 1;
            if (d <= 32) break;
        }
        if (cdep != kInvalid) {
            if (fs) {
                const uint64_t f = P.dep[d].anc | P.dep[cdep].anc;
                fail_set(d, f);
                fail_set(d - 1, fail_get(d - 1) | f);  // bit d is in anc[d]: never prunes
            }
            continue;
        }
        SLOT_SET(vid, d, v);
        C.nodes++;
        // ops of depth d for v
        conf = compute_ops(P, d, v, scr, ops, st, A.gallop_ratio, C);
        if (conf != kInvalid) {
            // NoCandidatesConflictCheckCache(0, d+1, conf) then PruneCheck(d)
            if (fs) {
                const uint64_t f = P.dep[conf].anc;
                fail_set(d, f);
                prune_check(d, f);
            }
            continue;
        }
        if (d + 2 == n) {
            // child is the last depth: count it in bulk and derive its failing set
            const OpState it = ops[P.dep[d + 1].iter_op];
            uint64_t cf = 0;
            const uint64_t k = cache_last_count(P, d + 1, it.p, it.len, slot_vid, cf, C);
            local += k;
            if (fs) {
                uint64_t f;
                if (k > 0) {
                    f = ALL;  // SuccessMatch (prune.h:143-146)
                } else {
                    f = P.dep[d + 1].anc;  // all skipped, or conflicts: anc[L] | anc[conflict depths]
                    uint64_t m = cf;
                    while (m) {
                        const int j = __ffsll((long long)m) - 1;
                        m &= m - 1;
                        f |= P.dep[j].anc;
                    }
                }
                fail_set(d, f);
                prune_check(d, f);
            }
            continue;
        }
        // descend: the child's entry resets its parent's accumulator (prune.h:162)
        ++d;
        if (fs) fail_set(d - 1, 0ull);
        enter(d);
    }
#undef vid0
#undef vid1
}

// ================================================================== kernel
// MINB = blocks of 256 threads the register allocation must leave room for
// on one SM (2: no register cap in practice; 3: at most 80 registers).
template <int MINB>
__global__ void __launch_bounds__(256, MINB) enum_kernel(EnumArgs A) {
    SMX_EXTERN_SMEM(smem);
    const uint32_t lane = lane_id();
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t wpb = blockDim.x >> 5;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    // shared layout: [wpb][stage buffer] [wpb][mbarrier] [wpb][max_ops op states]
    const size_t stage_bytes = ((size_t)(A.chunk + 8) * 4 + 15) & ~(size_t)15;
    Stage st;
    st.buf = reinterpret_cast<uint32_t*>(smem + stage_bytes * wib);
    st.mbar = reinterpret_cast<uint64_t*>(smem + stage_bytes * wpb) + wib;
    st.phase = 0;
    st.chunk = A.chunk;
    st.tma = A.use_tma != 0;
    st.failed = false;
    OpState* wops = reinterpret_cast<OpState*>(smem + stage_bytes * wpb + 16 * wpb) + (size_t)wib * A.max_ops;
#ifndef SMX_EMU
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(st.mbar)) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
#else
    st.tma = false;
#endif
    __syncwarp();
    uint32_t* scr = A.scratch + (size_t)gw * A.scratch_stride;
    // the bitmap starts empty; every task leaves it empty again
    uint32_t* bm = A.bitmap ? A.bitmap + (size_t)gw * A.bm_stride : nullptr;
    if (bm) {
        for (uint64_t i = lane; i < A.bm_stride; i += 32) bm[i] = 0;
        __syncwarp();
    }
    const uint64_t deadline = A.budget_ns && !A.per_query ? global_timer_ns() + A.budget_ns : 0;
    Counters C;
    Tally T;
    T.deadline = deadline;
    const uint64_t total = A.task_prefix[A.nq];
    uint32_t q = 0;
    uint64_t qlo = A.task_prefix[0], qhi = A.task_prefix[1];
    uint32_t grabs = 0;
    for (;;) {
        unsigned long long t0 = 0;
        if (lane == 0) t0 = atomicAdd(A.next_task, (unsigned long long)A.grab);
        t0 = __shfl_sync(kFull, t0, 0);
        if (t0 >= total) break;
        if ((grabs++ & 63u) == 0) check_global_stop(A, deadline);
        if (poll_abort(A)) break;
        const uint64_t t1 = min((uint64_t)t0 + A.grab, total);
        for (uint64_t t = t0; t < t1; ++t) {
            if (t < qlo || t >= qhi) {
                uint32_t lo = 0, hi = A.nq;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (A.task_prefix[mid] <= t) lo = mid; else hi = mid;
                }
                q = lo;
                qlo = A.task_prefix[q];
                qhi = A.task_prefix[q + 1];
            }
            if (query_stopped(A, q)) {
                // the query reached its limit: move the queue past its tasks
                // instead of draining them one grab at a time
                if (lane == 0) atomicMax(A.next_task, (unsigned long long)qhi);
                t = qhi - 1;
                continue;
            }
            const QPlan& P = A.plans[q];
            T.q = q;
            T.local = 0;
            if (A.per_query) {
                // the query's budget runs from its first task
                unsigned long long s0 = 0;
                if (lane == 0) {
                    const unsigned long long now = global_timer_ns();
                    s0 = atomicCAS(A.qstart + q, 0ull, now);
                    if (s0 == 0) s0 = now;
                }
                T.deadline = __shfl_sync(kFull, s0, 0) + A.budget_ns;
            }
            if (P.mode == SMX_EXPLORE_CANDIDATES) run_table_task(A, P, t - qlo, scr, bm, st, C, T);
            else run_cache_task(A, P, t - qlo, scr, wops, st, C, T);
            flush_tally(A, T);
            if (st.failed) break;
        }
        if (st.failed) {
            if (lane == 0) atomicCAS(A.status, 0, (int)SMX_CUDA_ERROR);
            break;
        }
    }
    if (lane == 0) {
        atomicAdd(A.stats + 0, C.isect);
        atomicAdd(A.stats + 1, C.nodes);
        atomicAdd(A.stats + 2, C.bytes);
        atomicAdd(A.stats + 3, C.tasks);
        atomicAdd(A.stats + 4, C.pruned);
    }
}

// ------------------------------------------------------------------ host side

struct HostPlanBuild {
    QPlan plan;
    std::vector<BnRef> bn;
    std::vector<OpInfo> op;
    std::vector<PartRef> part;
    uint64_t scratch_elems = 0;
    uint64_t bm_words = 0;  // last-depth bitmap words per warp (0: none)
};

int build_host_plan(const smx_graph* g, const HostQuery& q, const smx_cand* c, const uint32_t* order, int mode,
                    int lane_depth, bool use_bitmap, HostPlanBuild& hb) {
    const uint32_t n = q.n;
    std::memset(&hb.plan, 0, sizeof(QPlan));
    QPlan& P = hb.plan;
    P.n = n;
    P.qn = c->qn;
    P.mode = (uint32_t)mode;
    P.rank = c->d_rank;
    P.mask = c->d_mask;
    P.off = g->d_off;
    P.adj = g->d_adj;
    P.hub_id = g->d_hub_id;
    P.hub_bits = g->d_hub_bits;
    P.hub_words = g->hubs ? g->hub_words : 0;
    P.nroot = c->cnt[order[0]];
    std::vector<uint32_t> depth_of(n);
    for (uint32_t i = 0; i < n; ++i) depth_of[order[i]] = i;
    // backward neighbours ordered by position (GetPreviousNeb, common_ops.h:259-306)
    std::vector<std::vector<uint32_t>> bnd(n);
    for (uint32_t dd = 0; dd < n; ++dd) {
        const uint32_t u = order[dd];
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            const uint32_t p = depth_of[q.adj[e]];
            if (p < dd) bnd[dd].push_back(p);
        }
        std::sort(bnd[dd].begin(), bnd[dd].end());
        if (dd > 0 && bnd[dd].empty()) return fail(SMX_INVALID_ORDER, "order has a vertex without an earlier neighbour");
    }
    // DAF ancestors (prune.h:100-104)
    std::vector<uint64_t> anc(n, 0);
    for (uint32_t dd = 0; dd < n; ++dd) {
        anc[dd] = 1ull << dd;
        for (uint32_t p : bnd[dd]) anc[dd] |= anc[p];
    }
    uint64_t scr = 0;
    for (uint32_t dd = 0; dd < n; ++dd) {
        DepthInfo& D = P.dep[dd];
        D.u = order[dd];
        D.cand = c->cand_ptr(order[dd]);
        D.nbn = (uint32_t)bnd[dd].size();
        D.bn_begin = (uint32_t)hb.bn.size();
        D.anc = anc[dd];
        D.iter_op = kInvalid;
        for (uint32_t p : bnd[dd]) {
            BnRef r{};
            r.depth = p;
            if (mode == SMX_EXPLORE_CANDIDATES) {
                const int ti = c->tab_index[order[p]][order[dd]];
                if (ti < 0)
                    return fail(SMX_BAD_ARGUMENT,
                                "candidate-table enumeration needs the edge tables (smx_filter build_tables=1)");
                const DevTable& T = c->tables[ti];
                r.off = T.d_off;
                r.edge = T.d_edge;
                r.max_deg = T.max_deg;
            }
            hb.bn.push_back(r);
        }
        D.list_off = kInvalid;
    }
    P.leaf_inb = 0;
    P.leaf_bm = 0;
    P.leaf_gdepth = kInvalid;
    P.tail_depth = kInvalid;
    P.tail_bms = 0;
    P.leaf_g_bn = P.leaf_g_off = P.leaf_gp_off = kInvalid;
    if (mode == SMX_EXPLORE_CANDIDATES) {
        // partial-intersection buffers: word 0 the length, elements from word 4
        auto alloc = [&](uint64_t cap) {
            const uint64_t off = scr;
            scr += (4 + cap + 3) & ~3ull;
            return (uint32_t)off;
        };
        std::vector<std::vector<PartRef>> parts_at(n);
        for (uint32_t t = 2; t < n; ++t) {
            DepthInfo& D = P.dep[t];
            const uint32_t k = D.nbn;
            const bool leaf = t + 1 == n;
            const bool inb = leaf && bnd[t][k - 1] + 2 == n;
            // the last depth's row of depth n-2 is counted per lane, not materialised
            const uint32_t jmax = inb ? k - 1 : k;
            uint64_t cap = hb.bn[D.bn_begin].max_deg;
            uint32_t prev = kInvalid;
            for (uint32_t j = 2; j <= jmax; ++j) {
                const uint32_t e = D.bn_begin + j - 1;
                cap = std::min<uint64_t>(cap, hb.bn[e].max_deg);
                const uint32_t off = alloc(cap);
                parts_at[hb.bn[e].depth].push_back(PartRef{D.bn_begin, e, prev, off, t});
                prev = off;
            }
            if (!leaf) {
                D.list_off = k >= 2 ? prev : kInvalid;
            } else {
                P.leaf_inb = inb ? 1u : 0u;
                if (jmax >= 2) P.leaf_g_off = prev;
                else if (jmax == 1) P.leaf_g_bn = D.bn_begin;
                if (inb && jmax >= 1) {
                    P.leaf_gp_off = alloc(cap);
                    if (use_bitmap) {
                        P.leaf_bm = 1;
                        hb.bm_words = (uint64_t)c->cnt[order[t]] / 32 + 1;
                        // factored tail: S and G depend only on depths <= a; B is
                        // recomputed per depth-a node, so it pays only with at
                        // least three depths between a and n-2
                        uint32_t a = 0;
                        for (uint32_t p : bnd[n - 2]) a = std::max(a, p);
                        for (uint32_t j = 0; j < jmax; ++j) a = std::max(a, bnd[t][j]);
                        const int ti = c->tab_index[order[t]][order[n - 2]];
                        uint32_t ag = 0;
                        for (uint32_t j = 0; j < jmax; ++j) ag = std::max(ag, bnd[t][j]);
                        if (ag + 4 <= n) P.leaf_gdepth = ag;
                        if (n >= 5 && a + 6 <= n && ti >= 0) {
                            P.leaf_gdepth = kInvalid;  // the tail keeps its own marks
                            P.tail_depth = a;
                            P.tail_bms = (uint32_t)hb.bm_words;
                            hb.bm_words += (uint64_t)c->cnt[order[n - 2]] / 32 + 1;
                            const DevTable& T = c->tables[ti];
                            P.tail_rev.off = T.d_off;
                            P.tail_rev.edge = T.d_edge;
                            P.tail_rev.depth = t;
                            P.tail_rev.max_deg = T.max_deg;
                        }
                    }
                }
            }
        }
        for (uint32_t dd = 0; dd < n; ++dd) {
            P.dep[dd].part_begin = (uint32_t)hb.part.size();
            P.dep[dd].npart = (uint32_t)parts_at[dd].size();
            hb.part.insert(hb.part.end(), parts_at[dd].begin(), parts_at[dd].end());
        }
    }
    if (mode == SMX_EXPLORE_CANDIDATES) {
        P.ntasks = n >= 2 ? c->tables[c->tab_index[order[0]][order[1]]].e_cnt : 0;
        // lane depth: given by the caller, or (lane_depth < 0) the shallowest
        // depth T >= 2 below which (up to n-2) every candidate list is an
        // intersection of two or more rows.  A lane walks its lists serially,
        // so this pays only when those intersections stay short; rows of hub
        // vertices make it far slower than the warp-wide search, hence off
        // by default.
        uint32_t T = n >= 2 ? n - 2 : 0;
        if (lane_depth < 0) {
            for (uint32_t t = 2; t + 2 < n; ++t) {
                bool all = true;
                for (uint32_t e = t + 1; e + 2 <= n; ++e) all &= bnd[e].size() >= 2;
                if (all) {
                    T = t;
                    break;
                }
            }
        } else if (lane_depth >= 2) {
            T = std::min<uint32_t>((uint32_t)lane_depth, n >= 2 ? n - 2 : 0);
        }
        P.lane_depth = T;
    } else {
        Plan plan;
        if (!build_plan(q, order, plan)) return fail(SMX_INVALID_ORDER, "order has a vertex without an earlier neighbour");
        P.nops = (uint32_t)plan.ops.size();
        // op ids renumbered so the ops of each depth are contiguous
        std::vector<uint32_t> newid(plan.ops.size(), kInvalid);
        uint32_t next = 0;
        for (uint32_t dd = 0; dd < n; ++dd)
            for (uint32_t id : plan.ops_at[dd]) newid[id] = next++;
        hb.op.assign(plan.ops.size(), OpInfo{});
        for (uint32_t id = 0; id < plan.ops.size(); ++id) {
            const PlanOp& po = plan.ops[id];
            OpInfo& oi = hb.op[newid[id]];
            oi.parent = po.parent == kInvalid ? kInvalid : newid[po.parent];
            oi.vdepth = po.vdepth;
            oi.scr_off = 0;
            if (po.parent != kInvalid) {
                oi.scr_off = (uint32_t)scr;
                scr += ((uint64_t)g->h.max_deg + 8 + 3) & ~3ull;
            }
        }
        next = 0;
        for (uint32_t dd = 0; dd < n; ++dd) {
            P.dep[dd].ops_begin = next;
            P.dep[dd].nops = (uint32_t)plan.ops_at[dd].size();
            next += P.dep[dd].nops;
            P.dep[dd].iter_op = dd ? newid[plan.iter_op[dd]] : kInvalid;
        }
        P.ntasks = c->cnt[order[0]];
    }
    hb.scratch_elems = scr + 8;
    return SMX_OK;
}

}  // namespace

int device_enumerate(smx_graph* g, const std::vector<const HostQuery*>& qs, const std::vector<const smx_cand*>& cs,
                     const std::vector<const uint32_t*>& orders, const smx_enum_opts& o,
                     const std::vector<uint64_t>& limits, volatile uint32_t* stop, uint64_t* counts, smx_stats* st,
                     bool use_graph, int32_t* qstatus) {
    SMX_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const uint32_t nq = (uint32_t)qs.size();
    if (nq == 0) return SMX_OK;
    const int mode = o.explore;
    std::vector<HostPlanBuild> hb(nq);
    std::vector<uint64_t> prefix(nq + 1, 0);
    uint64_t scratch_elems = 8;
    uint64_t bm_words = 0;
    uint32_t max_ops = 1;
    for (uint32_t i = 0; i < nq; ++i) {
        int rc = build_host_plan(g, *qs[i], cs[i], orders[i], mode, o.lane_depth, o.bitmap_min >= 0, hb[i]);
        if (rc != SMX_OK) return rc;
        scratch_elems = std::max(scratch_elems, hb[i].scratch_elems);
        bm_words = std::max(bm_words, hb[i].bm_words);
        max_ops = std::max(max_ops, hb[i].plan.nops);
        prefix[i + 1] = prefix[i] + hb[i].plan.ntasks;
    }
    // device copies of plans; bn / op arrays in one pool
    size_t pool_bytes = 64;
    for (auto& h : hb)
        pool_bytes += h.bn.size() * sizeof(BnRef) + h.op.size() * sizeof(OpInfo) + h.part.size() * sizeof(PartRef) + 48;
    std::vector<char> pool(pool_bytes, 0);
    std::vector<QPlan> plans(nq);
    char* d_pool = nullptr;
    QPlan* d_plans = nullptr;
    SMX_CUDA_TRY(cudaMallocAsync(&d_pool, pool_bytes, s));
    SMX_CUDA_TRY(cudaMallocAsync(&d_plans, nq * sizeof(QPlan), s));
    size_t at = 0;
    for (uint32_t i = 0; i < nq; ++i) {
        plans[i] = hb[i].plan;
        at = (at + 15) & ~(size_t)15;
        if (!hb[i].bn.empty()) std::memcpy(pool.data() + at, hb[i].bn.data(), hb[i].bn.size() * sizeof(BnRef));
        plans[i].bn = reinterpret_cast<const BnRef*>(d_pool + at);
        at += hb[i].bn.size() * sizeof(BnRef);
        at = (at + 15) & ~(size_t)15;
        if (!hb[i].op.empty()) std::memcpy(pool.data() + at, hb[i].op.data(), hb[i].op.size() * sizeof(OpInfo));
        plans[i].op = reinterpret_cast<const OpInfo*>(d_pool + at);
        at += hb[i].op.size() * sizeof(OpInfo);
        at = (at + 15) & ~(size_t)15;
        if (!hb[i].part.empty())
            std::memcpy(pool.data() + at, hb[i].part.data(), hb[i].part.size() * sizeof(PartRef));
        plans[i].part = reinterpret_cast<const PartRef*>(d_pool + at);
        at += hb[i].part.size() * sizeof(PartRef);
    }
    SMX_CUDA_TRY(cudaMemcpyAsync(d_pool, pool.data(), pool_bytes, cudaMemcpyHostToDevice, s));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_plans, plans.data(), nq * sizeof(QPlan), cudaMemcpyHostToDevice, s));
    // launch shape
    const uint32_t wpb = o.warps_per_block > 0 ? std::min<uint32_t>((uint32_t)o.warps_per_block, 8u) : 8u;
    const uint32_t chunk = o.stage_chunk > 0 ? ((uint32_t)o.stage_chunk + 3) & ~3u : 1024u;
    const size_t stage_bytes = ((size_t)(chunk + 8) * 4 + 15) & ~(size_t)15;
    const size_t smem = stage_bytes * wpb + 16 * wpb + (size_t)max_ops * sizeof(OpState) * wpb;
    if (smem > 227 * 1024)
        return fail(SMX_TOO_LARGE, "shared memory per block above 227 KB: lower stage_chunk or warps_per_block");
    // blocks_per_sm >= 3 selects the register-capped build of the kernel
    const bool reg_capped = o.blocks_per_sm >= 3;
    auto kern = reg_capped ? enum_kernel<3> : enum_kernel<2>;
    SMX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int bps = 0;
    SMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, (int)(wpb * 32), smem));
    if (o.blocks_per_sm > 0) bps = std::min(bps, o.blocks_per_sm);
    if (bps < 1) return fail(SMX_TOO_LARGE, "enumeration kernel does not fit on an SM with this shared-memory size");
    uint32_t blocks = (uint32_t)(g->num_sms * bps);
    {
        // fewer resident warps when their scratch would not fit in free memory
        size_t free_b = 0, total_b = 0;
        SMX_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
        const double budget = 0.8 * (double)(free_b + g->scratch_bytes);
        const double per_block = (double)wpb * (double)(scratch_elems + bm_words) * 4.0;
        if (per_block * blocks > budget) {
            const uint32_t fit = (uint32_t)(budget / per_block);
            if (fit < 1) return fail(SMX_TOO_LARGE, "enumeration scratch for one block exceeds device memory");
            blocks = fit;
        }
    }
    const uint64_t nwarps = (uint64_t)blocks * wpb;
    // control block (explicit offsets) + per-warp scratch
    const size_t o_next = 0, o_status = 8, o_stats = 16;           // stats: 5 x u64
    const size_t o_qcount = 64;
    const size_t o_qlimit = o_qcount + (size_t)nq * 8;
    const size_t o_prefix = o_qlimit + (size_t)nq * 8;
    const size_t o_qstop = o_prefix + (size_t)(nq + 1) * 8;
    const size_t o_qstart = (o_qstop + (size_t)nq * 4 + 7) & ~(size_t)7;
    const size_t o_scr = (o_qstart + (size_t)nq * 8 + 255) & ~(size_t)255;
    const size_t o_bm = (o_scr + nwarps * scratch_elems * 4 + 255) & ~(size_t)255;
    const size_t total_bytes = o_bm + nwarps * bm_words * 4 + 64;
    int rc = ensure_scratch(g, total_bytes);
    if (rc != SMX_OK) return rc;
    char* base = static_cast<char*>(g->d_scratch);
    unsigned long long* d_next = reinterpret_cast<unsigned long long*>(base + o_next);
    int* d_status = reinterpret_cast<int*>(base + o_status);
    unsigned long long* d_stats = reinterpret_cast<unsigned long long*>(base + o_stats);
    unsigned long long* d_qcount = reinterpret_cast<unsigned long long*>(base + o_qcount);
    uint64_t* d_qlimit = reinterpret_cast<uint64_t*>(base + o_qlimit);
    uint64_t* d_prefix = reinterpret_cast<uint64_t*>(base + o_prefix);
    uint32_t* d_qstop = reinterpret_cast<uint32_t*>(base + o_qstop);
    unsigned long long* d_qstart = reinterpret_cast<unsigned long long*>(base + o_qstart);
    uint32_t* d_scr = reinterpret_cast<uint32_t*>(base + o_scr);
    SMX_CUDA_TRY(cudaMemcpyAsync(d_qlimit, limits.data(), nq * 8, cudaMemcpyHostToDevice, s));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_prefix, prefix.data(), (nq + 1) * 8, cudaMemcpyHostToDevice, s));
    // host-visible stop word: the device polls a mapped pointer
    const volatile uint32_t* d_host_stop = nullptr;
    if (stop) {
        void* dp = nullptr;
        if (cudaHostGetDevicePointer(&dp, (void*)stop, 0) == cudaSuccess) d_host_stop = static_cast<const volatile uint32_t*>(dp);
        else cudaGetLastError();
    }
    EnumArgs A;
    std::memset(&A, 0, sizeof(A));
    A.plans = d_plans;
    A.task_prefix = d_prefix;
    A.next_task = d_next;
    A.qcount = d_qcount;
    A.qstop = d_qstop;
    A.qstart = d_qstart;
    A.per_query = (o.budget_per_query && o.time_budget_ms > 0) ? 1u : 0u;
    A.qlimit = d_qlimit;
    A.scratch = d_scr;
    A.stats = d_stats;
    A.status = d_status;
    A.host_stop = d_host_stop;
    A.scratch_stride = scratch_elems;
    A.bitmap = bm_words ? reinterpret_cast<uint32_t*>(base + o_bm) : nullptr;
    A.bm_stride = bm_words;
    A.bitmap_min = o.bitmap_min > 0 ? (uint32_t)o.bitmap_min : 32u;
    A.budget_ns = o.time_budget_ms > 0 ? (uint64_t)(o.time_budget_ms * 1e6) : 0;
    A.nq = nq;
    A.max_ops = max_ops;
    A.grab = o.task_grab > 0 ? (uint32_t)o.task_grab : 4u;
    // many light tasks: larger grabs, so the queue's one counter is not the
    // bottleneck (each warp still takes >= 256 grabs on average)
    A.grab = (uint32_t)std::max<uint64_t>(A.grab, std::min<uint64_t>(prefix[nq] / (nwarps * 256), 1024));
    A.chunk = chunk;
    A.gallop_ratio = o.gallop_ratio > 0 ? (uint32_t)o.gallop_ratio : 16u;
    A.use_tma = o.use_tma ? 1u : 0u;
    A.failing_sets = o.failing_sets ? 1u : 0u;
    cudaEvent_t e0, e1;
    SMX_CUDA_TRY(cudaEventCreate(&e0));
    SMX_CUDA_TRY(cudaEventCreate(&e1));
    auto record = [&](cudaStream_t ss) -> cudaError_t {
        cudaError_t e;
        if ((e = cudaMemsetAsync(base, 0, 64, ss)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(d_qcount, 0, nq * 8, ss)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(d_qstop, 0, nq * 4, ss)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(d_qstart, 0, nq * 8, ss)) != cudaSuccess) return e;
        SMX_LAUNCH(kern, blocks, wpb * 32, smem, ss, A);
        return cudaGetLastError();
    };
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    if (use_graph) {
        SMX_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = record(s);
        cudaError_t ee = cudaStreamEndCapture(s, &graph);
        if (ce != cudaSuccess) return fail(SMX_CUDA_ERROR, std::string("capture: ") + cudaGetErrorString(ce));
        if (ee != cudaSuccess) return fail(SMX_CUDA_ERROR, std::string("end capture: ") + cudaGetErrorString(ee));
        SMX_CUDA_TRY(cudaGraphInstantiate(&exec, graph, 0));
        SMX_CUDA_TRY(cudaEventRecord(e0, s));
        SMX_CUDA_TRY(cudaGraphLaunch(exec, s));
        SMX_CUDA_TRY(cudaEventRecord(e1, s));
    } else {
        SMX_CUDA_TRY(cudaEventRecord(e0, s));
        cudaError_t ce = record(s);
        if (ce != cudaSuccess) return fail(SMX_CUDA_ERROR, std::string("enumeration launch: ") + cudaGetErrorString(ce));
        SMX_CUDA_TRY(cudaEventRecord(e1, s));
    }
    SMX_CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    SMX_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::vector<unsigned long long> qc(nq);
    std::vector<uint32_t> qs_stop(nq);
    unsigned long long stats[5];
    int status = 0;
    SMX_CUDA_TRY(cudaMemcpy(qc.data(), d_qcount, nq * 8, cudaMemcpyDeviceToHost));
    SMX_CUDA_TRY(cudaMemcpy(qs_stop.data(), d_qstop, nq * 4, cudaMemcpyDeviceToHost));
    SMX_CUDA_TRY(cudaMemcpy(stats, d_stats, sizeof(stats), cudaMemcpyDeviceToHost));
    SMX_CUDA_TRY(cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost));
    SMX_CUDA_TRY(cudaFreeAsync(d_pool, s));
    SMX_CUDA_TRY(cudaFreeAsync(d_plans, s));
    SMX_CUDA_TRY(cudaStreamSynchronize(s));
    uint64_t raw = 0, capped = 0;
    bool reached = false;
    for (uint32_t i = 0; i < nq; ++i) {
        raw += qc[i];
        uint64_t c = qc[i];
        if (limits[i] && c >= limits[i]) {
            c = limits[i];
            reached = true;
        }
        capped += c;
        if (counts) counts[i] = c;
        if (qstatus) qstatus[i] = qs_stop[i] == 2 ? SMX_TIMEOUT : SMX_OK;
        if (qs_stop[i] == 2 && status == 0) status = SMX_TIMEOUT;
    }
    if (st) {
        st->count = capped;
        st->raw_count = raw;
        st->intersections = stats[0];
        st->nodes = stats[1];
        st->bytes = stats[2];
        st->tasks = stats[3];
        st->pruned = stats[4];
        st->kernel_ms = ms;
        st->limit_reached = reached ? 1 : 0;
        st->status = status;
    }
    if (status == SMX_CUDA_ERROR) return fail(SMX_CUDA_ERROR, "bulk copy wait did not complete; enumeration aborted");
    if (status == SMX_TIMEOUT) set_error("time budget exhausted; the count is partial");
    if (status == SMX_STOPPED) set_error("stopped by the caller; the count is partial");
    return status;
}

int ensure_scratch(smx_graph* g, size_t bytes) {
    if (g->scratch_bytes >= bytes) return SMX_OK;
    // grow by at least half again, so a run of slightly larger queries does
    // not reallocate every time; fall back to the exact size if that fails
    size_t want = std::max(bytes, g->scratch_bytes + g->scratch_bytes / 2);
    if (g->d_scratch) SMX_CUDA_TRY(cudaFree(g->d_scratch));
    g->d_scratch = nullptr;
    g->scratch_bytes = 0;
    if (cudaMalloc(&g->d_scratch, want) != cudaSuccess) {
        cudaGetLastError();
        want = bytes;
        SMX_CUDA_TRY(cudaMalloc(&g->d_scratch, want));
    }
    g->scratch_bytes = want;
    return SMX_OK;
}

// ------------------------------------------------------------------ enumeration without allocation
// smx_enumerate allocates device memory on every call (plans, and scratch
// that grows with the query).  Some callers cannot allow that: a host
// framework whose own caching allocator has reserved the device memory, code
// that must not take cudaMalloc's implicit device synchronisation or its
// failure when memory is exhausted, or a process that has to keep its device
// footprint fixed after start-up.  For them smx_enumerate_noalloc runs the
// same kernel with all of its working memory (control block, plans, per-warp
// scratch and bitmaps) in the file-scope array below, reserved when the
// library is loaded on a GPU and held until the process exits.  The array is
// shared by every call on that device and keeps the last call's contents; the
// parts that must start at zero are cleared by each call.

static __device__ __align__(256) unsigned char g_noalloc_scratch[SMX_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;                       // calls never overlap on the GPU
void* g_noalloc_ptr[kNoAllocMaxDevices] = {};  // device address of the array, per device

// Once per device, with that device current: the array's device address.
// (Host code only sees a host-side stand-in under the array's name.)
int noalloc_setup(int device, unsigned char** out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(SMX_BAD_ARGUMENT, "device index out of range");
    if (!g_noalloc_ptr[device]) {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(SMX_CUDA_ERROR, std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                                            cudaGetErrorString(e));
        g_noalloc_ptr[device] = ptr;
    }
    *out = static_cast<unsigned char*>(g_noalloc_ptr[device]);
    return SMX_OK;
}
}  // namespace

int device_enumerate_noalloc(smx_graph* g, const HostQuery& q, const smx_cand* c, const uint32_t* order,
                             const smx_enum_opts& o, uint64_t limit, volatile uint32_t* stop, smx_stats* st) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    SMX_CUDA_TRY(cudaSetDevice(g->device));
    unsigned char* base = nullptr;
    int rc = noalloc_setup(g->device, &base);
    if (rc != SMX_OK) return rc;
    cudaStream_t s = g->stream;
    HostPlanBuild hb;
    rc = build_host_plan(g, q, c, order, o.explore, o.lane_depth, o.bitmap_min >= 0, hb);
    if (rc != SMX_OK) return rc;
    const uint64_t scratch_elems = std::max<uint64_t>(8, hb.scratch_elems);
    const uint64_t bm_words = hb.bm_words;
    const uint32_t max_ops = std::max<uint32_t>(1, hb.plan.nops);
    // layout of the array: control block | plan | bn / op / part pool | per-warp scratch | bitmaps
    const size_t o_next = 0, o_status = 8, o_stats = 16, o_qcount = 64, o_qlimit = 72, o_prefix = 80, o_qstop = 96;
    const size_t o_plan = 256;
    const size_t o_pool = (o_plan + sizeof(QPlan) + 255) & ~(size_t)255;
    size_t at = o_pool;
    auto place = [&](size_t bytes) {
        at = (at + 15) & ~(size_t)15;
        const size_t off = at;
        at += bytes;
        return off;
    };
    const size_t o_bn = place(hb.bn.size() * sizeof(BnRef));
    const size_t o_op = place(hb.op.size() * sizeof(OpInfo));
    const size_t o_part = place(hb.part.size() * sizeof(PartRef));
    const size_t o_scr = (at + 255) & ~(size_t)255;
    // launch shape as smx_enumerate, with no more warps than the array holds
    const uint32_t wpb = o.warps_per_block > 0 ? std::min<uint32_t>((uint32_t)o.warps_per_block, 8u) : 8u;
    const uint32_t chunk = o.stage_chunk > 0 ? ((uint32_t)o.stage_chunk + 3) & ~3u : 1024u;
    const size_t stage_bytes = ((size_t)(chunk + 8) * 4 + 15) & ~(size_t)15;
    const size_t smem = stage_bytes * wpb + 16 * wpb + (size_t)max_ops * sizeof(OpState) * wpb;
    if (smem > 227 * 1024)
        return fail(SMX_TOO_LARGE, "shared memory per block above 227 KB: lower stage_chunk or warps_per_block");
    auto kern = o.blocks_per_sm >= 3 ? enum_kernel<3> : enum_kernel<2>;
    SMX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int bps = 0;
    SMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, (int)(wpb * 32), smem));
    if (o.blocks_per_sm > 0) bps = std::min(bps, o.blocks_per_sm);
    if (bps < 1) return fail(SMX_TOO_LARGE, "enumeration kernel does not fit on an SM with this shared-memory size");
    const size_t per_warp = ((size_t)(scratch_elems + bm_words)) * 4;
    const size_t per_block = per_warp * wpb;
    const size_t cap = (size_t)SMX_NOALLOC_SCRATCH_BYTES;
    if (o_scr + per_block + 512 > cap)
        return fail(SMX_TOO_LARGE, "the query needs " + std::to_string(o_scr + per_block + 512) +
                                       " bytes of working memory for one block of " + std::to_string(wpb) +
                                       " warps; smx_enumerate_noalloc has " + std::to_string(cap) +
                                       " (SMX_NOALLOC_SCRATCH_BYTES): use smx_enumerate or fewer warps_per_block");
    const uint32_t blocks =
        (uint32_t)std::min<size_t>((size_t)g->num_sms * bps, (cap - o_scr - 512) / per_block);
    const uint64_t nwarps = (uint64_t)blocks * wpb;
    const size_t o_bm = (o_scr + nwarps * scratch_elems * 4 + 255) & ~(size_t)255;
    // control block (zeroed), limit, task prefix, plan and pool in one host image
    std::vector<unsigned char> img(o_scr, 0);
    std::memcpy(img.data() + o_qlimit, &limit, 8);
    const uint64_t prefix[2] = {0, hb.plan.ntasks};
    std::memcpy(img.data() + o_prefix, prefix, sizeof(prefix));
    QPlan plan = hb.plan;
    plan.bn = reinterpret_cast<const BnRef*>(base + o_bn);
    plan.op = reinterpret_cast<const OpInfo*>(base + o_op);
    plan.part = reinterpret_cast<const PartRef*>(base + o_part);
    std::memcpy(img.data() + o_plan, &plan, sizeof(QPlan));
    if (!hb.bn.empty()) std::memcpy(img.data() + o_bn, hb.bn.data(), hb.bn.size() * sizeof(BnRef));
    if (!hb.op.empty()) std::memcpy(img.data() + o_op, hb.op.data(), hb.op.size() * sizeof(OpInfo));
    if (!hb.part.empty()) std::memcpy(img.data() + o_part, hb.part.data(), hb.part.size() * sizeof(PartRef));
    SMX_CUDA_TRY(cudaMemcpyAsync(base, img.data(), img.size(), cudaMemcpyHostToDevice, s));
    const volatile uint32_t* d_host_stop = nullptr;
    if (stop) {
        void* dp = nullptr;
        if (cudaHostGetDevicePointer(&dp, (void*)stop, 0) == cudaSuccess) d_host_stop = static_cast<const volatile uint32_t*>(dp);
        else cudaGetLastError();
    }
    EnumArgs A;
    std::memset(&A, 0, sizeof(A));
    A.plans = reinterpret_cast<const QPlan*>(base + o_plan);
    A.task_prefix = reinterpret_cast<const uint64_t*>(base + o_prefix);
    A.next_task = reinterpret_cast<unsigned long long*>(base + o_next);
    A.qcount = reinterpret_cast<unsigned long long*>(base + o_qcount);
    A.qstop = reinterpret_cast<uint32_t*>(base + o_qstop);
    A.qlimit = reinterpret_cast<const uint64_t*>(base + o_qlimit);
    A.scratch = reinterpret_cast<uint32_t*>(base + o_scr);
    A.stats = reinterpret_cast<unsigned long long*>(base + o_stats);
    A.status = reinterpret_cast<int*>(base + o_status);
    A.host_stop = d_host_stop;
    A.scratch_stride = scratch_elems;
    A.bitmap = bm_words ? reinterpret_cast<uint32_t*>(base + o_bm) : nullptr;
    A.bm_stride = bm_words;
    A.bitmap_min = o.bitmap_min > 0 ? (uint32_t)o.bitmap_min : 32u;
    A.budget_ns = o.time_budget_ms > 0 ? (uint64_t)(o.time_budget_ms * 1e6) : 0;
    A.nq = 1;
    A.max_ops = max_ops;
    A.grab = o.task_grab > 0 ? (uint32_t)o.task_grab : 4u;
    A.chunk = chunk;
    A.gallop_ratio = o.gallop_ratio > 0 ? (uint32_t)o.gallop_ratio : 16u;
    A.use_tma = o.use_tma ? 1u : 0u;
    A.failing_sets = o.failing_sets ? 1u : 0u;
    const auto t0 = std::chrono::steady_clock::now();
    SMX_LAUNCH(kern, blocks, wpb * 32, smem, s, A);
    SMX_CUDA_TRY(cudaGetLastError());
    unsigned char back[128];
    SMX_CUDA_TRY(cudaMemcpyAsync(back, base, sizeof(back), cudaMemcpyDeviceToHost, s));
    SMX_CUDA_TRY(cudaStreamSynchronize(s));
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    unsigned long long qc = 0, stats[5];
    int status = 0;
    std::memcpy(&qc, back + o_qcount, 8);
    std::memcpy(stats, back + o_stats, sizeof(stats));
    std::memcpy(&status, back + o_status, sizeof(int));
    const bool reached = limit && qc >= limit;
    if (st) {
        st->count = reached ? limit : qc;
        st->raw_count = qc;
        st->intersections = stats[0];
        st->nodes = stats[1];
        st->bytes = stats[2];
        st->tasks = stats[3];
        st->pruned = stats[4];
        st->kernel_ms = ms;
        st->limit_reached = reached ? 1 : 0;
        st->status = status;
    }
    if (status == SMX_CUDA_ERROR) return fail(SMX_CUDA_ERROR, "bulk copy wait did not complete; enumeration aborted");
    if (status == SMX_TIMEOUT) set_error("time budget exhausted; the count is partial");
    if (status == SMX_STOPPED) set_error("stopped by the caller; the count is partial");
    return status;
}

}  // namespace smx
