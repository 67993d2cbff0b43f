// Device filtering: NLF candidate masks, GQL exact-twig refinement, candidate
// compaction with a rank directory, and the candidate-edge tables.
//
// Data layout in HBM (per data graph, built once):
//   d_off  uint64[n+1], d_adj uint32[2m] (rows ascending), d_lab uint32[n]
//   d_hist uint8[n * stride]  neighbour-label counts saturating at 255, only
//          for labelled graphs with at most 64 labels (query degrees are at
//          most 63, so saturation never changes a comparison).
// Per query (smx_cand):
//   d_mask uint64[n]      bit u set iff v is a candidate of query vertex u
//   d_rank uint2[n/32][q] per 32-vertex block: {bit row of u, candidates of u
//                         in earlier blocks}; rank of v in C(u) in one load
//   d_cand uint32[]       C(u) for every u, ascending, concatenated
//   tables                E[a][b]: uint32 offsets over C(a) and candidate
//                         indices into C(b) (edge_v is C(b)[edge], rebuilt on
//                         export), ascending rows, as buildTables (table.h:7-139)
#include <algorithm>
#include <numeric>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "smx_internal.h"

namespace smx {

namespace {

constexpr uint32_t kMaxNlf = kMaxQ * (kMaxQ - 1);

struct QInfo {
    uint32_t n;
    uint32_t data_labels;
    uint32_t hist_stride;
    uint32_t pad;
    uint32_t lab[kMaxQ];
    uint32_t deg[kMaxQ];
    uint32_t nlf_off[kMaxQ + 1];
    uint32_t nlf_lab[kMaxNlf];
    uint32_t nlf_cnt[kMaxNlf];
};

// ------------------------------------------------------------------ histogram
__global__ void hist_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                            const uint32_t* __restrict__ lab, uint32_t n, uint32_t stride, uint8_t* __restrict__ hist) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint8_t* h = hist + (size_t)v * stride;
        for (uint64_t e = off[v]; e < off[v + 1]; ++e) {
            uint32_t l = lab[adj[e]];
            if (l < stride && h[l] < 255) h[l]++;
        }
    }
}

// ------------------------------------------------------------------ NLF
// NLFByVertex (filter.h:24-58) for every query vertex at once, one thread per
// data vertex: bit u of mask[v] is set iff L(v) = L(u), deg(v) >= deg(u) and
// for every label l around u, v has at least as many l-labelled neighbours.
__global__ void nlf_mask_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj,
                                const uint32_t* __restrict__ lab, const uint8_t* __restrict__ hist, uint32_t n,
                                const QInfo* __restrict__ qi, uint64_t* __restrict__ mask) {
    SMX_SHARED_ARRAY(uint32_t, s_lab, kMaxQ);
    SMX_SHARED_ARRAY(uint32_t, s_deg, kMaxQ);
    SMX_SHARED_ARRAY(uint32_t, s_noff, kMaxQ + 1);
    const uint32_t qn = qi->n;
    for (uint32_t i = threadIdx.x; i < qn; i += blockDim.x) {
        s_lab[i] = qi->lab[i];
        s_deg[i] = qi->deg[i];
    }
    for (uint32_t i = threadIdx.x; i <= qn; i += blockDim.x) s_noff[i] = qi->nlf_off[i];
    __syncthreads();
    const uint32_t L = qi->data_labels, stride = qi->hist_stride;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t lv = lab[v];
        const uint64_t o0 = off[v], o1 = off[v + 1];
        const uint32_t dv = (uint32_t)(o1 - o0);
        uint64_t m = 0;
        for (uint32_t u = 0; u < qn; ++u) {
            if (s_lab[u] != lv || dv < s_deg[u]) continue;
            bool ok = true;
            for (uint32_t p = s_noff[u]; p < s_noff[u + 1] && ok; ++p) {
                const uint32_t l = qi->nlf_lab[p], c = qi->nlf_cnt[p];
                if (l >= L) {
                    ok = false;
                    break;
                }
                uint32_t have;
                if (L == 1) {
                    have = dv;
                } else if (hist) {
                    have = hist[(size_t)v * stride + l];
                } else {
                    have = 0;
                    for (uint64_t e = o0; e < o1 && have < c; ++e) have += (lab[adj[e]] == l);
                }
                ok = have >= c;
            }
            if (ok) m |= 1ull << u;
        }
        mask[v] = m;
    }
}

// ------------------------------------------------------------------ compaction
// One warp per 32-vertex block: bit rows of every query vertex into the rank
// directory, block counts into cnt[u][blk + 1] for the segmented scan.
__global__ void rank_bits_kernel(const uint64_t* __restrict__ mask, uint32_t n, uint32_t qn, uint32_t nblk,
                                 uint2* __restrict__ rank, uint32_t* __restrict__ cnt) {
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; blk < nblk; blk += warps) {
        const uint32_t v = blk * 32 + lane;
        const uint64_t m = v < n ? mask[v] : 0ull;
        uint32_t b_lo = 0, b_hi = 0;
        for (uint32_t u = 0; u < qn; ++u) {
            uint32_t b = __ballot_sync(kFull, (m >> u) & 1ull);
            if (lane == (u & 31u)) {
                if (u < 32) b_lo = b; else b_hi = b;
            }
        }
        if (lane < qn) {
            rank[(size_t)blk * qn + lane].x = b_lo;
            cnt[(size_t)lane * (nblk + 1) + blk + 1] = __popc(b_lo);
            if (blk == 0) cnt[(size_t)lane * (nblk + 1)] = 0;
        }
        if (lane + 32 < qn) {
            rank[(size_t)blk * qn + lane + 32].x = b_hi;
            cnt[(size_t)(lane + 32) * (nblk + 1) + blk + 1] = __popc(b_hi);
            if (blk == 0) cnt[(size_t)(lane + 32) * (nblk + 1)] = 0;
        }
    }
}

// After the scan cnt[u][blk] is the number of candidates of u in blocks
// before blk: fill the directory prefixes and write the sorted lists.
__global__ void compact_kernel(const uint64_t* __restrict__ mask, uint32_t n, uint32_t qn, uint32_t nblk,
                               uint2* __restrict__ rank, const uint32_t* __restrict__ cnt,
                               const uint64_t* __restrict__ cand_off, uint32_t* __restrict__ cand) {
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t blk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; blk < nblk; blk += warps) {
        const uint32_t v = blk * 32 + lane;
        const uint64_t m = v < n ? mask[v] : 0ull;
        if (lane < qn) rank[(size_t)blk * qn + lane].y = cnt[(size_t)lane * (nblk + 1) + blk];
        if (lane + 32 < qn) rank[(size_t)blk * qn + lane + 32].y = cnt[(size_t)(lane + 32) * (nblk + 1) + blk];
        for (uint32_t u = 0; u < qn; ++u) {
            const bool has = (m >> u) & 1ull;
            const uint32_t b = __ballot_sync(kFull, has);
            if (has) {
                uint64_t pos = cand_off[u] + cnt[(size_t)u * (nblk + 1) + blk] + __popc(b & lanemask_lt());
                cand[pos] = v;
            }
        }
    }
}

// ------------------------------------------------------------------ segmented scan
// In-place inclusive scan of uint32 segments (each segment's sum < 2^32).
struct ScanTile {
    uint64_t start;
    uint32_t len;
    uint32_t seg;
};
constexpr uint32_t kScanTile = 4096;
constexpr uint32_t kScanThreads = 256;

__global__ void tile_sum_kernel(const uint32_t* __restrict__ data, const ScanTile* __restrict__ tiles,
                                uint64_t* __restrict__ tsum) {
    SMX_SHARED_ARRAY(uint64_t, red, kScanThreads / 32);
    const ScanTile t = tiles[blockIdx.x];
    uint64_t s = 0;
    for (uint32_t i = threadIdx.x; i < t.len; i += blockDim.x) s += data[t.start + i];
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(kFull, s, o);
    if (lane_id() == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t tot = 0;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) tot += red[w];
        tsum[blockIdx.x] = tot;
    }
}

__global__ void seg_tiles_kernel(uint64_t* __restrict__ tsum, const uint32_t* __restrict__ seg_tile_begin, uint32_t nseg) {
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < nseg; s += gridDim.x * blockDim.x) {
        uint64_t run = 0;
        for (uint32_t t = seg_tile_begin[s]; t < seg_tile_begin[s + 1]; ++t) {
            uint64_t v = tsum[t];
            tsum[t] = run;
            run += v;
        }
    }
}

__global__ void tile_apply_kernel(uint32_t* __restrict__ data, const ScanTile* __restrict__ tiles,
                                  const uint64_t* __restrict__ tsum) {
    constexpr uint32_t kPer = kScanTile / kScanThreads;
    SMX_SHARED_ARRAY(uint32_t, wsum, kScanThreads / 32);
    const ScanTile t = tiles[blockIdx.x];
    uint32_t vals[kPer];
    const uint32_t base = threadIdx.x * kPer;
    uint32_t local = 0;
#pragma unroll
    for (uint32_t i = 0; i < kPer; ++i) {
        uint32_t x = (base + i < t.len) ? data[t.start + base + i] : 0u;
        local += x;
        vals[i] = local;
    }
    // block exclusive scan of the per-thread totals
    uint32_t incl = local;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(kFull, incl, o);
        if (lane_id() >= (uint32_t)o) incl += y;
    }
    if (lane_id() == 31) wsum[threadIdx.x >> 5] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t w = threadIdx.x < blockDim.x / 32 ? wsum[threadIdx.x] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(kFull, w, o);
            if (lane_id() >= (uint32_t)o) w += y;
        }
        if (threadIdx.x < blockDim.x / 32) wsum[threadIdx.x] = w;
    }
    __syncthreads();
    const uint32_t warp_prefix = (threadIdx.x >= 32) ? wsum[(threadIdx.x >> 5) - 1] : 0u;
    const uint32_t excl = (uint32_t)tsum[blockIdx.x] + warp_prefix + incl - local;
#pragma unroll
    for (uint32_t i = 0; i < kPer; ++i)
        if (base + i < t.len) data[t.start + base + i] = excl + vals[i];
}

int segmented_scan(smx_graph* g, uint32_t* d_data, const std::vector<uint64_t>& seg_start,
                   const std::vector<uint64_t>& seg_len) {
    std::vector<ScanTile> tiles;
    std::vector<uint32_t> seg_begin(seg_start.size() + 1, 0);
    for (size_t s = 0; s < seg_start.size(); ++s) {
        seg_begin[s] = (uint32_t)tiles.size();
        for (uint64_t o = 0; o < seg_len[s]; o += kScanTile)
            tiles.push_back({seg_start[s] + o, (uint32_t)std::min<uint64_t>(kScanTile, seg_len[s] - o), (uint32_t)s});
    }
    seg_begin[seg_start.size()] = (uint32_t)tiles.size();
    if (tiles.empty()) return SMX_OK;
    ScanTile* d_tiles = nullptr;
    uint64_t* d_tsum = nullptr;
    uint32_t* d_segb = nullptr;
    cudaStream_t st = g->stream;
    SMX_CUDA_TRY(cudaMallocAsync(&d_tiles, tiles.size() * sizeof(ScanTile), st));
    SMX_CUDA_TRY(cudaMallocAsync(&d_tsum, tiles.size() * sizeof(uint64_t), st));
    SMX_CUDA_TRY(cudaMallocAsync(&d_segb, seg_begin.size() * sizeof(uint32_t), st));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(ScanTile), cudaMemcpyHostToDevice, st));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_segb, seg_begin.data(), seg_begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    SMX_LAUNCH(tile_sum_kernel, (unsigned)tiles.size(), kScanThreads, 0, st, d_data, d_tiles, d_tsum);
    SMX_LAUNCH(seg_tiles_kernel, (unsigned)((seg_start.size() + 127) / 128), 128, 0, st, d_tsum, d_segb,
               (uint32_t)seg_start.size());
    SMX_LAUNCH(tile_apply_kernel, (unsigned)tiles.size(), kScanThreads, 0, st, d_data, d_tiles, d_tsum);
    SMX_CUDA_TRY(cudaGetLastError());
    SMX_CUDA_TRY(cudaFreeAsync(d_tiles, st));
    SMX_CUDA_TRY(cudaFreeAsync(d_tsum, st));
    SMX_CUDA_TRY(cudaFreeAsync(d_segb, st));
    // the host vectors above must outlive the async copies
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    return SMX_OK;
}

// ------------------------------------------------------------------ GQL
// verifyExactTwigIso (filter.h:168-204) for one (u, v): can every query
// neighbour of u be matched to a distinct data neighbour w of v that is still
// a valid candidate of it?  One warp per candidate.
//
// 1. Scan N(v) in chunks of 32; m_w = mask[w] restricted to N(u).  Keep w if
//    it is among the first k (= deg u) data neighbours of some query
//    neighbour (R').  Restricting the right side to R' preserves the answer:
//    a query neighbour with >= k neighbours in R' can always be rematched
//    inside R' (at most k-1 other query neighbours are matched).
// 2. If every query neighbour already has >= k options, Hall's condition
//    holds: saturated.  If some has none: not saturated.
// 3. Otherwise augmenting-path search (bit-parallel BFS over the query side,
//    lanes over R') for the query neighbours with fewer than k options; the
//    others are matched last.  Saturation is a property of the bipartite
//    graph, so the answer equals the reference's greedy + BFS matching
//    (filter.h:95-166), which computes a maximum matching.
__device__ bool twig_saturated(const uint32_t* __restrict__ nb, uint32_t dv, const uint64_t* mask, uint64_t L,
                               uint32_t k, uint64_t* rmask, uint8_t* matchR, uint8_t* pr, uint8_t* visR,
                               uint8_t* matchL, uint32_t rcap) {
    const uint32_t lane = lane_id();
    if (k == 0) return true;
    if (dv < k) return false;
    uint32_t c_lo = 0, c_hi = 0;  // lane j counts options of query vertex j and j + 32
    uint64_t uni = 0;
    uint32_t r = 0;
    for (uint32_t base = 0; base < dv; base += 32) {
        const uint32_t j = base + lane;
        uint64_t m = 0;
        if (j < dv) m = mask[nb[j]] & L;
        uni |= warp_or64(m);
        bool keep = false;
        uint64_t bits = L;
        while (bits) {
            const int i = __ffsll((long long)bits) - 1;
            bits &= bits - 1;
            const bool has = (m >> i) & 1ull;
            const uint32_t b = __ballot_sync(kFull, has);
            if (b == 0) continue;
            const uint32_t ci = __shfl_sync(kFull, i < 32 ? c_lo : c_hi, i & 31);
            if (has && ci + __popc(b & lanemask_lt()) < k) keep = true;
            if (lane == (uint32_t)(i & 31)) {
                if (i < 32) c_lo += __popc(b); else c_hi += __popc(b);
            }
        }
        const uint32_t kb = __ballot_sync(kFull, keep);
        if (keep) {
            const uint32_t p = r + __popc(kb & lanemask_lt());
            if (p < rcap) rmask[p] = m;
        }
        r += __popc(kb);
        const bool low = (((L >> lane) & 1ull) && c_lo < k) || (((L >> (lane + 32)) & 1ull) && c_hi < k);
        if (!__any_sync(kFull, low)) return true;
    }
    if (uni != L) return false;
    if (r > rcap) r = rcap;  // cannot happen: |R'| <= k * k <= rcap
    const uint32_t con_lo = __ballot_sync(kFull, ((L >> lane) & 1ull) && c_lo < k);
    const uint32_t con_hi = __ballot_sync(kFull, ((L >> (lane + 32)) & 1ull) && c_hi < k);
    uint64_t con = ((uint64_t)con_hi << 32) | con_lo;
    for (uint32_t j = lane; j < r; j += 32) matchR[j] = 0xff;
    matchL[lane] = 0xff;
    matchL[lane + 32] = 0xff;
    __syncwarp();
    while (con) {
        const int i = __ffsll((long long)con) - 1;
        con &= con - 1;
        for (uint32_t j = lane; j < r; j += 32) visR[j] = 0;
        __syncwarp();
        uint64_t F = 1ull << i, VL = F;
        uint32_t found = 0xffffffffu;
        for (uint32_t level = 0; F && level <= k; ++level) {
            uint64_t NF = 0;
            uint32_t fnd = 0xffffffffu;
            for (uint32_t j = lane; j < r; j += 32) {
                const uint64_t a = rmask[j] & F;
                if (a && !visR[j]) {
                    visR[j] = 1;
                    pr[j] = (uint8_t)(__ffsll((long long)a) - 1);
                    const uint8_t ml = matchR[j];
                    if (ml == 0xff) fnd = min(fnd, j);
                    else NF |= 1ull << ml;
                }
            }
            fnd = __reduce_min_sync(kFull, fnd);
            NF = warp_or64(NF);
            __syncwarp();
            if (fnd != 0xffffffffu) {
                found = fnd;
                break;
            }
            NF &= ~VL;
            VL |= NF;
            F = NF;
        }
        if (found == 0xffffffffu) return false;
        if (lane == 0) {
            uint32_t j = found;
            for (uint32_t guard = 0; guard <= k; ++guard) {
                const uint8_t l = pr[j];
                const uint8_t nj = matchL[l];
                matchR[j] = l;
                matchL[l] = (uint8_t)j;
                if ((int)l == i || nj == 0xff) break;
                j = nj;
            }
        }
        __syncwarp();
    }
    return true;
}

// One GQL step (filter.h:274-289 for one query vertex u): every still-valid
// candidate v of u is verified; failures clear bit u of mask[v].  Other
// warps only read bits of u's neighbours, which this launch never changes,
// so the order of updates inside the launch does not matter; launches run
// in query-vertex order within a round, as the reference's loop does.
__global__ void gql_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ adj, uint64_t* mask,
                           const uint32_t* __restrict__ list, uint32_t list_len, uint32_t u, uint64_t L, uint32_t k,
                           uint32_t rcap) {
    SMX_EXTERN_SMEM(smem);
    const uint32_t warp = threadIdx.x >> 5;
    const size_t per_warp = ((size_t)rcap * 11 + 64 + 15) & ~(size_t)15;
    unsigned char* base = smem + per_warp * warp;
    uint64_t* rmask = reinterpret_cast<uint64_t*>(base);
    uint8_t* matchR = base + (size_t)rcap * 8;
    uint8_t* pr = matchR + rcap;
    uint8_t* visR = pr + rcap;
    uint8_t* matchL = visR + rcap;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < list_len; i += warps) {
        const uint32_t v = list[i];
        if (!((mask[v] >> u) & 1ull)) continue;
        const uint64_t o0 = off[v];
        const uint32_t dv = (uint32_t)(off[v + 1] - o0);
        const bool ok = twig_saturated(adj + o0, dv, mask, L, k, rmask, matchR, pr, visR, matchL, rcap);
        if (!ok && lane_id() == 0) atomicAnd(reinterpret_cast<unsigned long long*>(mask + v), ~(1ull << u));
        __syncwarp();
    }
}

// ------------------------------------------------------------------ edge tables
struct TabDesc {
    const uint32_t* rows;   // C(a)
    uint32_t* edge;         // output
    uint64_t off_base;      // start of this table's offsets in the shared array
    uint32_t v_cnt;
    uint32_t b;
};

// Row i of E[a][b] (table.h:65-90): data neighbours of C(a)[i] that are
// candidates of b.  One warp per row; counts go to offs[base + i + 1].
__global__ void table_count_kernel(const TabDesc* __restrict__ td, const uint64_t* __restrict__ off,
                                   const uint32_t* __restrict__ adj, const uint64_t* __restrict__ mask,
                                   uint32_t* __restrict__ offs, uint32_t* __restrict__ tmax) {
    const TabDesc t = td[blockIdx.y];
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < t.v_cnt; i += warps) {
        const uint32_t v = __ldg(t.rows + i);
        const uint64_t o0 = __ldg(off + v), o1 = __ldg(off + v + 1);
        uint32_t c = 0;
        for (uint64_t e = o0; e < o1; e += 32) {
            bool f = false;
            if (e + lane < o1) f = (__ldg(mask + __ldg(adj + e + lane)) >> t.b) & 1ull;
            c += __popc(__ballot_sync(kFull, f));
        }
        if (lane == 0) {
            offs[t.off_base + i + 1] = c;
            atomicMax(tmax + blockIdx.y, c);
        }
    }
}

__global__ void table_fill_kernel(const TabDesc* __restrict__ td, const uint64_t* __restrict__ off,
                                  const uint32_t* __restrict__ adj, const uint64_t* __restrict__ mask,
                                  const uint32_t* __restrict__ offs, const uint2* __restrict__ rank, uint32_t qn) {
    const TabDesc t = td[blockIdx.y];
    const uint32_t lane = lane_id();
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < t.v_cnt; i += warps) {
        const uint32_t v = __ldg(t.rows + i);
        const uint64_t o0 = __ldg(off + v), o1 = __ldg(off + v + 1);
        uint32_t pos = offs[t.off_base + i];
        for (uint64_t e = o0; e < o1; e += 32) {
            bool f = false;
            uint32_t w = 0;
            if (e + lane < o1) {
                w = __ldg(adj + e + lane);
                f = (__ldg(mask + w) >> t.b) & 1ull;
            }
            const uint32_t b = __ballot_sync(kFull, f);
            if (f) t.edge[pos + __popc(b & lanemask_lt())] = cand_rank(rank, qn, t.b, w);
            pos += __popc(b);
        }
    }
}

struct Timer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit Timer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    double stop() {
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
    ~Timer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

unsigned grid_for(const smx_graph* g, uint64_t work, unsigned per_block) {
    uint64_t blocks = (work + per_block - 1) / per_block;
    uint64_t cap = (uint64_t)g->num_sms * 16;
    if (blocks > cap) blocks = cap;
    return (unsigned)std::max<uint64_t>(1, blocks);
}

// mask -> rank directory + sorted candidate lists + counts.
int compact(smx_graph* g, smx_cand* c) {
    cudaStream_t st = g->stream;
    const uint32_t n = g->h.n, qn = c->qn;
    const uint32_t nblk = (n + 31) / 32;
    if (!c->d_rank) SMX_CUDA_TRY(cudaMallocAsync(&c->d_rank, (size_t)nblk * qn * sizeof(uint2) + 16, st));
    uint32_t* d_cnt = nullptr;
    SMX_CUDA_TRY(cudaMallocAsync(&d_cnt, (size_t)qn * (nblk + 1) * sizeof(uint32_t), st));
    const unsigned warps_grid = grid_for(g, (uint64_t)nblk * 32, 256);
    SMX_LAUNCH(rank_bits_kernel, warps_grid, 256, 0, st, c->d_mask, n, qn, nblk, c->d_rank, d_cnt);
    SMX_CUDA_TRY(cudaGetLastError());
    std::vector<uint64_t> ss(qn), sl(qn);
    for (uint32_t u = 0; u < qn; ++u) {
        ss[u] = (uint64_t)u * (nblk + 1);
        sl[u] = nblk + 1;
    }
    int rc = segmented_scan(g, d_cnt, ss, sl);
    if (rc != SMX_OK) return rc;
    std::vector<uint32_t> tot(qn);
    for (uint32_t u = 0; u < qn; ++u)
        SMX_CUDA_TRY(cudaMemcpyAsync(&tot[u], d_cnt + (size_t)u * (nblk + 1) + nblk, 4, cudaMemcpyDeviceToHost, st));
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    c->cnt = tot;
    c->cand_off.assign(qn + 1, 0);
    for (uint32_t u = 0; u < qn; ++u) c->cand_off[u + 1] = c->cand_off[u] + tot[u];
    if (c->d_cand) SMX_CUDA_TRY(cudaFreeAsync(c->d_cand, st));
    SMX_CUDA_TRY(cudaMallocAsync(&c->d_cand, (c->cand_off[qn] + 8) * sizeof(uint32_t), st));
    uint64_t* d_coff = nullptr;
    SMX_CUDA_TRY(cudaMallocAsync(&d_coff, (qn + 1) * sizeof(uint64_t), st));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_coff, c->cand_off.data(), (qn + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    SMX_LAUNCH(compact_kernel, warps_grid, 256, 0, st, c->d_mask, n, qn, nblk, c->d_rank, d_cnt, d_coff, c->d_cand);
    SMX_CUDA_TRY(cudaGetLastError());
    SMX_CUDA_TRY(cudaFreeAsync(d_coff, st));
    SMX_CUDA_TRY(cudaFreeAsync(d_cnt, st));
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    return SMX_OK;
}

int build_tables(smx_graph* g, const HostQuery& q, smx_cand* c) {
    cudaStream_t st = g->stream;
    std::vector<TabDesc> td;
    std::vector<uint64_t> seg_start, seg_len;
    uint64_t off_total = 0;
    c->tables.clear();
    for (uint32_t a = 0; a < q.n; ++a)
        for (uint32_t e = q.off[a]; e < q.off[a + 1]; ++e) {
            const uint32_t b = q.adj[e];
            DevTable t;
            t.a = a;
            t.b = b;
            t.v_cnt = c->cnt[a];
            c->tab_index[a][b] = (int)c->tables.size();
            c->tables.push_back(t);
            td.push_back({c->cand_ptr(a), nullptr, off_total, t.v_cnt, b});
            seg_start.push_back(off_total);
            seg_len.push_back((uint64_t)t.v_cnt + 1);
            off_total += t.v_cnt + 1;
        }
    const size_t nt = td.size();
    if (nt == 0) return SMX_OK;
    uint32_t* d_offs = nullptr;
    uint32_t* d_tmax = nullptr;
    TabDesc* d_td = nullptr;
    SMX_CUDA_TRY(cudaMallocAsync(&d_offs, off_total * sizeof(uint32_t) + 16, st));
    c->d_table_off = d_offs;
    SMX_CUDA_TRY(cudaMallocAsync(&d_tmax, nt * sizeof(uint32_t), st));
    SMX_CUDA_TRY(cudaMallocAsync(&d_td, nt * sizeof(TabDesc), st));
    SMX_CUDA_TRY(cudaMemsetAsync(d_offs, 0, off_total * sizeof(uint32_t), st));
    SMX_CUDA_TRY(cudaMemsetAsync(d_tmax, 0, nt * sizeof(uint32_t), st));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_td, td.data(), nt * sizeof(TabDesc), cudaMemcpyHostToDevice, st));
    uint32_t max_rows = 0;
    for (auto& t : td) max_rows = std::max(max_rows, t.v_cnt);
    dim3 grid(std::min<unsigned>(256, grid_for(g, (uint64_t)max_rows * 32, 256)), (unsigned)nt);
    SMX_LAUNCH(table_count_kernel, grid, 256, 0, st, d_td, g->d_off, g->d_adj, c->d_mask, d_offs, d_tmax);
    SMX_CUDA_TRY(cudaGetLastError());
    // the per-table inclusive scan turns [0, c0, c1, ...] into offsets
    int rc = segmented_scan(g, d_offs, seg_start, seg_len);
    if (rc != SMX_OK) return rc;
    std::vector<uint32_t> tmax(nt), ecnt(nt);
    SMX_CUDA_TRY(cudaMemcpyAsync(tmax.data(), d_tmax, nt * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    for (size_t i = 0; i < nt; ++i)
        SMX_CUDA_TRY(cudaMemcpyAsync(&ecnt[i], d_offs + seg_start[i] + td[i].v_cnt, 4, cudaMemcpyDeviceToHost, st));
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < nt; ++i) {
        DevTable& t = c->tables[i];
        t.e_cnt = ecnt[i];
        t.max_deg = tmax[i];
        SMX_CUDA_TRY(cudaMallocAsync(&t.d_edge, (t.e_cnt + 8) * sizeof(uint32_t), st));
        t.d_off = d_offs + seg_start[i];
        td[i].edge = t.d_edge;
    }
    SMX_CUDA_TRY(cudaMemcpyAsync(d_td, td.data(), nt * sizeof(TabDesc), cudaMemcpyHostToDevice, st));
    SMX_LAUNCH(table_fill_kernel, grid, 256, 0, st, d_td, g->d_off, g->d_adj, c->d_mask, d_offs, c->d_rank, c->qn);
    SMX_CUDA_TRY(cudaGetLastError());
    SMX_CUDA_TRY(cudaFreeAsync(d_tmax, st));
    SMX_CUDA_TRY(cudaFreeAsync(d_td, st));
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    return SMX_OK;
}

}  // namespace

int upload_graph(smx_graph* g) {
    SMX_CUDA_TRY(cudaSetDevice(g->device));
    SMX_CUDA_TRY(cudaDeviceGetAttribute(&g->num_sms, cudaDevAttrMultiProcessorCount, g->device));
    SMX_CUDA_TRY(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    {
        // candidate sets and plans come from the device's default pool
        // (cudaMallocAsync); keep up to 8 GB of freed blocks in the pool
        // instead of returning them to the driver at every synchronisation,
        // which costs up to a second per filter / destroy on large graphs
        // (beyond 8 GB the pool gives memory back, so plain cudaMalloc of the
        // enumeration scratch still finds it)
        cudaMemPool_t pool;
        SMX_CUDA_TRY(cudaDeviceGetDefaultMemPool(&pool, g->device));
        uint64_t keep = 8ull << 30;
        SMX_CUDA_TRY(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    const HostGraph& h = g->h;
    cudaStream_t st = g->stream;
    SMX_CUDA_TRY(cudaMalloc(&g->d_off, (h.n + 1) * sizeof(uint64_t)));
    // 32 bytes of padding: rounded-up 16-byte bulk reads of the last row stay inside
    SMX_CUDA_TRY(cudaMalloc(&g->d_adj, h.m2 * sizeof(uint32_t) + 32));
    SMX_CUDA_TRY(cudaMalloc(&g->d_lab, (size_t)std::max<uint32_t>(h.n, 1) * sizeof(uint32_t)));
    SMX_CUDA_TRY(cudaMemsetAsync(g->d_adj, 0, h.m2 * sizeof(uint32_t) + 32, st));
    SMX_CUDA_TRY(cudaMemcpyAsync(g->d_off, h.off.data(), (h.n + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    if (h.m2) SMX_CUDA_TRY(cudaMemcpyAsync(g->d_adj, h.adj.data(), h.m2 * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    if (h.n) SMX_CUDA_TRY(cudaMemcpyAsync(g->d_lab, h.lab.data(), h.n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    if (h.label_cnt > 1 && h.label_cnt <= 64) {
        g->hist_stride = (h.label_cnt + 15) & ~15u;
        SMX_CUDA_TRY(cudaMalloc(&g->d_hist, (size_t)h.n * g->hist_stride));
        SMX_CUDA_TRY(cudaMemsetAsync(g->d_hist, 0, (size_t)h.n * g->hist_stride, st));
        SMX_LAUNCH(hist_kernel, grid_for(g, h.n, 256), 256, 0, st, g->d_off, g->d_adj, g->d_lab, h.n, g->hist_stride,
                   g->d_hist);
        SMX_CUDA_TRY(cudaGetLastError());
    }
    {
        // hub adjacency (used by the enumerator for membership tests)
        constexpr uint32_t kMaxHubs = 16384, kMinHubDeg = 16;
        std::vector<uint32_t> byd(h.n);
        std::iota(byd.begin(), byd.end(), 0u);
        const uint32_t k = std::min<uint32_t>(kMaxHubs, h.n);
        std::partial_sort(byd.begin(), byd.begin() + k, byd.end(), [&](uint32_t a, uint32_t b) {
            return h.deg(a) != h.deg(b) ? h.deg(a) > h.deg(b) : a < b;
        });
        uint32_t hubs = 0;
        while (hubs < k && h.deg(byd[hubs]) >= kMinHubDeg) ++hubs;
        g->hubs = hubs;
        g->hub_words = (hubs + 31) / 32;
        std::vector<uint32_t> hid(h.n, 0xffffffffu);
        for (uint32_t i = 0; i < hubs; ++i) hid[byd[i]] = i;
        std::vector<uint32_t> bits((size_t)hubs * g->hub_words, 0u);
        for (uint32_t i = 0; i < hubs; ++i) {
            const uint32_t v = byd[i];
            for (uint64_t e = h.off[v]; e < h.off[v + 1]; ++e) {
                const uint32_t j = hid[h.adj[e]];
                if (j != 0xffffffffu) bits[(size_t)i * g->hub_words + (j >> 5)] |= 1u << (j & 31);
            }
        }
        SMX_CUDA_TRY(cudaMalloc(&g->d_hub_id, (size_t)std::max<uint32_t>(h.n, 1) * 4));
        SMX_CUDA_TRY(cudaMalloc(&g->d_hub_bits, std::max<size_t>(bits.size(), 1) * 4));
        if (h.n) SMX_CUDA_TRY(cudaMemcpyAsync(g->d_hub_id, hid.data(), (size_t)h.n * 4, cudaMemcpyHostToDevice, st));
        if (!bits.empty())
            SMX_CUDA_TRY(cudaMemcpyAsync(g->d_hub_bits, bits.data(), bits.size() * 4, cudaMemcpyHostToDevice, st));
    }
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    return SMX_OK;
}

void free_cand_device(smx_cand* c) {
    if (!c || !c->g) return;  // no graph: freed when the graph was destroyed
    cudaSetDevice(c->g->device);
    cudaStream_t st = c->g->stream;
    if (c->d_mask) cudaFreeAsync(c->d_mask, st);
    if (c->d_rank) cudaFreeAsync(c->d_rank, st);
    if (c->d_cand) cudaFreeAsync(c->d_cand, st);
    for (size_t i = 0; i < c->tables.size(); ++i)
        if (c->tables[i].d_edge) cudaFreeAsync(c->tables[i].d_edge, st);
    if (c->d_table_off) cudaFreeAsync(c->d_table_off, st);
    cudaStreamSynchronize(st);
    c->d_mask = nullptr;
    c->d_rank = nullptr;
    c->d_cand = nullptr;
    c->d_table_off = nullptr;
    c->tables.clear();
}

// Filter_NLF / Filter_GQL + FilterParamConstruct (filter.h:1049-1063, :60-78).
int device_filter(smx_graph* g, const HostQuery& q, int kind, int build, smx_cand* c) {
    SMX_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t st = g->stream;
    const uint32_t n = g->h.n;
    c->g = g;
    c->qn = q.n;
    c->kind = kind;
    c->ok = 0;
    for (uint32_t a = 0; a < kMaxQ; ++a)
        for (uint32_t b = 0; b < kMaxQ; ++b) c->tab_index[a][b] = -1;
    // query description
    std::vector<QInfo> hqv(1);
    QInfo* hq = hqv.data();
    std::memset(hq, 0, sizeof(QInfo));
    hq->n = q.n;
    hq->data_labels = g->h.label_cnt;
    hq->hist_stride = g->hist_stride;
    uint32_t np = 0;
    for (uint32_t u = 0; u < q.n; ++u) {
        hq->lab[u] = q.lab[u];
        hq->deg[u] = q.deg(u);
        hq->nlf_off[u] = np;
        uint32_t start = np;
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            uint32_t l = q.lab[q.adj[e]];
            uint32_t k = start;
            while (k < np && hq->nlf_lab[k] != l) ++k;
            if (k == np) {
                hq->nlf_lab[np] = l;
                hq->nlf_cnt[np] = 0;
                ++np;
            }
            hq->nlf_cnt[k]++;
        }
    }
    hq->nlf_off[q.n] = np;
    QInfo* d_q = nullptr;
    SMX_CUDA_TRY(cudaMallocAsync(&d_q, sizeof(QInfo), st));
    SMX_CUDA_TRY(cudaMemcpyAsync(d_q, hq, sizeof(QInfo), cudaMemcpyHostToDevice, st));
    SMX_CUDA_TRY(cudaMallocAsync(&c->d_mask, (size_t)std::max<uint32_t>(n, 1) * sizeof(uint64_t) + 16, st));
    {
        Timer t(st);
        SMX_LAUNCH(nlf_mask_kernel, grid_for(g, n, 256), 256, 0, st, g->d_off, g->d_adj, g->d_lab, g->d_hist, n, d_q,
                   c->d_mask);
        SMX_CUDA_TRY(cudaGetLastError());
        c->ms[0] = t.stop();
    }
    SMX_CUDA_TRY(cudaFreeAsync(d_q, st));
    SMX_CUDA_TRY(cudaStreamSynchronize(st));
    {
        Timer t(st);
        int rc = compact(g, c);
        if (rc != SMX_OK) return rc;
        c->ms[2] = t.stop();
    }
    // _NLF_Filter stops at the first query vertex without candidates (filter.h:87-90)
    for (uint32_t u = 0; u < q.n; ++u)
        if (c->cnt[u] == 0) {
            for (uint32_t w = u + 1; w < q.n; ++w) c->cnt[w] = 0;
            return SMX_EMPTY_CANDIDATES;
        }
    if (kind == SMX_FILTER_GQL) {
        Timer t(st);
        // The lists of the NLF compaction stay the iteration sets of both
        // rounds (the reference iterates candidates[u] and skips INVALID).
        std::vector<uint64_t> off0 = c->cand_off;
        std::vector<uint32_t> cnt0 = c->cnt;
        uint32_t* list0 = c->d_cand;
        c->d_cand = nullptr;
        for (int round = 0; round < 2; ++round)
            for (uint32_t u = 0; u < q.n; ++u) {
                const uint32_t k = q.deg(u);
                const uint32_t rcap = std::max<uint32_t>(32, k * k);
                const size_t per_warp = ((size_t)rcap * 11 + 64 + 15) & ~(size_t)15;
                const uint32_t wpb = (uint32_t)std::min<size_t>(8, std::max<size_t>(1, (96 * 1024) / per_warp));
                const size_t smem = per_warp * wpb;
                if (smem > 48 * 1024)
                    SMX_CUDA_TRY(cudaFuncSetAttribute(gql_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                const unsigned grid = grid_for(g, (uint64_t)cnt0[u] * 32, wpb * 32);
                SMX_LAUNCH(gql_kernel, grid, wpb * 32, smem, st, g->d_off, g->d_adj, c->d_mask, list0 + off0[u], cnt0[u],
                           u, q.nbr_mask[u], k, rcap);
                SMX_CUDA_TRY(cudaGetLastError());
            }
        c->ms[1] = t.stop();
        SMX_CUDA_TRY(cudaFreeAsync(list0, st));
        Timer t2(st);
        int rc = compact(g, c);
        if (rc != SMX_OK) return rc;
        c->ms[2] += t2.stop();
        for (uint32_t u = 0; u < q.n; ++u)
            if (c->cnt[u] == 0) return SMX_EMPTY_CANDIDATES;  // isCandidateSetValid, filter.h:222-230
    }
    if (build) {
        Timer t(st);
        int rc = build_tables(g, q, c);
        if (rc != SMX_OK) return rc;
        c->ms[3] = t.stop();
    }
    c->ok = 1;
    return SMX_OK;
}

}  // namespace smx
