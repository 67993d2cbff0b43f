// Oracle driver over the reference implementation itself.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
// reference's own headers, read in place (filter.h, table.h, order.h,
// explore.h, code_gen.h, api.h, graph.h), into oracle/_ref/libsmx_refdriver.so
// by oracle/Makefile.  It exposes a plain C ABI so the tests, the golden-vector
// script and bench.py's reference arm can run the reference's own functions:
//
//   Graph::Load / Query::Load              graph.h:190-266, :474-478
//   Filter_NLF / Filter_GQL                filter.h:1049-1063
//   Order_RI / Order_GQL                   order.h:1138-1281, :563-597
//   explore_Intersection_Recursive<CandidatesBuffer>      explore.h:613-670
//   explore_Intersection_Cache_DAF_Filter                 explore.h:1073-1129
//   explore_Intersection_All<true,false,false,false,false> explore.h:2757-2848
//
// The reference drivers (src/*.cpp) hard-code output_limit=1e5, so this driver
// is the reference harness with exhaustive limits.  For multi-threaded runs the
// root loop (explore.h:638-663 / :1100-1122) is sharded across threads, each
// thread calling the reference's own recursive step (_explore_recur,
// explore.h:516, or _explore_recur_cache_daf_filter, explore.h:968) with its
// own buffer; the root loop is an independent sum, so the count is unchanged.
#include <atomic>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include <time.h>

#include "graph.h"
#include "filter.h"
#include "table.h"
#include "order.h"
#include "explore.h"
#include "code_gen.h"
#include "api.h"

namespace {

struct RefCand {
    CandidateParam* can = nullptr;
    bool ok = false;
};

double now_ms() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1000.0 + t.tv_nsec / 1e6;
}

}  // namespace

extern "C" {

void* smxref_graph_load(const char* path) {
    Graph* g = new Graph();
    g->Load(path);
    return g;
}

void* smxref_query_load(const char* path) {
    Query* q = new Query();
    q->Load(path);
    return q;
}

void smxref_graph_free(void* g) { delete static_cast<Graph*>(g); }
void smxref_query_free(void* q) { delete static_cast<Query*>(q); }

uint32_t smxref_graph_vcount(void* g) { return static_cast<Graph*>(g)->getVertexCnt(); }
uint32_t smxref_graph_ecount(void* g) { return static_cast<Graph*>(g)->getEdgeCnt(); }
uint32_t smxref_graph_maxdeg(void* g) { return static_cast<Graph*>(g)->getMaxDgree(); }
uint32_t smxref_graph_labelcnt(void* g) { return static_cast<Graph*>(g)->getLabelCnt(); }
uint32_t smxref_query_kcore(void* q, uint32_t v) { return static_cast<Query*>(q)->getKCoreValue(v); }

// kind: 0 = Filter_NLF, 1 = Filter_GQL.  Returns a handle (never null) whose
// smxref_cand_ok() tells whether the filter returned true.
void* smxref_filter(void* data, void* query, int kind, double* ms) {
    Graph* d = static_cast<Graph*>(data);
    Query* q = static_cast<Query*>(query);
    RefCand* rc = new RefCand();
    rc->can = new CandidateParam(*d, *q);
    double t0 = now_ms();
    if (kind == 0) rc->ok = Filter_NLF(*d, *q, *rc->can);
    else rc->ok = Filter_GQL(*d, *q, *rc->can);
    if (ms) *ms = now_ms() - t0;
    return rc;
}

int smxref_cand_ok(void* c) { return static_cast<RefCand*>(c)->ok ? 1 : 0; }

void smxref_cand_free(void* c) {
    RefCand* rc = static_cast<RefCand*>(c);
    delete rc->can;
    delete rc;
}

uint32_t smxref_cand_count(void* c, uint32_t u) {
    return static_cast<RefCand*>(c)->can->candidates_count[u];
}

void smxref_cand_copy(void* c, uint32_t u, uint32_t* out) {
    CandidateParam* can = static_cast<RefCand*>(c)->can;
    std::memcpy(out, can->candidates[u], sizeof(uint32_t) * can->candidates_count[u]);
}

// Edge table edge_matrix[a][b]: returns 0 when the table does not exist.
int smxref_table_info(void* c, uint32_t a, uint32_t b, uint32_t* v_cnt, uint32_t* e_cnt, uint32_t* max_deg) {
    CandidateParam* can = static_cast<RefCand*>(c)->can;
    Edges* e = can->edge_matrix[a][b];
    if (!e) return 0;
    *v_cnt = e->_v_cnt;
    *e_cnt = e->_e_cnt;
    *max_deg = e->_max_degree;
    return 1;
}

void smxref_table_copy(void* c, uint32_t a, uint32_t b, uint32_t* offset, uint32_t* edge, uint32_t* edge_v) {
    CandidateParam* can = static_cast<RefCand*>(c)->can;
    Edges* e = can->edge_matrix[a][b];
    std::memcpy(offset, e->_offset, sizeof(uint32_t) * (e->_v_cnt + 1));
    std::memcpy(edge, e->_edge, sizeof(uint32_t) * e->_e_cnt);
    std::memcpy(edge_v, e->_edge_v, sizeof(uint32_t) * e->_e_cnt);
}

void smxref_order_ri(void* query, uint32_t* out) {
    Order o;
    Order_RI(*static_cast<Query*>(query), o);
    for (size_t i = 0; i < o.size(); ++i) out[i] = o[i];
}

void smxref_order_gql(void* data, void* query, void* c, uint32_t* out) {
    Order o;
    Order_GQL(*static_cast<Graph*>(data), *static_cast<Query*>(query), *static_cast<RefCand*>(c)->can, o);
    for (size_t i = 0; i < o.size(); ++i) out[i] = o[i];
}

int smxref_order_valid(void* query, const uint32_t* order, uint32_t n) {
    Order o(order, order + n);
    return isValid(o, *static_cast<Query*>(query)) ? 1 : 0;
}

// explorer: 0 = explore_Intersection_Recursive<CandidatesBuffer>
//           1 = explore_Intersection_Cache_DAF_Filter
//           2 = explore_Intersection_All<true,false,false,false,false>  (1 thread only)
// limit: output_limit (0 = unlimited).  Returns the count; *ms is the wall time
// of the enumeration; *intersections is the Profiler's total_intersection sum.
uint64_t smxref_explore(void* data, void* query, void* c, const uint32_t* order_in, int explorer,
                        uint64_t limit, int threads, double* ms, uint64_t* intersections) {
    const Graph& d = *static_cast<Graph*>(data);
    const Query& q = *static_cast<Query*>(query);
    CandidateParam* can = static_cast<RefCand*>(c)->can;
    const uint32_t n = q.getVertexCnt();
    Order order(order_in, order_in + n);
    const uint64_t out_limit = limit ? limit : (uint64_t)-1;

    Config cfg;
    cfg.useFilter = true;
    cfg.can = can;
    ReuseParam* reuse = nullptr;
    if (explorer == 1) {
        reuse = new ReuseParam(q, order);
        cfg.useCache = true;
        cfg.reuse = reuse;
        cfg.useDAFFailingPrune = true;
    }

    std::atomic<uint64_t> total{0};
    std::atomic<uint64_t> inter{0};
    double t0 = now_ms();

    if (threads <= 1 || explorer == 2) {
        std::atomic<bool> stop{false};
        size_t ans = 0;
        double tm = 0.0;
        Profiler::getInst().reset();
        if (explorer == 0)
            explore_Intersection_Recursive<CandidatesBuffer>(d, q, order, cfg, tm, ans, stop, out_limit);
        else if (explorer == 1)
            explore_Intersection_Cache_DAF_Filter(d, q, order, cfg, tm, ans, stop, out_limit);
        else
            explore_Intersection_All<true, false, false, false, false>(d, q, order, cfg, tm, ans, stop, out_limit);
        total = ans;
        inter = Profiler::getInst().total_intersection;
    } else {
        const uint32_t u0 = order[0];
        const uint32_t roots = can->candidates_count[u0];
        std::atomic<uint32_t> next{0};
        std::atomic<bool> global_stop{false};
        auto worker = [&]() {
            Profiler::getInst().reset();
            std::atomic<bool> stop{false};
            if (explorer == 0) {
                CandidatesBuffer buf;
                buf.allocate(d, q, order, cfg);
                while (!global_stop.load()) {
                    uint32_t r = next.fetch_add(1);
                    if (r >= roots) break;
                    // Root step of explore.h:638-663.
                    buf.pos[0] = r;
                    buf.tot[0] = roots;
                    buf.valid_candidate_idx[0][r] = r;
                    VertexID v0 = can->candidates[u0][r];
                    if (d.getVertexLabel(v0) != q.getVertexLabel(u0)) continue;
                    buf.embedding[u0] = v0;
                    buf.idx_embedding[u0] = r;
                    buf.vis[v0] = true;
                    buf.reverse_embeddings_deps[v0] = 0;
                    size_t ans = 0;
                    uint64_t remaining = out_limit - std::min<uint64_t>(out_limit, total.load());
                    if (remaining == 0) { global_stop = true; break; }
                    _explore_recur<CandidatesBuffer>(d, q, order, cfg, &buf, 1, ans, stop, remaining);
                    buf.vis[v0] = false;
                    uint64_t t = total.fetch_add(ans) + ans;
                    if (t >= out_limit || stop.load()) global_stop = true;
                }
                buf.release();
            } else {
                CacheBuffer buf;
                buf.allocate(d, q, order, cfg);
                DAFFailingPrune fp;
                fp.Init(q, order);
                while (!global_stop.load()) {
                    uint32_t r = next.fetch_add(1);
                    if (r >= roots) break;
                    // Root step of explore.h:1100-1122.
                    buf.pos[0] = r;
                    buf.tot[0] = roots;
                    buf.valid_candidate_idx[0][r] = r;
                    VertexID v0 = can->candidates[u0][r];
                    buf.embedding[u0] = v0;
                    buf.idx_embedding[u0] = r;
                    buf.vis[v0] = true;
                    buf.reverse_embeddings_deps[v0] = 0;
                    size_t ans = 0;
                    uint64_t remaining = out_limit - std::min<uint64_t>(out_limit, total.load());
                    if (remaining == 0) { global_stop = true; break; }
                    _explore_recur_cache_daf_filter(d, q, order, cfg, &buf, &fp, 1, ans, stop, remaining);
                    buf.vis[v0] = false;
                    uint64_t t = total.fetch_add(ans) + ans;
                    if (t >= out_limit || stop.load()) global_stop = true;
                }
                buf.release();
            }
            inter += Profiler::getInst().total_intersection;
        };
        std::vector<std::thread> pool;
        for (int i = 0; i < threads; ++i) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }

    if (ms) *ms = now_ms() - t0;
    if (intersections) *intersections = inter.load();
    delete reuse;
    uint64_t t = total.load();
    return t < out_limit ? t : out_limit;
}

}  // extern "C"
