// The C ABI of libsmx (include/smx.h): argument checks, handle lifetime and
// status mapping around the host components (host.cpp) and the device
// pipeline (filter.cu, enumerate.cu).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "smx_internal.h"

using namespace smx;

namespace smx {
uint64_t launch_count();
}

namespace {
int check_device(int device) {
    if (device < 0) return SMX_OK;  // host-only graph
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(SMX_NO_DEVICE, "no CUDA device");
    }
    if (device >= n) return fail(SMX_BAD_ARGUMENT, "device index out of range");
    return SMX_OK;
}

// device < 0 keeps the graph on the host only (generators, text I/O, tests on
// machines without a GPU); filtering and enumeration need a device graph.
int finish_graph(smx_graph* g, int device, smx_graph** out) {
    g->device = device;
    if (device < 0) {
        *out = g;
        return SMX_OK;
    }
    int rc = upload_graph(g);
    if (rc != SMX_OK) {
        smx_graph_destroy(g);
        return rc;
    }
    *out = g;
    return SMX_OK;
}
}  // namespace

extern "C" {

const char* smx_status_str(int status) {
    switch (status) {
        case SMX_OK: return "ok";
        case SMX_EMPTY_CANDIDATES: return "empty candidate set";
        case SMX_INVALID_ORDER: return "invalid matching order";
        case SMX_TOO_LARGE: return "too large";
        case SMX_TIMEOUT: return "timeout";
        case SMX_CUDA_ERROR: return "CUDA error";
        case SMX_BAD_ARGUMENT: return "bad argument";
        case SMX_BAD_FORMAT: return "bad graph format";
        case SMX_IO_ERROR: return "I/O error";
        case SMX_STOPPED: return "stopped";
        case SMX_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* smx_last_error(void) { return last_error().c_str(); }

int smx_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

int smx_mark_begin(smx_graph* g) {
    if (!g || g->device < 0) return fail(SMX_BAD_ARGUMENT, "needs a device graph");
    SMX_CUDA_TRY(cudaSetDevice(g->device));
    for (auto& e : g->mark)
        if (!e) SMX_CUDA_TRY(cudaEventCreate(&e));
    SMX_CUDA_TRY(cudaEventRecord(g->mark[0], g->stream));
    return SMX_OK;
}

int smx_mark_end(smx_graph* g, double* ms) {
    if (!g || !ms || !g->mark[0]) return fail(SMX_BAD_ARGUMENT, "smx_mark_begin first");
    SMX_CUDA_TRY(cudaEventRecord(g->mark[1], g->stream));
    SMX_CUDA_TRY(cudaEventSynchronize(g->mark[1]));
    float f = 0;
    SMX_CUDA_TRY(cudaEventElapsedTime(&f, g->mark[0], g->mark[1]));
    *ms = f;
    return SMX_OK;
}

uint64_t smx_launch_count(void) { return launch_count(); }

// ------------------------------------------------------------------ graphs

int smx_graph_create(const uint64_t* offsets, const uint32_t* neighbors, const uint32_t* labels, uint32_t n,
                     uint64_t m2, int device, smx_graph** out) {
    if (!out || !offsets || (m2 && !neighbors)) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    int rc = check_device(device);
    if (rc != SMX_OK) return rc;
    if (offsets[0] != 0 || offsets[n] != m2) return fail(SMX_BAD_FORMAT, "offsets[0] must be 0 and offsets[n] the entry count");
    smx_graph* g = new (std::nothrow) smx_graph();
    if (!g) return fail(SMX_TOO_LARGE, "out of host memory");
    HostGraph& h = g->h;
    h.n = n;
    h.m2 = m2;
    h.off.assign(offsets, offsets + n + 1);
    h.adj.assign(neighbors, neighbors + m2);
    h.lab.assign(n, 0);
    if (labels) h.lab.assign(labels, labels + n);
    for (uint32_t v = 0; v < n; ++v) {
        if (h.off[v + 1] < h.off[v]) {
            delete g;
            return fail(SMX_BAD_FORMAT, "offsets decrease");
        }
        for (uint64_t e = h.off[v]; e < h.off[v + 1]; ++e) {
            if (h.adj[e] >= n || h.adj[e] == v) {
                delete g;
                return fail(SMX_BAD_FORMAT, "neighbour out of range or self loop");
            }
            if (e > h.off[v] && h.adj[e] <= h.adj[e - 1]) {
                delete g;
                return fail(SMX_BAD_FORMAT, "rows must be strictly ascending");
            }
        }
    }
    h.finish();
    return finish_graph(g, device, out);
}

int smx_graph_load_text(const char* path, int device, smx_graph** out) {
    if (!out || !path) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    int rc = check_device(device);
    if (rc != SMX_OK) return rc;
    smx_graph* g = new smx_graph();
    rc = parse_text_graph(path, g->h);
    if (rc != SMX_OK) {
        delete g;
        return rc;
    }
    return finish_graph(g, device, out);
}

int smx_graph_generate(uint32_t n, uint64_t m, double gamma, uint32_t num_labels, double zipf_s, uint64_t seed,
                       int device, smx_graph** out) {
    if (!out || n < 2 || gamma <= 1.0) return fail(SMX_BAD_ARGUMENT, "need n >= 2 and gamma > 1");
    *out = nullptr;
    int rc = check_device(device);
    if (rc != SMX_OK) return rc;
    smx_graph* g = new smx_graph();
    generate_chung_lu(n, m, gamma, num_labels, zipf_s, seed, g->h);
    return finish_graph(g, device, out);
}

int smx_graph_info(const smx_graph* g, uint32_t* n, uint64_t* m2, uint32_t* max_degree, uint32_t* label_count) {
    if (!g) return fail(SMX_BAD_ARGUMENT, "null graph");
    if (n) *n = g->h.n;
    if (m2) *m2 = g->h.m2;
    if (max_degree) *max_degree = g->h.max_deg;
    if (label_count) *label_count = g->h.label_cnt;
    return SMX_OK;
}

int smx_graph_export(const smx_graph* g, uint64_t* offsets, uint32_t* neighbors, uint32_t* labels) {
    if (!g) return fail(SMX_BAD_ARGUMENT, "null graph");
    if (offsets) std::memcpy(offsets, g->h.off.data(), (g->h.n + 1) * sizeof(uint64_t));
    if (neighbors && g->h.m2) std::memcpy(neighbors, g->h.adj.data(), g->h.m2 * sizeof(uint32_t));
    if (labels && g->h.n) std::memcpy(labels, g->h.lab.data(), g->h.n * sizeof(uint32_t));
    return SMX_OK;
}

int smx_graph_save_text(const smx_graph* g, const char* path) {
    if (!g || !path) return fail(SMX_BAD_ARGUMENT, "null argument");
    return write_text_graph(g->h, path);
}

void smx_graph_destroy(smx_graph* g) {
    if (!g) return;
    if (g->device < 0) {
        delete g;
        return;
    }
    cudaSetDevice(g->device);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (smx_cand* c : g->cands) {  // candidate sets still alive lose their device memory
        free_cand_device(c);
        c->g = nullptr;
    }
    cudaFree(g->d_off);
    cudaFree(g->d_adj);
    cudaFree(g->d_lab);
    cudaFree(g->d_hist);
    cudaFree(g->d_hub_id);
    cudaFree(g->d_hub_bits);
    cudaFree(g->d_scratch);
    for (auto& e : g->mark)
        if (e) cudaEventDestroy(e);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

// ------------------------------------------------------------------ queries

int smx_query_create(const uint32_t* offsets, const uint32_t* neighbors, const uint32_t* labels, uint32_t n,
                     smx_query** out) {
    if (!out || !offsets) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    if (n == 0) return fail(SMX_BAD_ARGUMENT, "empty query");
    if (n > kMaxQ) return fail(SMX_TOO_LARGE, "query has more than SMX_MAX_QUERY_VERTEX vertices");
    if (offsets[0] != 0) return fail(SMX_BAD_FORMAT, "offsets[0] must be 0");
    if (offsets[n] && !neighbors) return fail(SMX_BAD_ARGUMENT, "null neighbours");
    if (offsets[n] % 2) return fail(SMX_BAD_FORMAT, "odd number of adjacency entries");
    smx_query* q = new smx_query();
    HostQuery& h = q->h;
    h.n = n;
    h.off.assign(offsets, offsets + n + 1);
    h.adj.assign(neighbors, neighbors + offsets[n]);
    h.lab.assign(n, 0);
    if (labels) h.lab.assign(labels, labels + n);
    for (uint32_t u = 0; u < n; ++u) {
        if (h.off[u + 1] < h.off[u]) {
            delete q;
            return fail(SMX_BAD_FORMAT, "offsets decrease");
        }
        for (uint32_t e = h.off[u]; e < h.off[u + 1]; ++e) {
            if (h.adj[e] >= n || h.adj[e] == u) {
                delete q;
                return fail(SMX_BAD_FORMAT, "neighbour out of range or self loop");
            }
            if (e > h.off[u] && h.adj[e] <= h.adj[e - 1]) {
                delete q;
                return fail(SMX_BAD_FORMAT, "rows must be strictly ascending");
            }
        }
    }
    h.finish();
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t e = h.off[u]; e < h.off[u + 1]; ++e)
            if (!h.has_edge(h.adj[e], u)) {
                delete q;
                return fail(SMX_BAD_FORMAT, "adjacency is not symmetric");
            }
    kcore(h, q->core);
    *out = q;
    return SMX_OK;
}

int smx_query_load_text(const char* path, smx_query** out) {
    if (!out || !path) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    HostGraph g;
    int rc = parse_text_graph(path, g);
    if (rc != SMX_OK) return rc;
    if (g.n == 0) return fail(SMX_BAD_ARGUMENT, "empty query");
    if (g.n > kMaxQ) return fail(SMX_TOO_LARGE, "query has more than SMX_MAX_QUERY_VERTEX vertices");
    smx_query* q = new smx_query();
    query_from_host_graph(g, q->h);
    kcore(q->h, q->core);
    *out = q;
    return SMX_OK;
}

int smx_query_generate(const smx_graph* g, uint32_t k, int dense, uint64_t seed, smx_query** out) {
    if (!g || !out) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    if (k == 0 || k > kMaxQ) return fail(SMX_TOO_LARGE, "query size must be in [1, SMX_MAX_QUERY_VERTEX]");
    smx_query* q = new smx_query();
    if (!generate_walk_query(g->h, k, dense != 0, seed, q->h)) {
        delete q;
        return fail(SMX_BAD_ARGUMENT, "random walk could not reach the requested number of vertices");
    }
    kcore(q->h, q->core);
    *out = q;
    return SMX_OK;
}

int smx_query_info(const smx_query* q, uint32_t* n, uint32_t* m, uint32_t* max_degree) {
    if (!q) return fail(SMX_BAD_ARGUMENT, "null query");
    if (n) *n = q->h.n;
    if (m) *m = q->h.m;
    if (max_degree) *max_degree = q->h.max_deg;
    return SMX_OK;
}

int smx_query_export(const smx_query* q, uint32_t* offsets, uint32_t* neighbors, uint32_t* labels) {
    if (!q) return fail(SMX_BAD_ARGUMENT, "null query");
    if (offsets) std::memcpy(offsets, q->h.off.data(), (q->h.n + 1) * sizeof(uint32_t));
    if (neighbors && q->h.off[q->h.n]) std::memcpy(neighbors, q->h.adj.data(), q->h.off[q->h.n] * sizeof(uint32_t));
    if (labels) std::memcpy(labels, q->h.lab.data(), q->h.n * sizeof(uint32_t));
    return SMX_OK;
}

int smx_query_kcore(const smx_query* q, uint32_t* core) {
    if (!q || !core) return fail(SMX_BAD_ARGUMENT, "null argument");
    std::copy(q->core.begin(), q->core.end(), core);
    return SMX_OK;
}

int smx_query_save_text(const smx_query* q, const char* path) {
    if (!q || !path) return fail(SMX_BAD_ARGUMENT, "null argument");
    HostGraph g;
    g.n = q->h.n;
    g.m2 = q->h.off[q->h.n];
    g.off.assign(q->h.off.begin(), q->h.off.end());
    g.adj.assign(q->h.adj.begin(), q->h.adj.end());
    g.lab.assign(q->h.lab.begin(), q->h.lab.end());
    return write_text_graph(g, path);
}

void smx_query_destroy(smx_query* q) { delete q; }

// ------------------------------------------------------------------ orders

int smx_order_ri(const smx_query* q, uint32_t* order) {
    if (!q || !order) return fail(SMX_BAD_ARGUMENT, "null argument");
    order_ri(q->h, order);
    return SMX_OK;
}

int smx_order_gql(const smx_query* q, const smx_cand* c, uint32_t* order) {
    if (!q || !c || !order) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (c->qn != q->h.n) return fail(SMX_BAD_ARGUMENT, "candidates belong to another query");
    if (!c->g) return fail(SMX_BAD_ARGUMENT, "the candidate set's data graph was destroyed");
    order_gql(q->h, c->cnt.data(), c->g->h.n, order);
    return SMX_OK;
}

int smx_order_features(const smx_query* q, const smx_cand* c, const uint32_t* order, float* out) {
    if (!q || !c || !order || !out) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (c->qn != q->h.n) return fail(SMX_BAD_ARGUMENT, "candidates belong to another query");
    if (!order_valid(q->h, order)) return fail(SMX_INVALID_ORDER, "order is not a connected permutation of the query vertices");
    order_features(q->h, c->cnt.data(), order, out);
    return SMX_OK;
}

int smx_order_beam(const smx_query* q, const smx_cand* c, uint32_t beam, uint64_t seed, uint32_t* orders,
                   uint32_t* produced) {
    if (!q || !c || !orders || !produced) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (c->qn != q->h.n) return fail(SMX_BAD_ARGUMENT, "candidates belong to another query");
    if (!c->g) return fail(SMX_BAD_ARGUMENT, "the candidate set's data graph was destroyed");
    std::vector<std::vector<uint32_t>> out;
    order_beam(q->h, c->cnt.data(), c->g->h.n, beam, seed, out);
    for (size_t i = 0; i < out.size(); ++i) std::copy(out[i].begin(), out[i].end(), orders + i * q->h.n);
    *produced = (uint32_t)out.size();
    return SMX_OK;
}

int smx_order_learned(smx_mlp* m, const smx_query* q, const smx_cand* c, uint32_t beam, uint64_t seed,
                      uint32_t* order, float* predicted) {
    if (!m || !q || !c || !order) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (beam == 0) return fail(SMX_BAD_ARGUMENT, "beam must be at least 1");
    const uint32_t n = q->h.n;
    std::vector<uint32_t> orders((size_t)beam * n);
    uint32_t k = 0;
    int rc = smx_order_beam(q, c, beam, seed, orders.data(), &k);
    if (rc != SMX_OK) return rc;
    std::vector<float> x((size_t)k * SMX_MLP_INPUTS), y(k);
    for (uint32_t i = 0; i < k; ++i) order_features(q->h, c->cnt.data(), orders.data() + (size_t)i * n, x.data() + (size_t)i * SMX_MLP_INPUTS);
    rc = smx_mlp_forward(m, x.data(), k, y.data());
    if (rc != SMX_OK) return rc;
    uint32_t best = 0;
    for (uint32_t i = 1; i < k; ++i)
        if (y[i] < y[best]) best = i;
    std::copy(orders.begin() + (size_t)best * n, orders.begin() + (size_t)(best + 1) * n, order);
    if (predicted) *predicted = y[best];
    return SMX_OK;
}

int smx_order_valid(const smx_query* q, const uint32_t* order) {
    if (!q || !order) return 0;
    return order_valid(q->h, order) ? 1 : 0;
}

// ------------------------------------------------------------------ filtering

int smx_filter(smx_graph* g, const smx_query* q, int kind, int build_tables, smx_cand** out) {
    if (!g || !q || !out) return fail(SMX_BAD_ARGUMENT, "null argument");
    *out = nullptr;
    if (g->device < 0) return fail(SMX_NO_DEVICE, "graph was created host-only (device < 0)");
    if (kind != SMX_FILTER_NLF && kind != SMX_FILTER_GQL) return fail(SMX_BAD_ARGUMENT, "unknown filter kind");
    smx_cand* c = new smx_cand();
    int rc = device_filter(g, q->h, kind, build_tables, c);
    if (rc != SMX_OK && rc != SMX_EMPTY_CANDIDATES) {
        free_cand_device(c);
        delete c;
        return rc;
    }
    if (rc == SMX_EMPTY_CANDIDATES) set_error("a query vertex has no candidates");
    g->cands.push_back(c);
    *out = c;
    return rc;
}

int smx_cand_counts(const smx_cand* c, uint32_t* counts) {
    if (!c || !counts) return fail(SMX_BAD_ARGUMENT, "null argument");
    for (uint32_t u = 0; u < c->qn; ++u) counts[u] = u < c->cnt.size() ? c->cnt[u] : 0;
    return SMX_OK;
}

int smx_cand_export(const smx_cand* c, uint32_t u, uint32_t* out) {
    if (!c || !out) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (u >= c->qn) return fail(SMX_BAD_ARGUMENT, "query vertex out of range");
    if (!c->g) return fail(SMX_BAD_ARGUMENT, "the candidate set's data graph was destroyed");
    if (u >= c->cnt.size() || c->cnt[u] == 0 || !c->d_cand) return SMX_OK;
    cudaSetDevice(c->g->device);
    SMX_CUDA_TRY(cudaMemcpy(out, c->cand_ptr(u), c->cnt[u] * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return SMX_OK;
}

int smx_table_info(const smx_cand* c, uint32_t a, uint32_t b, uint32_t* v_cnt, uint32_t* e_cnt, uint32_t* max_degree) {
    if (!c) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (!c->g) return fail(SMX_BAD_ARGUMENT, "the candidate set's data graph was destroyed");
    if (a >= c->qn || b >= c->qn || c->tab_index[a][b] < 0) return fail(SMX_BAD_ARGUMENT, "no table for this pair");
    const DevTable& t = c->tables[c->tab_index[a][b]];
    if (v_cnt) *v_cnt = t.v_cnt;
    if (e_cnt) *e_cnt = (uint32_t)t.e_cnt;
    if (max_degree) *max_degree = t.max_deg;
    return SMX_OK;
}

int smx_table_export(const smx_cand* c, uint32_t a, uint32_t b, uint32_t* offsets, uint32_t* edge, uint32_t* edge_v) {
    if (!c) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (a >= c->qn || b >= c->qn || c->tab_index[a][b] < 0) return fail(SMX_BAD_ARGUMENT, "no table for this pair");
    if (!c->g) return fail(SMX_BAD_ARGUMENT, "the candidate set's data graph was destroyed");
    const DevTable& t = c->tables[c->tab_index[a][b]];
    cudaSetDevice(c->g->device);
    if (offsets) SMX_CUDA_TRY(cudaMemcpy(offsets, t.d_off, (t.v_cnt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> e(t.e_cnt);
    if (t.e_cnt) SMX_CUDA_TRY(cudaMemcpy(e.data(), t.d_edge, t.e_cnt * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (edge) std::copy(e.begin(), e.end(), edge);
    if (edge_v && t.e_cnt) {
        std::vector<uint32_t> cb(c->cnt[b]);
        SMX_CUDA_TRY(cudaMemcpy(cb.data(), c->cand_ptr(b), cb.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < t.e_cnt; ++i) edge_v[i] = cb[e[i]];
    }
    return SMX_OK;
}

int smx_cand_timing(const smx_cand* c, double* ms4) {
    if (!c || !ms4) return fail(SMX_BAD_ARGUMENT, "null argument");
    for (int i = 0; i < 4; ++i) ms4[i] = c->ms[i];
    return SMX_OK;
}

void smx_cand_destroy(smx_cand* c) {
    if (!c) return;
    if (c->g) {
        auto& v = c->g->cands;
        v.erase(std::remove(v.begin(), v.end(), c), v.end());
    }
    free_cand_device(c);
    delete c;
}

// ------------------------------------------------------------------ enumeration

void smx_enum_opts_default(smx_enum_opts* o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->explore = SMX_EXPLORE_CANDIDATES;
    o->warps_per_block = 8;
    o->blocks_per_sm = 0;
    o->task_grab = 4;
    o->stage_chunk = 1024;
    o->gallop_ratio = 16;
    o->bitmap_min = 0;
    o->use_tma = 1;
    o->failing_sets = 1;
    o->lane_depth = 0;
    o->time_budget_ms = 0;
}

int smx_enumerate(smx_graph* g, const smx_query* q, const smx_cand* c, const uint32_t* order,
                  const smx_enum_opts* opts, uint64_t limit, volatile uint32_t* stop, smx_stats* out) {
    if (!g || !q || !c) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (c->qn != q->h.n || c->g != g) return fail(SMX_BAD_ARGUMENT, "candidates belong to another query or graph");
    if (out) std::memset(out, 0, sizeof(*out));
    if (!c->ok) return fail(SMX_EMPTY_CANDIDATES, "candidate sets are empty");
    smx_enum_opts o;
    if (opts) o = *opts; else smx_enum_opts_default(&o);
    if (o.explore != SMX_EXPLORE_CANDIDATES && o.explore != SMX_EXPLORE_CACHE_DAF)
        return fail(SMX_BAD_ARGUMENT, "unknown explore kind");
    std::vector<uint32_t> ord(q->h.n);
    if (order) std::copy(order, order + q->h.n, ord.begin());
    else order_ri(q->h, ord.data());
    if (!order_valid(q->h, ord.data())) return fail(SMX_INVALID_ORDER, "order is not a connected permutation of the query vertices");
    if (q->h.n == 1) {
        const uint64_t raw = c->cnt[ord[0]];
        if (out) {
            out->count = limit && raw > limit ? limit : raw;
            out->raw_count = raw;
            out->limit_reached = limit && raw >= limit;
        }
        return SMX_OK;
    }
    std::vector<const HostQuery*> qs{&q->h};
    std::vector<const smx_cand*> cs{c};
    std::vector<const uint32_t*> os{ord.data()};
    std::vector<uint64_t> lim{limit};
    uint64_t count = 0;
    return device_enumerate(g, qs, cs, os, o, lim, stop, &count, out, false);
}

int smx_enumerate_noalloc(smx_graph* g, const smx_query* q, const smx_cand* c, const uint32_t* order,
                          const smx_enum_opts* opts, uint64_t limit, volatile uint32_t* stop, smx_stats* out) {
    if (!g || !q || !c) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (c->qn != q->h.n || c->g != g) return fail(SMX_BAD_ARGUMENT, "candidates belong to another query or graph");
    if (out) std::memset(out, 0, sizeof(*out));
    if (!c->ok) return fail(SMX_EMPTY_CANDIDATES, "candidate sets are empty");
    smx_enum_opts o;
    if (opts) o = *opts; else smx_enum_opts_default(&o);
    if (o.explore != SMX_EXPLORE_CANDIDATES && o.explore != SMX_EXPLORE_CACHE_DAF)
        return fail(SMX_BAD_ARGUMENT, "unknown explore kind");
    std::vector<uint32_t> ord(q->h.n);
    if (order) std::copy(order, order + q->h.n, ord.begin());
    else order_ri(q->h, ord.data());
    if (!order_valid(q->h, ord.data())) return fail(SMX_INVALID_ORDER, "order is not a connected permutation of the query vertices");
    if (q->h.n == 1) {
        const uint64_t raw = c->cnt[ord[0]];
        if (out) {
            out->count = limit && raw > limit ? limit : raw;
            out->raw_count = raw;
            out->limit_reached = limit && raw >= limit;
        }
        return SMX_OK;
    }
    return device_enumerate_noalloc(g, q->h, c, ord.data(), o, limit, stop, out);
}

int smx_stop_flag_create(int device, volatile uint32_t** flag) {
    if (!flag) return fail(SMX_BAD_ARGUMENT, "null argument");
    *flag = nullptr;
    int rc = check_device(device);
    if (rc != SMX_OK) return rc;
    if (device < 0) return fail(SMX_BAD_ARGUMENT, "a stop word needs a device");
    SMX_CUDA_TRY(cudaSetDevice(device));
    void* p = nullptr;
    SMX_CUDA_TRY(cudaHostAlloc(&p, 64, cudaHostAllocMapped | cudaHostAllocPortable));
    std::memset(p, 0, 64);
    *flag = static_cast<volatile uint32_t*>(p);
    return SMX_OK;
}

void smx_stop_flag_destroy(volatile uint32_t* flag) {
    if (flag) cudaFreeHost((void*)flag);
}

int smx_enumerate_batch(smx_graph* g, const smx_query* const* qs, const smx_cand* const* cs,
                        const uint32_t* const* orders, uint32_t nq, const smx_enum_opts* opts, uint64_t limit,
                        uint64_t* counts, smx_stats* out, int32_t* query_status) {
    if (!g || (nq && (!qs || !cs))) return fail(SMX_BAD_ARGUMENT, "null argument");
    if (out) std::memset(out, 0, sizeof(*out));
    if (query_status)
        for (uint32_t i = 0; i < nq; ++i) query_status[i] = SMX_OK;
    smx_enum_opts o;
    if (opts) o = *opts; else smx_enum_opts_default(&o);
    std::vector<std::vector<uint32_t>> ords(nq);
    std::vector<const HostQuery*> hq;
    std::vector<const smx_cand*> hc;
    std::vector<const uint32_t*> ho;
    std::vector<uint64_t> lim;
    std::vector<uint32_t> slot;
    for (uint32_t i = 0; i < nq; ++i) {
        if (counts) counts[i] = 0;
        const smx_query* q = qs[i];
        const smx_cand* c = cs[i];
        if (!q || !c || c->qn != q->h.n || c->g != g) return fail(SMX_BAD_ARGUMENT, "query / candidates mismatch in batch");
        if (!c->ok) continue;  // empty candidate sets: zero embeddings
        ords[i].resize(q->h.n);
        if (orders && orders[i]) std::copy(orders[i], orders[i] + q->h.n, ords[i].begin());
        else order_ri(q->h, ords[i].data());
        if (!order_valid(q->h, ords[i].data())) return fail(SMX_INVALID_ORDER, "batch order is not connected");
        if (q->h.n == 1) {
            uint64_t k = c->cnt[ords[i][0]];
            if (counts) counts[i] = limit && k > limit ? limit : k;
            continue;
        }
        hq.push_back(&q->h);
        hc.push_back(c);
        ho.push_back(ords[i].data());
        lim.push_back(limit);
        slot.push_back(i);
    }
    if (hq.empty()) return SMX_OK;
    std::vector<uint64_t> cnt(hq.size(), 0);
    std::vector<int32_t> qst(hq.size(), SMX_OK);
    int rc = device_enumerate(g, hq, hc, ho, o, lim, nullptr, cnt.data(), out, true, qst.data());
    for (size_t i = 0; i < slot.size(); ++i) {
        if (counts) counts[slot[i]] = cnt[i];
        if (query_status) query_status[slot[i]] = qst[i];
    }
    return rc;
}

}  // extern "C"
