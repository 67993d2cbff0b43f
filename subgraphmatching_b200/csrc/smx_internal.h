// Internal declarations shared by the host (C++) and device (CUDA) parts of
// libsmx.  Nothing here is part of the C ABI (include/smx.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "smx.h"

namespace smx {

constexpr uint32_t kMaxQ = SMX_MAX_QUERY_VERTEX;
constexpr uint32_t kInvalid = 0xffffffffu;

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
const std::string& last_error();
int fail(int status, const std::string& msg);
#define SMX_CUDA_TRY(expr)                                                                 \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return ::smx::fail(SMX_CUDA_ERROR, std::string(#expr ": ") + cudaGetErrorString(e_)); \
    } while (0)

// ------------------------------------------------------------------ host graphs
// Data graph in host memory: CSR with 64-bit offsets, rows sorted ascending.
struct HostGraph {
    uint32_t n = 0;
    uint64_t m2 = 0;  // directed entries (2 * undirected edges)
    uint32_t max_deg = 0;
    uint32_t label_cnt = 0;       // max(#distinct labels, max label + 1), graph.h:253
    uint32_t max_label_freq = 0;  // graph.h:255-256
    std::vector<uint64_t> off;
    std::vector<uint32_t> adj;
    std::vector<uint32_t> lab;
    uint32_t deg(uint32_t v) const { return (uint32_t)(off[v + 1] - off[v]); }
    void finish();  // label count, max degree, max label frequency
};

// Query graph: at most kMaxQ vertices, 32-bit CSR, adjacency bit masks.
struct HostQuery {
    uint32_t n = 0;
    uint32_t m = 0;  // undirected edges
    uint32_t max_deg = 0;
    std::vector<uint32_t> off, adj, lab;
    uint64_t nbr_mask[kMaxQ] = {0};
    uint32_t deg(uint32_t u) const { return off[u + 1] - off[u]; }
    bool has_edge(uint32_t a, uint32_t b) const { return (nbr_mask[a] >> b) & 1ull; }
    void finish();
};

int parse_text_graph(const char* path, HostGraph& g);  // graph.h:190-266 format
int write_text_graph(const HostGraph& g, const char* path);
void generate_chung_lu(uint32_t n, uint64_t m, double gamma, uint32_t num_labels, double zipf_s,
                       uint64_t seed, HostGraph& g);
bool generate_walk_query(const HostGraph& g, uint32_t k, bool dense, uint64_t seed, HostQuery& q);
void query_from_host_graph(const HostGraph& g, HostQuery& q);
void kcore(const HostQuery& q, std::vector<uint32_t>& core);
void order_ri(const HostQuery& q, uint32_t* order);
void order_gql(const HostQuery& q, const uint32_t* cand_counts, uint32_t data_n, uint32_t* order);
bool order_valid(const HostQuery& q, const uint32_t* order);
void order_features(const HostQuery& q, const uint32_t* cnt, const uint32_t* order, float* out);
void order_beam(const HostQuery& q, const uint32_t* cnt, uint32_t data_n, uint32_t beam, uint64_t seed,
                std::vector<std::vector<uint32_t>>& out);

// PlanIR (code_gen.h:682-847): deduplicated prefix-intersection ops.
struct PlanOp {
    uint32_t depth;       // depth at which the op is computed (its last prefix element)
    uint32_t vdepth;      // depth of the query vertex the op was created for
    uint32_t label;
    uint32_t parent;      // parent op id (prefix minus last element) or kInvalid
    std::vector<uint32_t> edges;  // prefix depths, ascending
};
struct Plan {
    std::vector<PlanOp> ops;
    std::vector<std::vector<uint32_t>> ops_at;  // ops computed at each depth
    std::vector<uint32_t> iter_op;              // op whose result is depth d's candidate set
};
bool build_plan(const HostQuery& q, const uint32_t* order, Plan& plan);

// ------------------------------------------------------------------ device handles
struct DevTable {
    uint32_t a = 0, b = 0;
    uint32_t v_cnt = 0;
    uint64_t e_cnt = 0;
    uint32_t max_deg = 0;
    uint32_t* d_off = nullptr;   // v_cnt + 1
    uint32_t* d_edge = nullptr;  // e_cnt (+8 padding), candidate indices into C(b)
};

}  // namespace smx

struct smx_graph {
    smx::HostGraph h;
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    uint64_t* d_off = nullptr;   // n + 1
    uint32_t* d_adj = nullptr;   // m2 (+ padding so 16-byte rounded reads stay inside)
    uint32_t* d_lab = nullptr;   // n
    uint8_t* d_hist = nullptr;   // n * hist_stride neighbour-label counts (saturating), labelled graphs only
    uint32_t hist_stride = 0;
    // hub adjacency: the (up to) 16,384 highest-degree vertices (degree >= 16)
    // get ids; bit (i, j) of a hub_words-per-row matrix says hubs i and j
    // are adjacent (32 MB at most, kept in L2 by the enumerator's probes)
    uint32_t* d_hub_id = nullptr;    // n: hub id or 0xffffffff
    uint32_t* d_hub_bits = nullptr;  // hubs * hub_words
    uint32_t hubs = 0, hub_words = 0;
    // scratch reused across calls
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaEvent_t mark[2] = {nullptr, nullptr};
    // candidate sets built on this graph: destroying the graph frees their
    // device memory and detaches them (their handles stay valid to destroy)
    std::vector<smx_cand*> cands;
};

struct smx_cand;

struct smx_query {
    smx::HostQuery h;
    std::vector<uint32_t> core;
};

struct smx_cand {
    smx_graph* g = nullptr;  // null once the graph was destroyed
    uint32_t qn = 0;
    int kind = 0;
    int ok = 0;
    uint64_t* d_mask = nullptr;   // per data vertex: bit u set iff v in C(u)
    uint2* d_rank = nullptr;      // [n/32 blocks][qn]: {bits of block, prefix count}
    uint32_t* d_cand = nullptr;   // concatenated candidate lists
    std::vector<uint64_t> cand_off;  // qn + 1
    std::vector<uint32_t> cnt;
    std::vector<smx::DevTable> tables;
    uint32_t* d_table_off = nullptr;  // offsets of all tables (one allocation)
    int tab_index[smx::kMaxQ][smx::kMaxQ];
    double ms[4] = {0, 0, 0, 0};
    const uint32_t* cand_ptr(uint32_t u) const { return d_cand + cand_off[u]; }
};

namespace smx {
int upload_graph(smx_graph* g);
void free_cand_device(smx_cand* c);
int device_filter(smx_graph* g, const HostQuery& q, int kind, int build_tables, smx_cand* c);
int device_enumerate(smx_graph* g, const std::vector<const HostQuery*>& qs, const std::vector<const smx_cand*>& cs,
                     const std::vector<const uint32_t*>& orders, const smx_enum_opts& o,
                     const std::vector<uint64_t>& limits, volatile uint32_t* stop, uint64_t* counts,
                     smx_stats* st, bool use_graph, int32_t* qstatus = nullptr);
int ensure_scratch(smx_graph* g, size_t bytes);
// smx_enumerate_noalloc: one query, all working memory in a file-scope device array
int device_enumerate_noalloc(smx_graph* g, const HostQuery& q, const smx_cand* c, const uint32_t* order,
                             const smx_enum_opts& o, uint64_t limit, volatile uint32_t* stop, smx_stats* st);
}  // namespace smx
