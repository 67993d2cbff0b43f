// Host-side components of libsmx: text I/O, seeded generators, query
// utilities, the static orders and the intersection plan.  Device code lives
// in filter.cu / enumerate.cu; the C ABI in capi.cpp.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "smx_internal.h"

namespace smx {

namespace {
thread_local std::string g_last_error;

// splitmix64: small, portable, seedable generator (identical on every host).
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

// Walker alias table for O(1) sampling proportional to weights.
struct Alias {
    std::vector<double> prob;
    std::vector<uint32_t> alias;
    explicit Alias(const std::vector<double>& w) {
        size_t n = w.size();
        prob.resize(n);
        alias.resize(n);
        double sum = 0;
        for (double x : w) sum += x;
        std::vector<double> p(n);
        std::vector<uint32_t> small, large;
        for (size_t i = 0; i < n; ++i) {
            p[i] = w[i] * n / sum;
            (p[i] < 1.0 ? small : large).push_back((uint32_t)i);
        }
        while (!small.empty() && !large.empty()) {
            uint32_t s = small.back();
            small.pop_back();
            uint32_t l = large.back();
            prob[s] = p[s];
            alias[s] = l;
            p[l] = (p[l] + p[s]) - 1.0;
            if (p[l] < 1.0) {
                large.pop_back();
                small.push_back(l);
            }
        }
        for (uint32_t i : large) { prob[i] = 1.0; alias[i] = i; }
        for (uint32_t i : small) { prob[i] = 1.0; alias[i] = i; }
    }
    uint32_t sample(Rng& r) const {
        uint32_t i = (uint32_t)r.below(prob.size());
        return r.uniform() < prob[i] ? i : alias[i];
    }
};
}  // namespace

namespace {
std::atomic<uint64_t> g_launches{0};
}
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(); }

void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& last_error() { return g_last_error; }
int fail(int status, const std::string& msg) {
    g_last_error = msg;
    return status;
}

// ------------------------------------------------------------------ graphs

void HostGraph::finish() {
    max_deg = 0;
    for (uint32_t v = 0; v < n; ++v) max_deg = std::max(max_deg, deg(v));
    uint32_t maxl = 0;
    for (uint32_t v = 0; v < n; ++v) maxl = std::max(maxl, lab[v]);
    std::vector<uint32_t> freq(n ? (size_t)maxl + 1 : 0, 0);
    for (uint32_t v = 0; v < n; ++v) freq[lab[v]]++;
    uint32_t distinct = 0;
    max_label_freq = 0;
    for (uint32_t f : freq) {
        if (f) distinct++;
        max_label_freq = std::max(max_label_freq, f);
    }
    label_cnt = n ? std::max(distinct, maxl + 1) : 0;
}

void HostQuery::finish() {
    m = off[n] / 2;
    max_deg = 0;
    for (uint32_t u = 0; u < kMaxQ; ++u) nbr_mask[u] = 0;
    for (uint32_t u = 0; u < n; ++u) {
        max_deg = std::max(max_deg, deg(u));
        for (uint32_t e = off[u]; e < off[u + 1]; ++e) nbr_mask[u] |= 1ull << adj[e];
    }
}

namespace {
// Minimal fast tokenizer over a whole file in memory.
struct Scanner {
    const char* p;
    const char* e;
    bool skip_ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
        return p < e;
    }
    bool ch(char& c) {
        if (!skip_ws()) return false;
        c = *p++;
        return true;
    }
    bool num(uint64_t& x) {
        if (!skip_ws()) return false;
        if (*p < '0' || *p > '9') return false;
        x = 0;
        while (p < e && *p >= '0' && *p <= '9') x = x * 10 + (uint64_t)(*p++ - '0');
        return true;
    }
};
}  // namespace

// Graph::Load (graph.h:190-266).  Unlike the reference, which trusts the
// degree field of each "v" line to lay out the rows, the degrees are checked
// against the edges and a mismatch is an error (SMX_BAD_FORMAT) instead of a
// silently corrupt CSR.  Duplicate edges and self loops are errors too.
int parse_text_graph(const char* path, HostGraph& g) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(SMX_IO_ERROR, std::string("cannot open ") + path);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string buf((size_t)std::max(sz, 0L), '\0');
    size_t got = sz > 0 ? std::fread(&buf[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    if ((long)got != sz) return fail(SMX_IO_ERROR, std::string("short read on ") + path);
    Scanner s{buf.data(), buf.data() + buf.size()};
    char c;
    uint64_t n, m;
    if (!s.ch(c) || c != 't' || !s.num(n) || !s.num(m)) return fail(SMX_BAD_FORMAT, "missing 't N M' header");
    if (n > 0xfffffffeull) return fail(SMX_TOO_LARGE, "more than 2^32-2 vertices");
    g.n = (uint32_t)n;
    g.m2 = 2 * m;
    g.off.assign(n + 1, 0);
    g.lab.assign(n, 0);
    g.adj.assign(2 * m, 0);
    std::vector<uint64_t> decl(n, 0);
    std::vector<uint64_t> fill(n, 0);
    std::vector<uint8_t> seen(n, 0);
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    edges.reserve(m);
    while (s.ch(c)) {
        if (c == 'v') {
            uint64_t id, l, d;
            if (!s.num(id) || !s.num(l) || !s.num(d)) return fail(SMX_BAD_FORMAT, "bad 'v' line");
            if (id >= n) return fail(SMX_BAD_FORMAT, "vertex id out of range");
            g.lab[id] = (uint32_t)l;
            decl[id] = d;
            seen[id] = 1;
        } else if (c == 'e') {
            uint64_t a, b;
            if (!s.num(a) || !s.num(b)) return fail(SMX_BAD_FORMAT, "bad 'e' line");
            if (a >= n || b >= n) return fail(SMX_BAD_FORMAT, "edge endpoint out of range");
            if (a == b) return fail(SMX_BAD_FORMAT, "self loop");
            edges.emplace_back((uint32_t)a, (uint32_t)b);
        } else {
            return fail(SMX_BAD_FORMAT, std::string("unexpected record '") + c + "'");
        }
    }
    if (edges.size() != m) return fail(SMX_BAD_FORMAT, "edge count differs from header");
    std::vector<uint64_t> deg(n, 0);
    for (auto& e : edges) { deg[e.first]++; deg[e.second]++; }
    for (uint64_t v = 0; v < n; ++v) {
        if (seen[v] && decl[v] != deg[v])
            return fail(SMX_BAD_FORMAT, "declared degree differs from edges at vertex " + std::to_string(v));
        g.off[v + 1] = g.off[v] + deg[v];
    }
    for (auto& e : edges) {
        g.adj[g.off[e.first] + fill[e.first]++] = e.second;
        g.adj[g.off[e.second] + fill[e.second]++] = e.first;
    }
    for (uint32_t v = 0; v < g.n; ++v) {
        std::sort(g.adj.begin() + g.off[v], g.adj.begin() + g.off[v + 1]);
        for (uint64_t i = g.off[v] + 1; i < g.off[v + 1]; ++i)
            if (g.adj[i] == g.adj[i - 1]) return fail(SMX_BAD_FORMAT, "duplicate edge at vertex " + std::to_string(v));
    }
    g.finish();
    return SMX_OK;
}

int write_text_graph(const HostGraph& g, const char* path) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return fail(SMX_IO_ERROR, std::string("cannot write ") + path);
    std::string out;
    out.reserve(1 << 20);
    auto flush = [&]() {
        std::fwrite(out.data(), 1, out.size(), f);
        out.clear();
    };
    out += "t " + std::to_string(g.n) + " " + std::to_string(g.m2 / 2) + "\n";
    char line[96];
    for (uint32_t v = 0; v < g.n; ++v) {
        int k = std::snprintf(line, sizeof line, "v %u %u %u\n", v, g.lab[v], g.deg(v));
        out.append(line, k);
        if (out.size() > (1 << 20)) flush();
    }
    for (uint32_t v = 0; v < g.n; ++v)
        for (uint64_t e = g.off[v]; e < g.off[v + 1]; ++e)
            if (g.adj[e] > v) {
                int k = std::snprintf(line, sizeof line, "e %u %u\n", v, g.adj[e]);
                out.append(line, k);
                if (out.size() > (1 << 20)) flush();
            }
    flush();
    std::fclose(f);
    return SMX_OK;
}

// Chung-Lu graph with an exact edge count.  Expected degrees follow
// w_i = (i + i0)^(-1/(gamma-1)) scaled to sum to 2m, with i0 chosen so the
// largest expected degree equals the structural cutoff sqrt(2m) (which keeps
// w_i w_j / 2m <= 1, the Chung-Lu condition; on 9,500 vertices / 35,000 edges
// it gives a largest degree near 255, the scale of the reference's bundled
// hprd graph's 247).  Endpoints are drawn in proportion to w (alias table);
// self loops and repeats are redrawn until m distinct edges exist.  Vertex ids
// are then permuted by a seeded shuffle so hubs are spread over the id range.
// Labels (if num_labels > 1) are drawn Zipf(zipf_s) over [0, num_labels).
void generate_chung_lu(uint32_t n, uint64_t m, double gamma, uint32_t num_labels, double zipf_s,
                       uint64_t seed, HostGraph& g) {
    Rng rng(seed);
    const double a = 1.0 / (gamma - 1.0);
    const double target_max = std::sqrt(2.0 * (double)m);
    // sum_{i<n} (i + i0)^-a: exact head, midpoint-rule tail (relative error < 1e-9)
    auto weight_sum = [&](double i0) {
        const uint32_t head = std::min<uint32_t>(n, 4096);
        double sum = 0;
        for (uint32_t i = 0; i < head; ++i) sum += std::pow(i + i0, -a);
        if (n > head) {
            const double lo = head + i0 - 0.5, hi = n + i0 - 0.5;
            sum += (std::pow(hi, 1.0 - a) - std::pow(lo, 1.0 - a)) / (1.0 - a);
        }
        return sum;
    };
    auto max_expected = [&](double i0) { return 2.0 * (double)m * std::pow(i0, -a) / weight_sum(i0); };
    double lo = 1.0, hi = 1.0;
    if (max_expected(1.0) > target_max) {
        hi = 2.0;
        while (max_expected(hi) > target_max && hi < 1e12) hi *= 2.0;
        for (int it = 0; it < 60; ++it) {
            double mid = 0.5 * (lo + hi);
            if (max_expected(mid) > target_max) lo = mid; else hi = mid;
        }
    }
    const double i0 = hi;
    std::vector<double> w(n);
    for (uint32_t i = 0; i < n; ++i) w[i] = std::pow(i + i0, -a);
    Alias alias(w);
    const uint64_t max_pairs = (uint64_t)n * (n - 1) / 2;
    if (m > max_pairs) m = max_pairs;
    // open-addressing set of undirected edges
    uint64_t cap = 1;
    while (cap < 2 * m + 16) cap <<= 1;
    std::vector<uint64_t> table(cap, ~0ull);
    std::vector<std::pair<uint32_t, uint32_t>> edges;
    edges.reserve(m);
    while (edges.size() < m) {
        uint32_t x = alias.sample(rng), y = alias.sample(rng);
        if (x == y) continue;
        if (x > y) std::swap(x, y);
        uint64_t key = ((uint64_t)x << 32) | y;
        uint64_t h = (key * 0x9E3779B97F4A7C15ull) & (cap - 1);
        bool dup = false;
        while (table[h] != ~0ull) {
            if (table[h] == key) { dup = true; break; }
            h = (h + 1) & (cap - 1);
        }
        if (dup) continue;
        table[h] = key;
        edges.emplace_back(x, y);
    }
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    for (uint32_t i = n; i > 1; --i) std::swap(perm[i - 1], perm[rng.below(i)]);
    g.n = n;
    g.m2 = 2 * m;
    g.off.assign((size_t)n + 1, 0);
    for (auto& e : edges) { g.off[perm[e.first] + 1]++; g.off[perm[e.second] + 1]++; }
    for (uint32_t v = 0; v < n; ++v) g.off[v + 1] += g.off[v];
    g.adj.assign(g.m2, 0);
    std::vector<uint64_t> fill(g.off.begin(), g.off.end() - 1);
    for (auto& e : edges) {
        uint32_t x = perm[e.first], y = perm[e.second];
        g.adj[fill[x]++] = y;
        g.adj[fill[y]++] = x;
    }
    for (uint32_t v = 0; v < n; ++v) std::sort(g.adj.begin() + g.off[v], g.adj.begin() + g.off[v + 1]);
    g.lab.assign(n, 0);
    if (num_labels > 1) {
        std::vector<double> zw(num_labels);
        for (uint32_t l = 0; l < num_labels; ++l) zw[l] = 1.0 / std::pow((double)(l + 1), zipf_s);
        Alias za(zw);
        for (uint32_t v = 0; v < n; ++v) g.lab[v] = za.sample(rng);
    }
    g.finish();
}

void query_from_host_graph(const HostGraph& g, HostQuery& q) {
    q.n = g.n;
    q.off.assign(g.n + 1, 0);
    for (uint32_t v = 0; v <= g.n; ++v) q.off[v] = (uint32_t)g.off[v];
    q.adj.assign(g.adj.begin(), g.adj.end());
    q.lab.assign(g.lab.begin(), g.lab.end());
    q.finish();
}

// Seeded query extraction.
//   Sparse: a random walk from a seeded vertex of degree >= 2 records every
//   vertex in order of first visit until k are seen; the query holds only the
//   edges the walk traversed (a tree plus the walk's repeat crossings).
//   Dense: from a seeded start vertex the set grows one vertex at a time,
//   taking among the set's neighbours (hub rows sampled to 64 entries) the one
//   with the most links into the set (ties broken at random); the query is
//   the induced subgraph.  Retried from new starts until the average degree
//   exceeds 3 (the densest attempt wins otherwise).
// Query vertex ids follow the order in which vertices joined; labels are
// inherited from the data graph.
namespace {
bool adjacent(const HostGraph& g, uint32_t a, uint32_t b) {
    return std::binary_search(g.adj.begin() + g.off[a], g.adj.begin() + g.off[a + 1], b);
}
}  // namespace

bool generate_walk_query(const HostGraph& g, uint32_t k, bool dense, uint64_t seed, HostQuery& q) {
    if (k == 0 || k > kMaxQ || g.n == 0) return false;
    Rng rng(seed ^ 0x5bd1e9955bd1e995ull);
    std::vector<uint32_t> best_vs;
    std::vector<std::pair<uint32_t, uint32_t>> best_es;
    double best_avg = -1.0;
    const int attempts = dense ? 48 : 16;
    for (int att = 0; att < attempts; ++att) {
        uint32_t start = 0;
        for (int t = 0; t < 1000; ++t) {
            start = (uint32_t)rng.below(g.n);
            if (g.deg(start) >= (dense ? 3u : 2u)) break;
        }
        std::vector<uint32_t> vs{start};
        std::vector<std::pair<uint32_t, uint32_t>> es;
        auto idx_of = [&](uint32_t v) -> int {
            for (size_t i = 0; i < vs.size(); ++i)
                if (vs[i] == v) return (int)i;
            return -1;
        };
        if (!dense) {
            uint32_t cur = start;
            uint64_t steps = 0;
            while (vs.size() < k && steps < 100000ull * k) {
                ++steps;
                uint32_t d = g.deg(cur);
                if (d == 0) break;
                uint32_t nxt = g.adj[g.off[cur] + rng.below(d)];
                int a = idx_of(cur), b = idx_of(nxt);
                if (b < 0) {
                    vs.push_back(nxt);
                    b = (int)vs.size() - 1;
                }
                uint32_t x = (uint32_t)std::min(a, b), y = (uint32_t)std::max(a, b);
                if (x != y && std::find(es.begin(), es.end(), std::make_pair(x, y)) == es.end()) es.emplace_back(x, y);
                cur = nxt;
            }
        } else {
            while (vs.size() < k) {
                std::vector<uint32_t> cand;
                for (uint32_t v : vs) {
                    const uint32_t d = g.deg(v);
                    if (d <= 64) {
                        for (uint64_t e = g.off[v]; e < g.off[v + 1]; ++e) cand.push_back(g.adj[e]);
                    } else {
                        for (int t = 0; t < 64; ++t) cand.push_back(g.adj[g.off[v] + rng.below(d)]);
                    }
                }
                std::sort(cand.begin(), cand.end());
                cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
                uint32_t best = kInvalid, best_links = 0, ties = 0;
                for (uint32_t w : cand) {
                    if (idx_of(w) >= 0) continue;
                    uint32_t links = 0;
                    for (uint32_t v : vs) links += adjacent(g, w, v);
                    if (best == kInvalid || links > best_links) {
                        best = w;
                        best_links = links;
                        ties = 1;
                    } else if (links == best_links && rng.below(++ties) == 0) {
                        best = w;
                    }
                }
                if (best == kInvalid) break;
                vs.push_back(best);
            }
            if (vs.size() == k)
                for (uint32_t i = 0; i < k; ++i)
                    for (uint32_t j = i + 1; j < k; ++j)
                        if (adjacent(g, vs[i], vs[j])) es.emplace_back(i, j);
        }
        if (vs.size() < k) continue;
        double avg = 2.0 * es.size() / k;
        if (avg > best_avg) {
            best_avg = avg;
            best_vs = vs;
            best_es = es;
        }
        if (!dense || avg > 3.0) break;
    }
    if (best_vs.size() < k) return false;
    std::sort(best_es.begin(), best_es.end());
    q.n = k;
    std::vector<uint32_t> deg(k, 0);
    for (auto& e : best_es) {
        deg[e.first]++;
        deg[e.second]++;
    }
    q.off.assign(k + 1, 0);
    for (uint32_t i = 0; i < k; ++i) q.off[i + 1] = q.off[i] + deg[i];
    q.adj.assign(q.off[k], 0);
    std::vector<uint32_t> fill(q.off.begin(), q.off.end() - 1);
    for (auto& e : best_es) {
        q.adj[fill[e.first]++] = e.second;
        q.adj[fill[e.second]++] = e.first;
    }
    for (uint32_t i = 0; i < k; ++i) std::sort(q.adj.begin() + q.off[i], q.adj.begin() + q.off[i + 1]);
    q.lab.resize(k);
    for (uint32_t i = 0; i < k; ++i) q.lab[i] = g.lab[best_vs[i]];
    q.finish();
    return true;
}

// Query::KCore (graph.h:387-458): bin-sorted core decomposition.
void kcore(const HostQuery& q, std::vector<uint32_t>& core) {
    const uint32_t n = q.n;
    const uint32_t md = q.max_deg;
    std::vector<int> c(n), vert(n), pos(n), bin(md + 2, 0), offs(md + 2, 0);
    for (uint32_t i = 0; i < n; ++i) { c[i] = (int)q.deg(i); bin[c[i]]++; }
    int start = 0;
    for (uint32_t i = 0; i <= md; ++i) { offs[i] = start; start += bin[i]; }
    for (uint32_t i = 0; i < n; ++i) {
        int d = (int)q.deg(i);
        pos[i] = offs[d];
        vert[pos[i]] = (int)i;
        offs[d]++;
    }
    for (uint32_t i = md; i > 0; --i) offs[i] = offs[i - 1];
    offs[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        int w = vert[i];
        for (uint32_t e = q.off[w]; e < q.off[w + 1]; ++e) {
            int u = (int)q.adj[e];
            if (c[u] > c[w]) {
                int du = c[u], pu = pos[u], pw = offs[du], x = vert[pw];
                if (u != x) {
                    pos[u] = pw;
                    pos[x] = pu;
                    vert[pu] = x;
                    vert[pw] = u;
                }
                offs[du]++;
                c[u]--;
            }
        }
    }
    core.assign(c.begin(), c.end());
}

// Order_RI (order.h:1138-1281): start at the maximum-degree vertex (lowest id
// on ties), then repeatedly take the unvisited vertex with the most ordered
// neighbours; ties go to the vertex with the most ordered vertices that share
// an unvisited neighbour with it, then to the one with the most unvisited
// neighbours adjacent to no ordered vertex, then to the lowest id.
void order_ri(const HostQuery& q, uint32_t* order) {
    const uint32_t n = q.n;
    uint64_t visited = 0;
    order[0] = 0;
    for (uint32_t i = 1; i < n; ++i)
        if (q.deg(i) > q.deg(order[0])) order[0] = i;
    visited |= 1ull << order[0];
    std::vector<uint32_t> tie, tmp;
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t max_bn = 0;
        tie.clear();
        for (uint32_t u = 0; u < n; ++u) {
            if ((visited >> u) & 1) continue;
            uint32_t bn = __builtin_popcountll(q.nbr_mask[u] & visited);
            if (bn > max_bn) {
                max_bn = bn;
                tie.clear();
                tie.push_back(u);
            } else if (bn == max_bn) {
                tie.push_back(u);
            }
        }
        if (tie.size() != 1) {
            tmp.swap(tie);
            tie.clear();
            uint32_t best = 0;
            for (uint32_t u : tmp) {
                uint64_t unvisited_nbrs = q.nbr_mask[u] & ~visited;
                uint32_t cur = 0;
                for (uint32_t j = 0; j < i; ++j)
                    if (q.nbr_mask[order[j]] & unvisited_nbrs) ++cur;
                if (cur > best) {
                    best = cur;
                    tie.clear();
                    tie.push_back(u);
                } else if (cur == best) {
                    tie.push_back(u);
                }
            }
        }
        if (tie.size() != 1) {
            tmp.swap(tie);
            tie.clear();
            uint32_t best = 0;
            for (uint32_t u : tmp) {
                uint64_t unvisited_nbrs = q.nbr_mask[u] & ~visited;
                uint32_t cur = 0;
                for (uint32_t x = 0; x < n; ++x)
                    if (((unvisited_nbrs >> x) & 1) && !(q.nbr_mask[x] & visited)) ++cur;
                if (cur > best) {
                    best = cur;
                    tie.clear();
                    tie.push_back(u);
                } else if (cur == best) {
                    tie.push_back(u);
                }
            }
        }
        order[i] = tie[0];
        visited |= 1ull << order[i];
    }
}

// Order_GQL (order.h:563-597) with GQLStartVertex (order.h:11-35): start at
// the fewest candidates (larger degree on ties), then repeatedly take the
// adjacent unvisited vertex with the fewest candidates.
void order_gql(const HostQuery& q, const uint32_t* cnt, uint32_t data_n, uint32_t* order) {
    const uint32_t n = q.n;
    uint32_t s = 0;
    for (uint32_t i = 1; i < n; ++i) {
        if (cnt[i] < cnt[s]) s = i;
        else if (cnt[i] == cnt[s] && q.deg(i) > q.deg(s)) s = i;
    }
    uint64_t visited = 1ull << s, adjacent = q.nbr_mask[s];
    order[0] = s;
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t next = 0;
        uint64_t minv = (uint64_t)data_n + 1;
        for (uint32_t j = 0; j < n; ++j) {
            if (((visited >> j) & 1) || !((adjacent >> j) & 1)) continue;
            if (cnt[j] < minv) {
                minv = cnt[j];
                next = j;
            } else if (cnt[j] == minv && q.deg(j) > q.deg(next)) {
                next = j;
            }
        }
        order[i] = next;
        visited |= 1ull << next;
        adjacent |= q.nbr_mask[next];
    }
}

// ------------------------------------------------------------------ learned order: features and beam
// Features of a (query, order) pair for the cost model (64 floats, all
// roughly in [0, 2]): query size and degree / core statistics, per position
// (first 24) the log candidate count and the number of backward neighbours,
// and the cumulative estimated log tree size at positions 1, 2, 3, 4, 6, 8,
// 12, 16 (log candidate count minus 4 bits per extra backward neighbour).
void order_features(const HostQuery& q, const uint32_t* cnt, const uint32_t* order, float* f) {
    const uint32_t n = q.n;
    for (int i = 0; i < SMX_MLP_INPUTS; ++i) f[i] = 0.f;
    std::vector<uint32_t> core;
    kcore(q, core);
    uint32_t maxc = 0, maxd = 0;
    double sumc = 0, suml = 0, minl = 1e30;
    for (uint32_t u = 0; u < n; ++u) {
        maxc = std::max(maxc, core[u]);
        sumc += core[u];
        maxd = std::max(maxd, q.deg(u));
        const double l = std::log2(1.0 + cnt[u]);
        suml += l;
        minl = std::min(minl, l);
    }
    f[0] = n / 32.f;
    f[1] = q.m / 64.f;
    f[2] = n ? (2.f * q.m / n) / 8.f : 0.f;
    f[3] = maxd / 16.f;
    f[4] = maxc / 8.f;
    f[5] = n ? (float)(sumc / n) / 8.f : 0.f;
    f[6] = n ? (float)(suml / n) / 20.f : 0.f;
    f[7] = n ? (float)minl / 20.f : 0.f;
    uint64_t seen = 0;
    std::vector<double> est(n, 0.0);
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t u = order[i];
        const uint32_t nbn = (uint32_t)__builtin_popcountll(q.nbr_mask[u] & seen);
        const double l = std::log2(1.0 + cnt[u]);
        if (i < 24) {
            f[8 + i] = (float)l / 20.f;
            f[32 + i] = nbn / 8.f;
        }
        est[i] = std::max(0.0, l - 4.0 * (nbn > 0 ? nbn - 1 : 0));
        seen |= 1ull << u;
    }
    const uint32_t at[8] = {1, 2, 3, 4, 6, 8, 12, 16};
    for (int k = 0; k < 8; ++k) {
        double c = 0;
        for (uint32_t i = 0; i < std::min(at[k], n); ++i) c += est[i];
        f[56 + k] = (float)c / 64.f;
    }
}

// Candidate orders: RI, GQL, then randomized greedy orders (start drawn with
// weight 1 / (1 + |C(u)|), each next vertex the frontier vertex with the best
// score "2 x backward neighbours - log2 |C| / 4 + noise"), without repeats.
void order_beam(const HostQuery& q, const uint32_t* cnt, uint32_t data_n, uint32_t beam, uint64_t seed,
                std::vector<std::vector<uint32_t>>& out) {
    const uint32_t n = q.n;
    out.clear();
    auto add = [&](const std::vector<uint32_t>& o) {
        for (const auto& x : out)
            if (x == o) return;
        out.push_back(o);
    };
    std::vector<uint32_t> o(n);
    order_ri(q, o.data());
    if (beam > out.size()) add(o);
    order_gql(q, cnt, data_n, o.data());
    if (beam > out.size()) add(o);
    uint64_t st = seed * 0x9e3779b97f4a7c15ULL + 0x1234567ULL;
    auto rnd = [&]() {
        st += 0x9e3779b97f4a7c15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return ((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
    };
    for (uint32_t attempt = 0; out.size() < beam && attempt < 8 * beam + 16; ++attempt) {
        double tot = 0;
        for (uint32_t u = 0; u < n; ++u) tot += 1.0 / (1.0 + cnt[u]);
        double r = rnd() * tot;
        uint32_t s = n - 1;
        for (uint32_t u = 0; u < n; ++u) {
            r -= 1.0 / (1.0 + cnt[u]);
            if (r <= 0) {
                s = u;
                break;
            }
        }
        const double noise = 0.5 + 2.0 * rnd();
        uint64_t seen = 1ull << s;
        o[0] = s;
        for (uint32_t i = 1; i < n; ++i) {
            double best = -1e300;
            uint32_t pick = n;
            for (uint32_t u = 0; u < n; ++u) {
                if (((seen >> u) & 1) || !(q.nbr_mask[u] & seen)) continue;
                const double sc = 2.0 * __builtin_popcountll(q.nbr_mask[u] & seen) -
                                  std::log2(1.0 + cnt[u]) / 4.0 + noise * rnd();
                if (sc > best) {
                    best = sc;
                    pick = u;
                }
            }
            o[i] = pick;
            seen |= 1ull << pick;
        }
        add(o);
    }
}

// isValid (order.h:104-124) plus a permutation check.
bool order_valid(const HostQuery& q, const uint32_t* order) {
    uint64_t seen = 0;
    for (uint32_t i = 0; i < q.n; ++i) {
        if (order[i] >= q.n || ((seen >> order[i]) & 1)) return false;
        if (i > 0 && !(q.nbr_mask[order[i]] & seen)) return false;
        seen |= 1ull << order[i];
    }
    return true;
}

// PlanIR (code_gen.h:682-847).  For the vertex at depth f and every depth
// d < f, its backward neighbours at depths <= d form a prefix; the op for
// (d, f) is that prefix with the vertex's label.  Ops with equal label and
// prefix are one op (the first in the order of code_gen.h:633-650 is kept:
// computed at the depth of its last prefix element).  An op's parent is the op
// with the same label and the prefix minus its last element; the candidates
// of depth f are the op holding all its backward neighbours.
bool build_plan(const HostQuery& q, const uint32_t* order, Plan& plan) {
    const uint32_t n = q.n;
    std::vector<uint32_t> depth_of(n);
    for (uint32_t i = 0; i < n; ++i) depth_of[order[i]] = i;
    std::vector<std::vector<uint32_t>> bn(n);  // backward-neighbour depths, ascending
    for (uint32_t f = 0; f < n; ++f) {
        uint32_t u = order[f];
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            uint32_t d = depth_of[q.adj[e]];
            if (d < f) bn[f].push_back(d);
        }
        std::sort(bn[f].begin(), bn[f].end());
        if (f > 0 && bn[f].empty()) return false;
    }
    plan.ops.clear();
    plan.ops_at.assign(n, {});
    plan.iter_op.assign(n, kInvalid);
    auto find = [&](uint32_t label, const std::vector<uint32_t>& edges) -> uint32_t {
        for (uint32_t i = 0; i < plan.ops.size(); ++i)
            if (plan.ops[i].label == label && plan.ops[i].edges == edges) return i;
        return kInvalid;
    };
    struct Cand {
        uint32_t depth, label, vdepth;
        std::vector<uint32_t> edges;
    };
    std::vector<Cand> all;
    for (uint32_t f = 1; f < n; ++f)
        for (size_t j = 0; j < bn[f].size(); ++j) {
            std::vector<uint32_t> pre(bn[f].begin(), bn[f].begin() + j + 1);
            all.push_back({bn[f][j], q.lab[order[f]], f, pre});
        }
    std::stable_sort(all.begin(), all.end(), [](const Cand& x, const Cand& y) {
        if (x.depth != y.depth) return x.depth < y.depth;
        if (x.label != y.label) return x.label < y.label;
        if (x.edges.size() != y.edges.size()) return x.edges.size() < y.edges.size();
        return x.edges < y.edges;
    });
    for (auto& c : all) {
        if (find(c.label, c.edges) != kInvalid) continue;
        PlanOp op;
        op.depth = c.depth;
        op.vdepth = c.vdepth;
        op.label = c.label;
        op.edges = c.edges;
        op.parent = kInvalid;
        if (c.edges.size() > 1) {
            std::vector<uint32_t> pre(c.edges.begin(), c.edges.end() - 1);
            op.parent = find(c.label, pre);
        }
        plan.ops_at[op.depth].push_back((uint32_t)plan.ops.size());
        plan.ops.push_back(op);
    }
    for (uint32_t f = 1; f < n; ++f) plan.iter_op[f] = find(q.lab[order[f]], bn[f]);
    return true;
}

}  // namespace smx
