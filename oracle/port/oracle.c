/*
 * CPU restatement of the reference's filter -> edge table -> order -> enumerate
 * path (Orrinn/SubgraphMatching, header-only C++20).
 *
 * TEST INFRASTRUCTURE ONLY: this library is the checker used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg.  The product
 * (libsmx) never links or calls it.
 *
 * Every function names the reference file:line it restates.  Parity of this
 * restatement is pinned against the reference compiled from its own sources
 * (oracle/_ref, oracle/Makefile) and against known answers on the reference's
 * bundled hprd graph (7,362,038 embeddings for the densest 4-vertex subgraph
 * of n16_query, 34,149,984 for the 5-vertex one).
 *
 * Conventions match the reference: vertex and label ids are uint32, adjacency
 * rows sorted ascending, candidate lists ascending, edge-table rows ascending
 * candidate indices; at most 64 query vertices (common_type.h:29).
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define SMXO_MAXQ 64
#define SMXO_INVALID 0xffffffffu

typedef struct {
    uint32_t n;          /* vertices */
    uint64_t m;          /* undirected edges as declared in the "t" line */
    uint32_t max_deg;
    uint32_t label_cnt;  /* max(#distinct labels, max label + 1), graph.h:253 */
    uint32_t max_label_freq;
    uint64_t* off;       /* n + 1 */
    uint32_t* adj;       /* 2m, rows sorted */
    uint32_t* lab;       /* n */
    uint32_t* by_label_off; /* label_cnt + 1 */
    uint32_t* by_label;     /* n, ascending ids within each label */
} og_graph;

typedef struct {
    uint32_t v_cnt, e_cnt, max_deg;
    uint32_t* off;   /* v_cnt + 1 */
    uint32_t* edge;  /* candidate indices into C(b) */
    uint32_t* edge_v;/* vertex ids */
} og_table;

typedef struct {
    uint32_t qn;
    int ok;
    uint32_t* cnt;          /* qn */
    uint32_t** cand;        /* qn lists */
    og_table* tab[SMXO_MAXQ][SMXO_MAXQ];
} og_cand;

static double now_ms(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1000.0 + t.tv_nsec / 1e6;
}

static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return x < y ? -1 : (x > y);
}

static inline uint32_t og_deg(const og_graph* g, uint32_t v) { return (uint32_t)(g->off[v + 1] - g->off[v]); }

static int og_has_edge(const og_graph* g, uint32_t u, uint32_t v) {
    /* graph.h:376-378: binary search in the sorted row of u */
    uint64_t lo = g->off[u], hi = g->off[u + 1];
    while (lo < hi) {
        uint64_t mid = (lo + hi) / 2;
        if (g->adj[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo < g->off[u + 1] && g->adj[lo] == v;
}

/* Label index, graph.h:94-109 (buckets in ascending vertex id). */
static void og_finish(og_graph* g) {
    uint32_t maxl = 0;
    uint32_t distinct = 0;
    for (uint32_t v = 0; v < g->n; ++v) if (g->lab[v] > maxl) maxl = g->lab[v];
    uint32_t* freq = calloc((size_t)maxl + 2, sizeof(uint32_t));
    for (uint32_t v = 0; v < g->n; ++v) freq[g->lab[v]]++;
    for (uint32_t l = 0; l <= maxl; ++l) if (freq[l]) distinct++;
    g->label_cnt = g->n ? (distinct > maxl + 1 ? distinct : maxl + 1) : 0;
    g->max_label_freq = 0;
    for (uint32_t l = 0; l <= maxl; ++l) if (freq[l] > g->max_label_freq) g->max_label_freq = freq[l];
    g->by_label_off = calloc((size_t)g->label_cnt + 1, sizeof(uint32_t));
    for (uint32_t l = 0; l < g->label_cnt; ++l) g->by_label_off[l + 1] = g->by_label_off[l] + freq[l];
    g->by_label = malloc(sizeof(uint32_t) * (g->n ? g->n : 1));
    uint32_t* fill = calloc((size_t)g->label_cnt + 1, sizeof(uint32_t));
    for (uint32_t v = 0; v < g->n; ++v) {
        uint32_t l = g->lab[v];
        g->by_label[g->by_label_off[l] + fill[l]++] = v;
    }
    free(fill);
    free(freq);
    g->max_deg = 0;
    for (uint32_t v = 0; v < g->n; ++v) if (og_deg(g, v) > g->max_deg) g->max_deg = og_deg(g, v);
}

/* Graph::Load, graph.h:190-266: "t N M", "v id label deg" (the degree field
 * sets the row offsets), "e u v" (both directions), rows sorted afterwards. */
void* smxo_graph_load(const char* path) {
    FILE* f = fopen(path, "r");
    if (!f) return NULL;
    og_graph* g = calloc(1, sizeof(og_graph));
    char type;
    unsigned long long n = 0, m = 0;
    if (fscanf(f, " %c %llu %llu", &type, &n, &m) != 3) { fclose(f); free(g); return NULL; }
    g->n = (uint32_t)n;
    g->m = m;
    g->off = calloc(n + 1, sizeof(uint64_t));
    g->adj = calloc(2 * m + 1, sizeof(uint32_t));
    g->lab = calloc(n + 1, sizeof(uint32_t));
    uint64_t* fill = calloc(n + 1, sizeof(uint64_t));
    while (fscanf(f, " %c", &type) == 1) {
        if (type == 'v') {
            unsigned long long id, l, d;
            if (fscanf(f, "%llu %llu %llu", &id, &l, &d) != 3) break;
            g->lab[id] = (uint32_t)l;
            g->off[id + 1] = g->off[id] + d;
        } else {
            unsigned long long a, b;
            if (fscanf(f, "%llu %llu", &a, &b) != 2) break;
            g->adj[g->off[a] + fill[a]++] = (uint32_t)b;
            g->adj[g->off[b] + fill[b]++] = (uint32_t)a;
        }
    }
    fclose(f);
    free(fill);
    for (uint32_t v = 0; v < g->n; ++v)
        qsort(g->adj + g->off[v], og_deg(g, v), sizeof(uint32_t), cmp_u32);
    og_finish(g);
    return g;
}

/* Build from a CSR that the caller already holds (rows must be sorted). */
void* smxo_graph_from_csr(uint32_t n, const uint64_t* off, const uint32_t* adj, const uint32_t* lab) {
    og_graph* g = calloc(1, sizeof(og_graph));
    g->n = n;
    g->m = off[n] / 2;
    g->off = malloc(sizeof(uint64_t) * (n + 1));
    memcpy(g->off, off, sizeof(uint64_t) * (n + 1));
    g->adj = malloc(sizeof(uint32_t) * (off[n] ? off[n] : 1));
    memcpy(g->adj, adj, sizeof(uint32_t) * off[n]);
    g->lab = malloc(sizeof(uint32_t) * (n ? n : 1));
    if (lab) memcpy(g->lab, lab, sizeof(uint32_t) * n); else memset(g->lab, 0, sizeof(uint32_t) * n);
    og_finish(g);
    return g;
}

void smxo_graph_free(void* p) {
    og_graph* g = p;
    if (!g) return;
    free(g->off); free(g->adj); free(g->lab); free(g->by_label_off); free(g->by_label);
    free(g);
}

uint32_t smxo_graph_vcount(void* p) { return ((og_graph*)p)->n; }
uint32_t smxo_graph_maxdeg(void* p) { return ((og_graph*)p)->max_deg; }
uint32_t smxo_graph_labelcnt(void* p) { return ((og_graph*)p)->label_cnt; }

/* ---------------------------------------------------------------- filters */

/* NLFByVertex, filter.h:24-58: same label, degree >= query degree, and for
 * every label in the query vertex's neighbourhood the data vertex has at
 * least as many neighbours of that label. */
static uint32_t nlf_by_vertex(const og_graph* d, const og_graph* q, uint32_t u, uint32_t* out,
                              uint32_t* lab_count /* d->label_cnt scratch, zeroed */) {
    uint32_t ql = q->lab[u];
    if (ql >= d->label_cnt) return 0;
    uint32_t qdeg = og_deg(q, u);
    /* query NLF as (label, count) pairs */
    uint32_t ql_lab[SMXO_MAXQ], ql_cnt[SMXO_MAXQ], nq = 0;
    for (uint64_t e = q->off[u]; e < q->off[u + 1]; ++e) {
        uint32_t l = q->lab[q->adj[e]];
        uint32_t k = 0;
        while (k < nq && ql_lab[k] != l) ++k;
        if (k == nq) { ql_lab[nq] = l; ql_cnt[nq] = 0; ++nq; }
        ql_cnt[k]++;
    }
    uint32_t c = 0;
    for (uint32_t i = d->by_label_off[ql]; i < d->by_label_off[ql + 1]; ++i) {
        uint32_t v = d->by_label[i];
        if (og_deg(d, v) < qdeg) continue;
        int ok = 1;
        for (uint32_t k = 0; k < nq; ++k) if (ql_lab[k] >= d->label_cnt) ok = 0;
        if (ok) {
            for (uint64_t e = d->off[v]; e < d->off[v + 1]; ++e) lab_count[d->lab[d->adj[e]]]++;
            for (uint32_t k = 0; k < nq && ok; ++k) if (lab_count[ql_lab[k]] < ql_cnt[k]) ok = 0;
            for (uint64_t e = d->off[v]; e < d->off[v + 1]; ++e) lab_count[d->lab[d->adj[e]]] = 0;
        }
        if (ok) out[c++] = v;
    }
    return c;
}

/* old_cheap, filter.h:95-110: greedy initial matching. */
static void cheap_match(const int* cp, const int* ci, int* match, int* row_match, int n) {
    for (int i = 0; i < n; ++i)
        for (int p = cp[i]; p < cp[i + 1]; ++p) {
            int r = ci[p];
            if (row_match[r] == -1) { match[i] = r; row_match[r] = i; break; }
        }
}

/* match_bfs, filter.h:112-166: BFS augmenting paths from each free column;
 * rows of a failed search tree are retired (-1) for the rest of the call. */
static void bfs_match(const int* cp, const int* ci, int* match, int* row_match, int* visited, int* queue,
                      int* previous, int n, int m) {
    cheap_match(cp, ci, match, row_match, n);
    memset(visited, 0, sizeof(int) * (size_t)m);
    int stamp = 1;
    for (int i = 0; i < n; ++i) {
        if (match[i] != -1 || cp[i] == cp[i + 1]) continue;
        int head = 0, size = 1;
        queue[0] = i;
        while (size > head) {
            int col = queue[head++];
            for (int p = cp[col]; p < cp[col + 1]; ++p) {
                int row = ci[p];
                int t = visited[row];
                if (t == stamp || t == -1) continue;
                previous[row] = col;
                visited[row] = stamp;
                int mc = row_match[row];
                if (mc == -1) {
                    while (row != -1) {           /* flip the augmenting path */
                        int c = previous[row];
                        int nxt = match[c];
                        match[c] = row;
                        row_match[row] = c;
                        row = nxt;
                    }
                    ++stamp;
                    size = 0;
                    break;
                }
                queue[size++] = mc;
            }
        }
        if (match[i] == -1)
            for (int j = 1; j < size; ++j) visited[match[queue[j]]] = -1;
    }
}

typedef struct {
    int *cp, *ci, *lm, *rm, *vis, *queue, *prev;
} match_scratch;

/* verifyExactTwigIso, filter.h:168-204: N(u) must be saturated by a
 * matching into N(v) along pairs (u', w) with w still a valid candidate of u'. */
static int twig_ok(const og_graph* d, const og_graph* q, uint32_t v, uint32_t u, uint8_t** valid, match_scratch* s) {
    uint32_t ln = og_deg(q, u), rn = og_deg(d, v);
    const uint32_t* qn = q->adj + q->off[u];
    const uint32_t* dn = d->adj + d->off[v];
    int ec = 0;
    for (uint32_t i = 0; i < ln; ++i) {
        s->cp[i] = ec;
        for (uint32_t j = 0; j < rn; ++j)
            if (valid[qn[i]][dn[j]]) s->ci[ec++] = (int)j;
    }
    s->cp[ln] = ec;
    for (uint32_t i = 0; i < ln; ++i) s->lm[i] = -1;
    for (uint32_t j = 0; j < rn; ++j) s->rm[j] = -1;
    bfs_match(s->cp, s->ci, s->lm, s->rm, s->vis, s->queue, s->prev, (int)ln, (int)rn);
    for (uint32_t i = 0; i < ln; ++i) if (s->lm[i] == -1) return 0;
    return 1;
}

/* buildTables, table.h:7-139, restated as the function it computes: for each
 * query edge (a, b) and each candidate index i of a, row i of table[a][b]
 * lists, ascending, the indices j with C(b)[j] adjacent to C(a)[i]. */
static void build_tables(const og_graph* d, const og_graph* q, og_cand* c) {
    uint32_t* flag = calloc(d->n ? d->n : 1, sizeof(uint32_t));
    for (uint32_t a = 0; a < q->n; ++a) {
        for (uint64_t qe = q->off[a]; qe < q->off[a + 1]; ++qe) {
            uint32_t b = q->adj[qe];
            for (uint32_t j = 0; j < c->cnt[b]; ++j) flag[c->cand[b][j]] = j + 1;
            og_table* t = calloc(1, sizeof(og_table));
            t->v_cnt = c->cnt[a];
            t->off = calloc((size_t)t->v_cnt + 1, sizeof(uint32_t));
            uint64_t total = 0;
            for (uint32_t i = 0; i < c->cnt[a]; ++i) {
                uint32_t v = c->cand[a][i];
                uint32_t k = 0;
                for (uint64_t e = d->off[v]; e < d->off[v + 1]; ++e) if (flag[d->adj[e]]) ++k;
                t->off[i + 1] = t->off[i] + k;
                if (k > t->max_deg) t->max_deg = k;
                total += k;
            }
            t->e_cnt = (uint32_t)total;
            t->edge = malloc(sizeof(uint32_t) * (total ? total : 1));
            t->edge_v = malloc(sizeof(uint32_t) * (total ? total : 1));
            for (uint32_t i = 0; i < c->cnt[a]; ++i) {
                uint32_t v = c->cand[a][i], w = t->off[i];
                for (uint64_t e = d->off[v]; e < d->off[v + 1]; ++e) {
                    uint32_t x = d->adj[e];
                    if (flag[x]) { t->edge[w] = flag[x] - 1; t->edge_v[w] = x; ++w; }
                }
            }
            for (uint32_t j = 0; j < c->cnt[b]; ++j) flag[c->cand[b][j]] = 0;
            c->tab[a][b] = t;
        }
    }
    free(flag);
}

/* Filter_NLF / Filter_GQL (filter.h:1049-1063): _NLF_Filter (filter.h:80-93),
 * then for GQL two Gauss-Seidel rounds of exact-twig verification in query
 * vertex order (filter.h:273-290) and compaction (filter.h:206-220), then
 * FilterParamConstruct (filter.h:60-78): sorted candidates + edge tables.
 * kind: 0 = NLF, 1 = GQL. */
void* smxo_filter(void* dp, void* qp, int kind, double* ms) {
    const og_graph* d = dp;
    const og_graph* q = qp;
    double t0 = now_ms();
    og_cand* c = calloc(1, sizeof(og_cand));
    c->qn = q->n;
    c->cnt = calloc(q->n, sizeof(uint32_t));
    c->cand = calloc(q->n, sizeof(uint32_t*));
    uint32_t* lab_count = calloc((size_t)d->label_cnt + 1, sizeof(uint32_t));
    c->ok = 1;
    for (uint32_t u = 0; u < q->n; ++u) {
        c->cand[u] = malloc(sizeof(uint32_t) * (d->max_label_freq ? d->max_label_freq : 1));
        if (!c->ok) continue;
        c->cnt[u] = nlf_by_vertex(d, q, u, c->cand[u], lab_count);
        if (c->cnt[u] == 0) c->ok = 0;   /* filter.h:87-90 stops at the first empty set */
    }
    free(lab_count);
    if (c->ok && kind == 1) {
        uint8_t** valid = malloc(sizeof(uint8_t*) * q->n);
        for (uint32_t u = 0; u < q->n; ++u) {
            valid[u] = calloc(d->n ? d->n : 1, 1);
            for (uint32_t j = 0; j < c->cnt[u]; ++j) valid[u][c->cand[u][j]] = 1;
        }
        match_scratch s;
        uint32_t qmax = q->max_deg, dmax = d->max_deg;
        s.cp = malloc(sizeof(int) * (qmax + 2));
        s.ci = malloc(sizeof(int) * ((size_t)qmax * dmax + 1));
        s.lm = malloc(sizeof(int) * (qmax + 1));
        s.rm = malloc(sizeof(int) * (dmax + 1));
        s.vis = malloc(sizeof(int) * (dmax + 1));
        s.queue = malloc(sizeof(int) * (q->n + 1));
        s.prev = malloc(sizeof(int) * (dmax + 1));
        for (int round = 0; round < 2; ++round)
            for (uint32_t u = 0; u < q->n; ++u)
                for (uint32_t j = 0; j < c->cnt[u]; ++j) {
                    uint32_t v = c->cand[u][j];
                    if (v == SMXO_INVALID) continue;
                    if (!twig_ok(d, q, v, u, valid, &s)) {
                        c->cand[u][j] = SMXO_INVALID;
                        valid[u][v] = 0;
                    }
                }
        for (uint32_t u = 0; u < q->n; ++u) {
            uint32_t k = 0;
            for (uint32_t j = 0; j < c->cnt[u]; ++j)
                if (c->cand[u][j] != SMXO_INVALID) c->cand[u][k++] = c->cand[u][j];
            c->cnt[u] = k;
            if (k == 0) c->ok = 0;          /* isCandidateSetValid, filter.h:222-230 */
            free(valid[u]);
        }
        free(valid);
        free(s.cp); free(s.ci); free(s.lm); free(s.rm); free(s.vis); free(s.queue); free(s.prev);
    }
    if (c->ok) {
        for (uint32_t u = 0; u < q->n; ++u) qsort(c->cand[u], c->cnt[u], sizeof(uint32_t), cmp_u32);
        build_tables(d, q, c);
    }
    if (ms) *ms = now_ms() - t0;
    return c;
}

int smxo_cand_ok(void* p) { return ((og_cand*)p)->ok; }
uint32_t smxo_cand_count(void* p, uint32_t u) { return ((og_cand*)p)->cnt[u]; }
void smxo_cand_copy(void* p, uint32_t u, uint32_t* out) {
    og_cand* c = p;
    memcpy(out, c->cand[u], sizeof(uint32_t) * c->cnt[u]);
}
int smxo_table_info(void* p, uint32_t a, uint32_t b, uint32_t* v_cnt, uint32_t* e_cnt, uint32_t* max_deg) {
    og_cand* c = p;
    og_table* t = c->tab[a][b];
    if (!t) return 0;
    *v_cnt = t->v_cnt; *e_cnt = t->e_cnt; *max_deg = t->max_deg;
    return 1;
}
void smxo_table_copy(void* p, uint32_t a, uint32_t b, uint32_t* off, uint32_t* edge, uint32_t* edge_v) {
    og_table* t = ((og_cand*)p)->tab[a][b];
    memcpy(off, t->off, sizeof(uint32_t) * (t->v_cnt + 1));
    memcpy(edge, t->edge, sizeof(uint32_t) * t->e_cnt);
    memcpy(edge_v, t->edge_v, sizeof(uint32_t) * t->e_cnt);
}
void smxo_cand_free(void* p) {
    og_cand* c = p;
    if (!c) return;
    for (uint32_t a = 0; a < c->qn; ++a) {
        free(c->cand[a]);
        for (uint32_t b = 0; b < c->qn; ++b) {
            og_table* t = c->tab[a][b];
            if (t) { free(t->off); free(t->edge); free(t->edge_v); free(t); }
        }
    }
    free(c->cand); free(c->cnt); free(c);
}

/* ---------------------------------------------------------------- orders */

/* Order_RI, order.h:1138-1281. */
void smxo_order_ri(void* qp, uint32_t* order) {
    const og_graph* q = qp;
    uint32_t n = q->n;
    uint8_t visited[SMXO_MAXQ] = {0};
    uint32_t tie[SMXO_MAXQ], tmp[SMXO_MAXQ], nt, ntmp;
    order[0] = 0;
    for (uint32_t i = 1; i < n; ++i) if (og_deg(q, i) > og_deg(q, order[0])) order[0] = i;
    visited[order[0]] = 1;
    for (uint32_t i = 1; i < n; ++i) {
        /* most backward neighbours */
        uint32_t max_bn = 0;
        nt = 0;
        for (uint32_t u = 0; u < n; ++u) {
            if (visited[u]) continue;
            uint32_t bn = 0;
            for (uint32_t j = 0; j < i; ++j) if (og_has_edge(q, u, order[j])) ++bn;
            if (bn > max_bn) { max_bn = bn; nt = 0; tie[nt++] = u; }
            else if (bn == max_bn) tie[nt++] = u;
        }
        if (nt != 1) {
            /* ordered vertices sharing an unvisited neighbour with u */
            memcpy(tmp, tie, sizeof(uint32_t) * nt); ntmp = nt; nt = 0;
            uint32_t best = 0;
            for (uint32_t k = 0; k < ntmp; ++k) {
                uint32_t u = tmp[k];
                uint32_t cur = 0;
                for (uint32_t j = 0; j < i; ++j) {
                    uint32_t uu = order[j];
                    int common = 0;
                    for (uint64_t e = q->off[u]; e < q->off[u + 1] && !common; ++e) {
                        uint32_t x = q->adj[e];
                        if (!visited[x] && og_has_edge(q, uu, x)) common = 1;
                    }
                    if (common) ++cur;
                }
                if (cur > best) { best = cur; nt = 0; tie[nt++] = u; }
                else if (cur == best) tie[nt++] = u;
            }
        }
        if (nt != 1) {
            /* unvisited neighbours of u not adjacent to any ordered vertex */
            memcpy(tmp, tie, sizeof(uint32_t) * nt); ntmp = nt; nt = 0;
            uint32_t best = 0;
            for (uint32_t k = 0; k < ntmp; ++k) {
                uint32_t u = tmp[k];
                uint32_t cur = 0;
                for (uint64_t e = q->off[u]; e < q->off[u + 1]; ++e) {
                    uint32_t x = q->adj[e];
                    if (visited[x]) continue;
                    int ok = 1;
                    for (uint32_t j = 0; j < i && ok; ++j) if (og_has_edge(q, x, order[j])) ok = 0;
                    if (ok) ++cur;
                }
                if (cur > best) { best = cur; nt = 0; tie[nt++] = u; }
                else if (cur == best) tie[nt++] = u;
            }
        }
        order[i] = tie[0];
        visited[order[i]] = 1;
    }
}

/* Order_GQL, order.h:563-597 with GQLStartVertex, order.h:11-35. */
void smxo_order_gql(void* dp, void* qp, void* cp, uint32_t* order) {
    const og_graph* d = dp;
    const og_graph* q = qp;
    const og_cand* c = cp;
    uint32_t n = q->n;
    uint8_t visited[SMXO_MAXQ] = {0}, adjacent[SMXO_MAXQ] = {0};
    uint32_t s = 0;
    for (uint32_t i = 1; i < n; ++i) {
        if (c->cnt[i] < c->cnt[s]) s = i;
        else if (c->cnt[i] == c->cnt[s] && og_deg(q, i) > og_deg(q, s)) s = i;
    }
    order[0] = s;
    visited[s] = 1;
    for (uint64_t e = q->off[s]; e < q->off[s + 1]; ++e) adjacent[q->adj[e]] = 1;
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t next = 0, minv = d->n + 1;
        for (uint32_t j = 0; j < n; ++j) {
            if (visited[j] || !adjacent[j]) continue;
            if (c->cnt[j] < minv) { minv = c->cnt[j]; next = j; }
            else if (c->cnt[j] == minv && og_deg(q, j) > og_deg(q, next)) next = j;
        }
        order[i] = next;
        visited[next] = 1;
        for (uint64_t e = q->off[next]; e < q->off[next + 1]; ++e) adjacent[q->adj[e]] = 1;
    }
}

/* isValid, order.h:104-124: every vertex after the first has an earlier neighbour. */
int smxo_order_valid(void* qp, const uint32_t* order, uint32_t n) {
    const og_graph* q = qp;
    if (n != q->n) return 0;
    for (uint32_t i = 1; i < n; ++i) {
        int ok = 0;
        for (uint32_t j = 0; j < i && !ok; ++j) if (og_has_edge(q, order[i], order[j])) ok = 1;
        if (!ok) return 0;
    }
    return 1;
}

/* ------------------------------------------------------------ enumeration */

/* Candidate-table enumeration, explore.h:255-358 (CandidatesBuffer) and
 * :513-670 (_explore_recur / explore_Intersection_Recursive): the candidates
 * at depth d are the table row of the first backward neighbour (by order
 * position, common_ops.h:259-306), intersected with the rows of the others;
 * a vertex already in the partial embedding is skipped; every surviving
 * candidate at the last depth is one embedding.  The root loop is sharded
 * across threads (an independent sum); `limit` (0 = none) caps the count. */
typedef struct {
    const og_graph* d;
    const og_graph* q;
    const og_cand* c;
    uint32_t n;
    uint32_t order[SMXO_MAXQ];
    uint32_t nbn[SMXO_MAXQ];
    uint32_t bn[SMXO_MAXQ][SMXO_MAXQ];   /* backward neighbours as depths */
    uint64_t limit;
    volatile uint64_t total;
    volatile uint32_t next_root;
    volatile int stop;
    uint64_t work_bytes;
    pthread_mutex_t mu;
} enum_ctx;

static uint32_t isect(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t* out) {
    uint32_t i = 0, j = 0, k = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) ++i;
        else if (a[i] > b[j]) ++j;
        else { out[k++] = a[i]; ++i; ++j; }
    }
    return k;
}

static void* enum_worker(void* arg) {
    enum_ctx* x = arg;
    const og_graph* d = x->d;
    const og_cand* c = x->c;
    uint32_t n = x->n;
    uint32_t maxc = 1;
    for (uint32_t u = 0; u < n; ++u) if (c->cnt[u] > maxc) maxc = c->cnt[u];
    uint32_t* lists[SMXO_MAXQ];
    uint32_t* tmpb = malloc(sizeof(uint32_t) * maxc);
    for (uint32_t i = 0; i < n; ++i) lists[i] = malloc(sizeof(uint32_t) * maxc);
    uint8_t* vis = calloc(d->n ? d->n : 1, 1);
    uint32_t cnt[SMXO_MAXQ], pos[SMXO_MAXQ], idx[SMXO_MAXQ], vid[SMXO_MAXQ];
    uint64_t local_bytes = 0;
    uint32_t u0 = x->order[0];
    for (;;) {
        if (x->stop) break;
        uint32_t r = __atomic_fetch_add(&x->next_root, 1, __ATOMIC_RELAXED);
        if (r >= c->cnt[u0]) break;
        uint64_t ans = 0;
        idx[0] = r;
        vid[0] = c->cand[u0][r];
        vis[vid[0]] = 1;
        int depth = 1;
        int fresh = 1;
        while (depth >= 1 && !x->stop) {
            if (fresh) {
                /* getNextCandidatesImpl, explore.h:284-354 */
                uint32_t u = x->order[depth];
                uint32_t p0 = x->bn[depth][0];
                og_table* t = c->tab[x->order[p0]][u];
                uint32_t rs = t->off[idx[p0]], rl = t->off[idx[p0] + 1] - rs;
                memcpy(lists[depth], t->edge + rs, sizeof(uint32_t) * rl);
                local_bytes += 4ull * rl;
                uint32_t k = rl;
                for (uint32_t b = 1; b < x->nbn[depth] && k; ++b) {
                    uint32_t pb = x->bn[depth][b];
                    og_table* tb = c->tab[x->order[pb]][u];
                    uint32_t s2 = tb->off[idx[pb]], l2 = tb->off[idx[pb] + 1] - s2;
                    local_bytes += 4ull * (k + l2);
                    k = isect(tb->edge + s2, l2, lists[depth], k, tmpb);
                    memcpy(lists[depth], tmpb, sizeof(uint32_t) * k);
                }
                cnt[depth] = k;
                pos[depth] = 0;
                fresh = 0;
            }
            if (pos[depth] >= cnt[depth]) {
                --depth;
                if (depth >= 1) vis[vid[depth]] = 0;
                continue;
            }
            uint32_t ci = lists[depth][pos[depth]++];
            uint32_t v = c->cand[x->order[depth]][ci];
            if (vis[v]) continue;                  /* explore.h:548 */
            if ((uint32_t)depth == n - 1) {
                ++ans;
                /* the reference stops at ans == output_limit (explore.h:587-590) */
                if (x->limit && (ans & 1023) == 0 && x->total + ans >= x->limit) { x->stop = 1; break; }
                continue;
            }
            idx[depth] = ci;
            vid[depth] = v;
            vis[v] = 1;
            ++depth;
            fresh = 1;
        }
        for (int dd = 1; dd < depth && dd < (int)n; ++dd) vis[vid[dd]] = 0;
        vis[vid[0]] = 0;
        uint64_t t = __atomic_add_fetch(&x->total, ans, __ATOMIC_RELAXED);
        if (x->limit && t >= x->limit) x->stop = 1;
    }
    pthread_mutex_lock(&x->mu);
    x->work_bytes += local_bytes;
    pthread_mutex_unlock(&x->mu);
    free(tmpb);
    for (uint32_t i = 0; i < n; ++i) free(lists[i]);
    free(vis);
    return NULL;
}

/* GetPreviousNeb, common_ops.h:259-306: backward neighbours sorted by order
 * position; returns 0 if some vertex after the first has none. */
static int prev_neighbours(const og_graph* q, const uint32_t* order, enum_ctx* x) {
    for (uint32_t dd = 0; dd < q->n; ++dd) {
        uint32_t u = order[dd];
        x->nbn[dd] = 0;
        for (uint32_t p = 0; p < dd; ++p)
            if (og_has_edge(q, u, order[p])) x->bn[dd][x->nbn[dd]++] = p;
        if (dd > 0 && x->nbn[dd] == 0) return 0;
    }
    return 1;
}

uint64_t smxo_explore(void* dp, void* qp, void* cp, const uint32_t* order, uint64_t limit, int threads,
                      double* ms, uint64_t* work_bytes) {
    const og_graph* q = qp;
    enum_ctx* x = calloc(1, sizeof(enum_ctx));
    x->d = dp; x->q = qp; x->c = cp; x->n = q->n; x->limit = limit;
    memcpy(x->order, order, sizeof(uint32_t) * q->n);
    pthread_mutex_init(&x->mu, NULL);
    double t0 = now_ms();
    uint64_t res = 0;
    if (((og_cand*)cp)->ok && prev_neighbours(q, order, x)) {
        if (q->n == 1) {
            res = ((og_cand*)cp)->cnt[order[0]];
        } else {
            if (threads < 1) threads = 1;
            pthread_t* th = malloc(sizeof(pthread_t) * threads);
            for (int i = 0; i < threads; ++i) pthread_create(&th[i], NULL, enum_worker, x);
            for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
            free(th);
            res = x->total;
        }
    }
    if (limit && res > limit) res = limit;
    if (ms) *ms = now_ms() - t0;
    if (work_bytes) *work_bytes = x->work_bytes;
    pthread_mutex_destroy(&x->mu);
    free(x);
    return res;
}

/* Query::KCore, graph.h:387-458 (bin-sort core decomposition). */
uint32_t smxo_query_kcore(void* qp, uint32_t v) {
    const og_graph* q = qp;
    uint32_t n = q->n;
    int core[SMXO_MAXQ], vert[SMXO_MAXQ], pos[SMXO_MAXQ];
    int md = (int)q->max_deg;
    int* bin = calloc((size_t)md + 2, sizeof(int));
    int* offs = calloc((size_t)md + 2, sizeof(int));
    for (uint32_t i = 0; i < n; ++i) { core[i] = (int)og_deg(q, i); bin[core[i]]++; }
    int start = 0;
    for (int i = 0; i <= md; ++i) { offs[i] = start; start += bin[i]; }
    for (uint32_t i = 0; i < n; ++i) { int dg = (int)og_deg(q, i); pos[i] = offs[dg]; vert[pos[i]] = (int)i; offs[dg]++; }
    for (int i = md; i > 0; --i) offs[i] = offs[i - 1];
    offs[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        int w = vert[i];
        for (uint64_t e = q->off[w]; e < q->off[w + 1]; ++e) {
            int u = (int)q->adj[e];
            if (core[u] > core[w]) {
                int du = core[u], pu = pos[u], pw = offs[du], x = vert[pw];
                if (u != x) { pos[u] = pw; pos[x] = pu; vert[pu] = x; vert[pw] = u; }
                offs[du]++;
                core[u]--;
            }
        }
    }
    free(bin); free(offs);
    return (uint32_t)core[v];
}
