/*
 * CPU ORACLE — test infrastructure, not product code.  See hn_oracle.h for
 * what each function restates; the reference line numbers are repeated at
 * each definition.  Single-threaded on purpose: the reference's host
 * verifiers are single-threaded, and this file doubles as the "port" CPU
 * baseline.  The one exception is the input generator hno_gen_rmat, which
 * is not timed.
 */
#include "hn_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- small helpers --------------------------------------------------- */

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

static uint64_t pack(int32_t u, int32_t v) {
    return ((uint64_t)(uint32_t)u << 32) | (uint32_t)v;
}

/* LSD radix sort of 64-bit keys, 16 bits per pass (skipping passes whose
 * digit is the same for every key). */
static void radix_sort_u64(uint64_t* k, int64_t n) {
    if (n < 2) return;
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * 65536);
    uint64_t* a = k;
    uint64_t* b = tmp;
    for (int shift = 0; shift < 64; shift += 16) {
        memset(cnt, 0, sizeof(int64_t) * 65536);
        for (int64_t i = 0; i < n; i++) cnt[(a[i] >> shift) & 0xFFFF]++;
        if (cnt[(a[0] >> shift) & 0xFFFF] == n) continue;
        int64_t sum = 0;
        for (int d = 0; d < 65536; d++) {
            int64_t c = cnt[d];
            cnt[d] = sum;
            sum += c;
        }
        for (int64_t i = 0; i < n; i++) b[cnt[(a[i] >> shift) & 0xFFFF]++] = a[i];
        uint64_t* t = a;
        a = b;
        b = t;
    }
    if (a != k) memcpy(k, a, sizeof(uint64_t) * (size_t)n);
    free(tmp);
    free(cnt);
}

/* Build a CSR (int64 offsets) from sorted packed keys. */
static void keys_to_csr(int32_t nV, const uint64_t* k, int64_t n, int64_t* off,
                        int32_t* adj) {
    memset(off, 0, sizeof(int64_t) * ((size_t)nV + 1));
    for (int64_t i = 0; i < n; i++) off[(k[i] >> 32) + 1]++;
    for (int32_t v = 0; v < nV; v++) off[v + 1] += off[v];
    for (int64_t i = 0; i < n; i++) adj[i] = (int32_t)(uint32_t)k[i];
}

/* ---- CSR construction ------------------------------------------------ */

/* xlib/src/Graph/GraphStd.cpp:174-206 (mirror, drop self loops, sort+unique)
 * and :306-310 (sorted adjacency). */
int64_t hno_build_csr_undirected(int32_t nV, int64_t np, const int32_t* src,
                                 const int32_t* dst, int64_t* off, int32_t* adj) {
    uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(2 * np + 1));
    int64_t n = 0;
    for (int64_t i = 0; i < np; i++) {
        if (src[i] == dst[i]) continue;
        k[n++] = pack(src[i], dst[i]);
        k[n++] = pack(dst[i], src[i]);
    }
    radix_sort_u64(k, n);
    int64_t m = 0;
    for (int64_t i = 0; i < n; i++)
        if (i == 0 || k[i] != k[i - 1]) k[m++] = k[i];
    keys_to_csr(nV, k, m, off, adj);
    free(k);
    return m;
}

/* xlib/src/Graph/GraphStd.cpp:247-268: u->v survives iff
 * (deg_u < deg_v) || (deg_u == deg_v && u < v); degrees are those of the
 * undirected graph.  Input lists are sorted, so output lists stay sorted. */
int64_t hno_orient_by_degree(int32_t nV, const int64_t* off, const int32_t* adj,
                             int64_t* out_off, int32_t* out_adj) {
    int64_t c = 0;
    out_off[0] = 0;
    for (int32_t u = 0; u < nV; u++) {
        int64_t du = off[u + 1] - off[u];
        for (int64_t e = off[u]; e < off[u + 1]; e++) {
            int32_t v = adj[e];
            int64_t dv = off[v + 1] - off[v];
            if (du < dv || (du == dv && u < v)) out_adj[c++] = v;
        }
        out_off[u + 1] = c;
    }
    return c;
}

/* ---- update model ---------------------------------------------------- */

/* Sorted batch keys, with the BatchUpdate preprocessing applied.
 * Returns the number of keys or -1 on a bad id. */
static int64_t sorted_batch(int32_t nV, int64_t b, const int32_t* s,
                            const int32_t* d, int dedup, uint64_t** out) {
    uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(b + 1));
    for (int64_t i = 0; i < b; i++) {
        if (s[i] < 0 || s[i] >= nV || d[i] < 0 || d[i] >= nV) {
            free(k);
            return -1;
        }
        k[i] = pack(s[i], d[i]);
    }
    /* sort_batch: stable sort by dst then by src == lexicographic
     * (hornet/include/Core/SoA/impl/SoAPtr.i.cuh:560-613) */
    qsort(k, (size_t)b, sizeof(uint64_t), cmp_u64);
    int64_t n = b;
    if (dedup) { /* thrust::unique_copy, BatchUpdate.i.cuh:218-240 */
        n = 0;
        for (int64_t i = 0; i < b; i++)
            if (i == 0 || k[i] != k[i - 1]) k[n++] = k[i];
    }
    *out = k;
    return n;
}

static int contains(const int32_t* a, int64_t n, int32_t x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) / 2;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo < n && a[lo] == x;
}

/* HornetInsert.i.cuh:12-27; BatchUpdate.i.cuh:485-502.
 * Graph de-duplication (BatchUpdate.i.cuh:353-392, BatchUpdateKernels.cuh:27-58)
 * walks every graph edge (u,x) of a touched source, finds the FIRST batch
 * entry equal to (u,x) (xlib lower_bound_left) and clears its flag, so
 * exactly the first element of each run of equal batch edges is dropped
 * when (u,x) is already present. */
int64_t hno_insert(int32_t nV, const int64_t* off, const int32_t* adj,
                   int64_t b, const int32_t* bsrc, const int32_t* bdst,
                   unsigned flags, int64_t* out_off, int32_t* out_adj) {
    uint64_t* k = NULL;
    int64_t n = sorted_batch(nV, b, bsrc, bdst, (flags & HNO_DEDUP_BATCH) != 0, &k);
    if (n < 0) return -1;
    if (flags & HNO_DEDUP_GRAPH) {
        int64_t w = 0;
        for (int64_t i = 0; i < n; i++) {
            int first = (i == 0) || (k[i] != k[i - 1]);
            int32_t u = (int32_t)(k[i] >> 32), x = (int32_t)(uint32_t)k[i];
            if (first && contains(adj + off[u], off[u + 1] - off[u], x)) continue;
            k[w++] = k[i];
        }
        n = w;
    }
    /* multiset union, lists re-sorted: the reference appends
     * (BatchUpdateKernels.cuh:243-261) and compares sorted COO
     * (hornet/test/HornetInsertTest.cu:42-75). */
    int64_t bi = 0, o = 0;
    out_off[0] = 0;
    for (int32_t u = 0; u < nV; u++) {
        int64_t e = off[u], ee = off[u + 1];
        while (e < ee || (bi < n && (int32_t)(k[bi] >> 32) == u)) {
            int take_batch;
            if (e >= ee) take_batch = 1;
            else if (bi >= n || (int32_t)(k[bi] >> 32) != u) take_batch = 0;
            else take_batch = (int32_t)(uint32_t)k[bi] < adj[e];
            out_adj[o++] = take_batch ? (int32_t)(uint32_t)k[bi++] : adj[e++];
        }
        out_off[u + 1] = o;
    }
    free(k);
    return n;
}

/* HornetInsert.i.cuh:71-89; BatchUpdate.i.cuh:504-524, :638-700;
 * BatchUpdateKernels.cuh:263-300 (atomicSub on the per-run count, so each
 * run of c_b equal batch edges removes min(c_b, c_g) graph copies) and
 * :335-393 (run counts).  Lists stay sorted here; the reference refills
 * holes from the tail (:395-410) and its tests compare sorted COO
 * (hornet/test/HornetDeleteTest.cu:87-120). */
int64_t hno_erase(int32_t nV, const int64_t* off, const int32_t* adj,
                  int64_t b, const int32_t* bsrc, const int32_t* bdst,
                  unsigned flags, int64_t* out_off, int32_t* out_adj) {
    uint64_t* k = NULL;
    int64_t n = sorted_batch(nV, b, bsrc, bdst, (flags & HNO_DEDUP_BATCH) != 0, &k);
    if (n < 0) return -1;
    int64_t bi = 0, o = 0, removed = 0;
    out_off[0] = 0;
    for (int32_t u = 0; u < nV; u++) {
        int64_t e = off[u], ee = off[u + 1];
        while (e < ee) {
            int32_t x = adj[e];
            /* skip batch entries of u smaller than x */
            while (bi < n && (k[bi] >> 32) == (uint64_t)(uint32_t)u &&
                   (int32_t)(uint32_t)k[bi] < x) bi++;
            int64_t cb = 0;
            while (bi + cb < n && k[bi + cb] == pack(u, x)) cb++;
            int64_t cg = 0;
            while (e + cg < ee && adj[e + cg] == x) cg++;
            int64_t del = cb < cg ? cb : cg;
            removed += del;
            for (int64_t j = del; j < cg; j++) out_adj[o++] = x;
            e += cg;
            bi += cb;
        }
        while (bi < n && (int32_t)(k[bi] >> 32) == u) bi++;
        out_off[u + 1] = o;
    }
    free(k);
    return removed;
}

/* ---- traversal ------------------------------------------------------- */

/* xlib/src/Graph/BFS.cpp:54-76: FIFO queue, distances[dest] =
 * distances[current] + 1 on first discovery; INF = INT32_MAX
 * (TopDown.cu:42).  The level-synchronous GPU TopDown produces the same
 * distances. */
int64_t hno_bfs(int32_t nV, const int64_t* off, const int32_t* adj, int32_t src,
                int32_t* dist) {
    for (int32_t v = 0; v < nV; v++) dist[v] = HNO_INF;
    if (src < 0 || src >= nV) return 0;
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)nV);
    int64_t head = 0, tail = 0, scanned = 0;
    q[tail++] = src;
    dist[src] = 0;
    while (head < tail) {
        int32_t c = q[head++];
        scanned += off[c + 1] - off[c];
        for (int64_t e = off[c]; e < off[c + 1]; e++) {
            int32_t d = adj[e];
            if (dist[d] == HNO_INF) {
                dist[d] = dist[c] + 1;
                q[tail++] = d;
            }
        }
    }
    free(q);
    return scanned;
}

/* ---- triangle counting ----------------------------------------------- */

/* hornetsnest/test/TriangleTest2.cu:22-46 (hostSingleIntersection): a
 * two-pointer merge counting equal pairs. */
static int64_t single_intersection(const int32_t* a, int64_t alen,
                                   const int32_t* b, int64_t blen,
                                   uint64_t* per_vertex) {
    if (!alen || !blen || a[alen - 1] < b[0] || b[blen - 1] < a[0]) return 0;
    int64_t i = 0, j = 0, out = 0;
    while (i < alen && j < blen) {
        if (a[i] == b[j]) {
            if (per_vertex) per_vertex[a[i]]++;
            i++, j++, out++;
        } else if (a[i] < b[j]) {
            i++;
        } else {
            j++;
        }
    }
    return out;
}

/* hornetsnest/test/TriangleTest2.cu:48-69 (hostCountTriangles). */
uint64_t hno_tc_oriented(int32_t nV, const int64_t* off, const int32_t* adj,
                         uint64_t* per_vertex) {
    if (per_vertex) memset(per_vertex, 0, sizeof(uint64_t) * (size_t)nV);
    uint64_t sum = 0;
    for (int32_t s = 0; s < nV; s++) {
        for (int64_t it = off[s]; it < off[s + 1]; it++) {
            int32_t d = adj[it];
            int64_t t = single_intersection(adj + off[s], off[s + 1] - off[s],
                                            adj + off[d], off[d + 1] - off[d],
                                            per_vertex);
            if (per_vertex) {
                per_vertex[s] += (uint64_t)t;
                per_vertex[d] += (uint64_t)t;
            }
            sum += (uint64_t)t;
        }
    }
    return sum;
}

/* hostCountTriangles restricted to the oriented edges first, first + stride,
 * ... in CSR order (a uniform edge sample, for a bounded CPU timing);
 * *edges receives the number of sampled edges. */
uint64_t hno_tc_oriented_sample(int32_t nV, const int64_t* off, const int32_t* adj,
                                int32_t first, int32_t stride, int64_t* edges) {
    uint64_t sum = 0;
    int64_t e = 0;
    for (int32_t s = 0; s < nV; s++) {
        int64_t it = off[s];
        if (it < first) it = first;
        else if ((it - first) % stride) it += stride - (it - first) % stride;
        for (; it < off[s + 1]; it += stride) {
            int32_t d = adj[it];
            sum += (uint64_t)single_intersection(adj + off[s], off[s + 1] - off[s],
                                                 adj + off[d], off[d + 1] - off[d], NULL);
            e++;
        }
    }
    if (edges) *edges = e;
    return sum;
}

/* ---- connected components -------------------------------------------- */

/* xlib/src/Graph/WCC.cpp:54-98 (undirected branch): components are found in
 * order of their smallest vertex id, so relabelling component c to the
 * source that opened it gives the min-id label directly. */
int32_t hno_cc_min_label(int32_t nV, const int64_t* off, const int32_t* adj,
                         int32_t* label) {
    int32_t* q = (int32_t*)malloc(sizeof(int32_t) * (size_t)(nV + 1));
    for (int32_t v = 0; v < nV; v++) label[v] = -1;
    int32_t ncomp = 0;
    for (int32_t s = 0; s < nV; s++) {
        if (label[s] != -1) continue;
        int64_t head = 0, tail = 0;
        label[s] = s;
        q[tail++] = s;
        while (head < tail) {
            int32_t c = q[head++];
            for (int64_t e = off[c]; e < off[c + 1]; e++) {
                int32_t d = adj[e];
                if (label[d] == -1) {
                    label[d] = s;
                    q[tail++] = d;
                }
            }
        }
        ncomp++;
    }
    free(q);
    return ncomp;
}

/* hornetsnest/src/Static/ConnectedComponents/CC.cu:133-156: BFS-colour the
 * component of max_degree_id() with 0; every other vertex starts at id+1
 * (BuildVertexEnqueue, :65-75) and the pair queue propagates the MAX colour
 * (ColoringOperator, :86-106) to a fixed point, i.e. max(id)+1 per
 * component.  max_degree_id is thrust::max_element: lowest id on ties
 * (hornet/include/Core/HornetOperations/HornetQuery.i.cuh:10-21). */
void hno_cc_reference_colors(int32_t nV, const int64_t* off, const int32_t* adj,
                             int32_t* color) {
    if (nV <= 0) return;
    int32_t* lab = (int32_t*)malloc(sizeof(int32_t) * (size_t)nV);
    int32_t* mx = (int32_t*)malloc(sizeof(int32_t) * (size_t)nV);
    hno_cc_min_label(nV, off, adj, lab);
    int32_t best = 0;
    int64_t bestd = -1;
    for (int32_t v = 0; v < nV; v++) {
        int64_t d = off[v + 1] - off[v];
        if (d > bestd) { bestd = d; best = v; }
        mx[v] = -1;
    }
    for (int32_t v = 0; v < nV; v++)
        if (v > mx[lab[v]]) mx[lab[v]] = v;
    for (int32_t v = 0; v < nV; v++)
        color[v] = (lab[v] == lab[best]) ? 0 : mx[lab[v]] + 1;
    free(lab);
    free(mx);
}

/* ---- k-truss ------------------------------------------------------------ */

/* Support of every alive directed edge: |alive N(u) ∩ alive N(v)|
 * (KTrussSupport.cu:212-294 intersectCount over the current graph). */
static void supports(int32_t nV, const int64_t* off, const int32_t* adj,
                     const unsigned char* alive, int32_t* sup) {
    for (int32_t u = 0; u < nV; u++) {
        for (int64_t e = off[u]; e < off[u + 1]; e++) {
            sup[e] = 0;
            if (!alive[e]) continue;
            int32_t v = adj[e];
            int64_t i = off[u], j = off[v];
            while (i < off[u + 1] && j < off[v + 1]) {
                if (!alive[i]) { i++; continue; }
                if (!alive[j]) { j++; continue; }
                if (adj[i] == adj[j]) { sup[e]++; i++; j++; }
                else if (adj[i] < adj[j]) i++;
                else j++;
            }
        }
    }
}

/* hornetsnest/src/Static/KTruss/KTruss.cu:90-174.  run(): max_K starts at 3;
 * findTrussOfK repeats {recompute every support; delete every edge whose
 * support < max_K - 2} until a pass deletes nothing; when no edge is left
 * max_K-- and stop, otherwise max_K++ on the peeled graph. */
int32_t hno_ktruss(int32_t nV, const int64_t* off, const int32_t* adj,
                   int32_t* edge_truss) {
    int64_t m = off[nV];
    unsigned char* alive = (unsigned char*)malloc((size_t)m + 1);
    int32_t* sup = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    memset(alive, 1, (size_t)m);
    for (int64_t e = 0; e < m; e++) edge_truss[e] = 2;
    int64_t remaining = m;
    int32_t K = 3;
    for (;;) {
        for (;;) {
            if (remaining <= 0) break;
            supports(nV, off, adj, alive, sup);
            int64_t del = 0;
            for (int64_t e = 0; e < m; e++)
                if (alive[e] && sup[e] < K - 2) { alive[e] = 0; del++; }
            if (del == 0) break;
            remaining -= del;
        }
        if (remaining <= 0) { K--; break; }
        for (int64_t e = 0; e < m; e++)
            if (alive[e]) edge_truss[e] = K;
        K++;
    }
    free(alive);
    free(sup);
    return K;
}

/* Truss decomposition by support peeling (J. Wang and J. Cheng, "Truss
 * Decomposition in Massive Networks", PVLDB 5(9), 2012): supports are
 * computed once, then for k = 2, 3, ... every edge whose support is at most
 * k-2 is removed (truss number k), each removal decrementing the two other
 * edges of every triangle it destroys.  The truss numbers are those of
 * hno_ktruss (the reference's recompute-from-scratch loop), in far less
 * time; the tests check the two against each other. */
static int64_t find_pos(const int64_t* off, const int32_t* adj, int32_t u, int32_t v) {
    int64_t lo = off[u], hi = off[u + 1];
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (adj[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

/* Calls f(pos in x's list, pos in y's list) for every common neighbour of
 * x and y: a merge when the lists are of similar length, else the shorter
 * list probes the longer one by binary search. */
#define FOR_COMMON(x, y, PA, PB, ...)                                               \
    do {                                                                           \
        int64_t dx_ = off[(x) + 1] - off[x], dy_ = off[(y) + 1] - off[y];          \
        int32_t s_ = dx_ <= dy_ ? (x) : (y), l_ = dx_ <= dy_ ? (y) : (x);          \
        int64_t ds_ = dx_ <= dy_ ? dx_ : dy_, dl_ = dx_ <= dy_ ? dy_ : dx_;        \
        if (dl_ > 16 * ds_) {                                                      \
            for (int64_t a_ = off[s_]; a_ < off[s_ + 1]; a_++) {                    \
                int64_t b_ = find_pos(off, adj, l_, adj[a_]);                      \
                if (b_ >= off[l_ + 1] || adj[b_] != adj[a_]) continue;             \
                int64_t PA = s_ == (x) ? a_ : b_, PB = s_ == (x) ? b_ : a_;        \
                __VA_ARGS__                                                        \
            }                                                                      \
        } else {                                                                   \
            int64_t a_ = off[x], ae_ = off[(x) + 1], b_ = off[y], be_ = off[(y) + 1]; \
            while (a_ < ae_ && b_ < be_) {                                         \
                if (adj[a_] < adj[b_]) a_++;                                       \
                else if (adj[a_] > adj[b_]) b_++;                                  \
                else {                                                             \
                    int64_t PA = a_, PB = b_;                                      \
                    __VA_ARGS__                                                    \
                    a_++;                                                          \
                    b_++;                                                          \
                }                                                                  \
            }                                                                      \
        }                                                                          \
    } while (0)

int32_t hno_ktruss_peel(int32_t nV, const int64_t* off, const int32_t* adj,
                        int32_t* edge_truss) {
    int64_t m = off[nV];
    int64_t* canon = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    int32_t* esrc = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    int32_t* sup = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    int32_t* truss = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m + 1));
    unsigned char* alive = (unsigned char*)malloc((size_t)m + 1);
    int64_t* stack = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    int64_t* alist = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m + 1));
    for (int32_t u = 0; u < nV; u++)
        for (int64_t p = off[u]; p < off[u + 1]; p++) {
            int32_t v = adj[p];
            esrc[p] = u;
            canon[p] = u < v ? p : find_pos(off, adj, v, u);
        }
    int64_t na = 0;
    for (int64_t p = 0; p < m; p++) {
        alive[p] = 0;
        truss[p] = 2;
        sup[p] = 0;
        int32_t u = esrc[p], v = adj[p];
        if (u >= v) continue;
        alive[p] = 1;
        alist[na++] = p;
        int32_t c = 0;
        FOR_COMMON(u, v, pa, pb, { (void)pa; (void)pb; c++; });
        sup[p] = c;
    }
    int32_t k = 2, maxk = 2;
    while (na > 0) {
        int64_t top = 0;
        for (int64_t i = 0; i < na; i++)
            if (sup[alist[i]] <= k - 2) stack[top++] = alist[i];
        while (top > 0) {
            int64_t e = stack[--top];
            if (!alive[e]) continue;
            alive[e] = 0;
            truss[e] = k;
            maxk = k;
            int32_t u = esrc[e], v = adj[e];
            FOR_COMMON(u, v, pa, pb, {
                int64_t e1 = canon[pa], e2 = canon[pb];
                if (alive[e1] && alive[e2]) {
                    if (--sup[e1] == k - 2) stack[top++] = e1;
                    if (--sup[e2] == k - 2) stack[top++] = e2;
                }
            });
        }
        int64_t w = 0;
        for (int64_t i = 0; i < na; i++)
            if (alive[alist[i]]) alist[w++] = alist[i];
        na = w;
        k++;
    }
    for (int64_t p = 0; p < m; p++) edge_truss[p] = truss[canon[p]];
    free(canon);
    free(esrc);
    free(sup);
    free(truss);
    free(alive);
    free(stack);
    free(alist);
    return maxk;
}

/* ---- synthetic inputs and checksums ---------------------------------- */

/* SplitMix64 (S. Vigna's published finaliser). */
static uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

typedef struct {
    int scale, n;
    uint64_t ta, tb, tc, seed;
    int64_t i0, i1;
    int32_t *src, *dst;
} rmat_job;

/* Pair i: a counter-based SplitMix64 stream per pair, one 32-bit uniform per
 * recursion level (two per draw), quadrant thresholds a, a+b, a+b+c scaled to
 * 2^32; a pair with an endpoint >= n is redrawn from the next attempt
 * counter (64 attempts, then folded into range). */
static void* rmat_worker(void* arg) {
    rmat_job* j = (rmat_job*)arg;
    for (int64_t i = j->i0; i < j->i1; i++) {
        uint64_t base = splitmix64(j->seed ^ ((uint64_t)i * 0xD1B54A32D192ED03ull));
        int done = 0;
        for (int attempt = 0; attempt < 64 && !done; attempt++) {
            uint64_t ctr = base + (uint64_t)attempt * 0x10000ull;
            uint32_t u = 0, v = 0;
            uint64_t bits = 0;
            for (int l = 0; l < j->scale; l++) {
                if ((l & 1) == 0) bits = splitmix64(ctr + (uint64_t)(l >> 1));
                uint64_t r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
                /* quadrants: [0,ta) -> (0,0), [ta,tb) -> (0,1),
                 * [tb,tc) -> (1,0), [tc,2^32) -> (1,1) */
                uint32_t ub = r >= j->tb;
                uint32_t vb = (r >= j->ta && r < j->tb) || r >= j->tc;
                u = (u << 1) | ub;
                v = (v << 1) | vb;
            }
            if ((int32_t)u < j->n && (int32_t)v < j->n) {
                j->src[i] = (int32_t)u;
                j->dst[i] = (int32_t)v;
                done = 1;
            }
        }
        if (!done) {
            j->src[i] = (int32_t)(base % (uint64_t)j->n);
            j->dst[i] = (int32_t)((base >> 32) % (uint64_t)j->n);
        }
    }
    return NULL;
}

/* The R-MAT pairs of this repository's input generator (hn_gen_rmat_host in
 * hornet_b200/csrc/hn_gen.cu): the reference has no R-MAT generator, so the
 * inputs are defined by this function and the library's, which the tests
 * keep bit-identical. */
int hno_gen_rmat(int32_t scale, int32_t n, int64_t np, double a, double b, double c,
                 uint64_t seed, int32_t* src, int32_t* dst, int32_t nthreads) {
    if (scale < 1 || scale > 31 || n <= 0 || (int64_t)n > ((int64_t)1 << scale)) return -1;
    if (a < 0 || b < 0 || c < 0 || a + b + c > 1.0) return -1;
    const double two32 = 4294967296.0;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    rmat_job jobs[256];
    for (int t = 0; t < nthreads; t++) {
        rmat_job* j = &jobs[t];
        j->scale = scale;
        j->n = n;
        j->ta = (uint64_t)(a * two32);
        j->tb = (uint64_t)((a + b) * two32);
        j->tc = (uint64_t)((a + b + c) * two32);
        j->seed = seed;
        j->i0 = np * t / nthreads;
        j->i1 = np * (t + 1) / nthreads;
        j->src = src;
        j->dst = dst;
        if (pthread_create(&th[t], NULL, rmat_worker, j) != 0) {
            rmat_worker(j);
            th[t] = 0;
        }
    }
    for (int t = 0; t < nthreads; t++)
        if (th[t]) pthread_join(th[t], NULL);
    return 0;
}

/* Order-independent checksum of a CSR's edge multiset:
 * sum over edges (u, v) of splitmix64(u << 32 | v), mod 2^64. */
uint64_t hno_adjacency_hash(int32_t nV, const int64_t* off, const int32_t* adj) {
    uint64_t h = 0;
    for (int32_t u = 0; u < nV; u++)
        for (int64_t e = off[u]; e < off[u + 1]; e++) h += splitmix64(pack(u, adj[e]));
    return h;
}
