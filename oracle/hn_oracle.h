/*
 * CPU ORACLE — test infrastructure, not product code.
 *
 * A plain-C restatement of the reference algorithms on the Hornet hot path,
 * used only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * as the checker.  Every function cites the reference file:line it follows
 * (paths relative to the hornet-gt/hornet source tree).
 *
 * Pinning: the CSR builder, BFS and CC are checked against the reference's own
 * host code (xlib GraphStd / BFS / WCC compiled into oracle/_ref/ref_driver)
 * and against the hand-checked fixtures in tests/golden/; the update model is
 * checked the way hornet/test/HornetInsertTest.cu and HornetDeleteTest.cu
 * check the GPU (sorted COO multiset union / difference).
 *
 * Graphs are CSR with int64 offsets and int32 neighbour ids; adjacency lists
 * are sorted ascending (multisets allowed where stated).
 */
#ifndef HN_ORACLE_H
#define HN_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HNO_INF 2147483647
#define HNO_DEDUP_BATCH 1u
#define HNO_DEDUP_GRAPH 2u

/* Undirected CSR from an edge-pair list: mirror every pair, drop self loops,
 * sort, remove duplicates (xlib/src/Graph/GraphStd.cpp:174-206, :306-310).
 * adj must hold 2*np entries.  Returns the number of directed edges m. */
int64_t hno_build_csr_undirected(int32_t nV, int64_t np, const int32_t* src,
                                 const int32_t* dst, int64_t* off, int32_t* adj);

/* Degree-oriented graph for triangle counting: keep u->v iff
 * deg(u) < deg(v) or (deg(u) == deg(v) and u < v)
 * (xlib/src/Graph/GraphStd.cpp:247-268), lists sorted.  out_adj holds m/2+1.
 * Returns the number of oriented edges. */
int64_t hno_orient_by_degree(int32_t nV, const int64_t* off, const int32_t* adj,
                             int64_t* out_off, int32_t* out_adj);

/* Batch insert on a sorted multiset CSR (hornet/include/Core/HornetOperations/
 * HornetInsert.i.cuh:12-27 with BatchUpdate.i.cuh:485-502 preprocessing).
 * out_adj must hold nE + b entries.  Returns the number of batch edges
 * applied, or -1 if a batch id is outside [0, nV). */
int64_t hno_insert(int32_t nV, const int64_t* off, const int32_t* adj,
                   int64_t b, const int32_t* bsrc, const int32_t* bdst,
                   unsigned flags, int64_t* out_off, int32_t* out_adj);

/* Batch erase on a sorted multiset CSR (HornetInsert.i.cuh:71-89 with
 * BatchUpdate.i.cuh:504-524, BatchUpdateKernels.cuh:263-300, :335-393):
 * every distinct (u,v) removes min(batch multiplicity, graph multiplicity)
 * copies.  Returns the number of edges removed, or -1 on a bad id. */
int64_t hno_erase(int32_t nV, const int64_t* off, const int32_t* adj,
                  int64_t b, const int32_t* bsrc, const int32_t* bdst,
                  unsigned flags, int64_t* out_off, int32_t* out_adj);

/* BFS distances from src, INF = INT32_MAX (xlib/src/Graph/BFS.cpp:54-76,
 * hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:42).  Returns the
 * number of directed edges scanned (sum of degrees of visited vertices). */
int64_t hno_bfs(int32_t nV, const int64_t* off, const int32_t* adj, int32_t src,
                int32_t* dist);

/* Triangle count on a degree-oriented sorted graph: the restated
 * hostCountTriangles / hostSingleIntersection
 * (hornetsnest/test/TriangleTest2.cu:22-69).  If per_vertex is non-null it
 * receives, for every vertex, the number of triangles that contain it. */
uint64_t hno_tc_oriented(int32_t nV, const int64_t* off, const int32_t* adj,
                         uint64_t* per_vertex);

/* hno_tc_oriented over the oriented edges first, first + stride, ... (CSR
 * order) only: a uniform edge sample for a bounded CPU timing; *edges = the
 * number of sampled edges. */
uint64_t hno_tc_oriented_sample(int32_t nV, const int64_t* off, const int32_t* adj,
                                int32_t first, int32_t stride, int64_t* edges);

/* Connected components of an undirected graph labelled by the minimum vertex
 * id of each component (xlib/src/Graph/WCC.cpp:54-98 relabelled).  Returns
 * the number of components. */
int32_t hno_cc_min_label(int32_t nV, const int64_t* off, const int32_t* adj,
                         int32_t* label);

/* The colours hornetsnest CC::run produces (ConnectedComponents/CC.cu:133-156):
 * the component of the max-degree vertex (lowest id on ties,
 * HornetQuery.i.cuh:10-21) gets 0, every other component gets
 * max(id) + 1 over its members. */
void hno_cc_reference_colors(int32_t nV, const int64_t* off, const int32_t* adj,
                             int32_t* color);

/* k-truss by iterated peeling (hornetsnest/src/Static/KTruss/KTruss.cu:90-174,
 * support = |N(u) ∩ N(v)| as KTrussSupport.cu:375-449 counts it) on a simple
 * undirected sorted graph.  edge_truss[e] (CSR order) = the largest k whose
 * k-truss holds edge e, 2 if none.  Returns max_K (2 when no 3-truss). */
int32_t hno_ktruss(int32_t nV, const int64_t* off, const int32_t* adj,
                   int32_t* edge_truss);

/* The same truss numbers by support peeling (Wang & Cheng, PVLDB 2012):
 * supports once, then decremented per destroyed triangle.  An independent
 * second computation, fast enough for the benchmark-scale pins; checked
 * against hno_ktruss by the tests. */
int32_t hno_ktruss_peel(int32_t nV, const int64_t* off, const int32_t* adj,
                        int32_t* edge_truss);

/* R-MAT edge pairs of this repository's input generator (restated from
 * hn_gen_rmat_host, hornet_b200/csrc/hn_gen.cu; the reference has none):
 * pair i depends only on (seed, i).  nthreads host threads.  Returns 0, or
 * -1 on bad parameters. */
int hno_gen_rmat(int32_t scale, int32_t n, int64_t np, double a, double b, double c,
                 uint64_t seed, int32_t* src, int32_t* dst, int32_t nthreads);

/* Order-independent checksum of the edge multiset of a CSR:
 * sum of splitmix64(u << 32 | v) over its edges, mod 2^64. */
uint64_t hno_adjacency_hash(int32_t nV, const int64_t* off, const int32_t* adj);

#ifdef __cplusplus
}
#endif
#endif
