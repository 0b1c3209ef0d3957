/*
 * hornet_b200 — C ABI of the B200-native Hornet dynamic-graph hot path.
 *
 * Every entry point returns an int status (HN_OK or HN_ERR_*), never exits
 * the process, and records a message readable with hn_last_error_string().
 * The reference's error path prints, asserts and exits
 * (xlib/src/Device/Util/SafeCudaAPI.cpp:71-94); this layer reports instead.
 *
 * Ids are int32 (VID_T = DEGREE_T = int, hornet/include/Core/Conf/
 * HornetConf.cuh:41-42).  Unless an entry point says otherwise, pointer
 * arguments name HOST memory when `mem` is HN_MEM_HOST and DEVICE memory on
 * the graph's device when it is HN_MEM_DEVICE.  Calls on one handle must be
 * serialised by the caller; handles on different devices are independent
 * (the reference's multi-GPU use is one replica per device,
 * hornet/test/HornetMultiGPUInsertTest.cu:43-81).
 *
 * All calls are synchronous with respect to the host, as the reference's
 * are (every operator ends in CHECK_CUDA_ERROR), except those documented
 * as asynchronous on the graph's stream.
 */
#ifndef HORNET_B200_H
#define HORNET_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define HN_OK            0
#define HN_ERR_INVALID   1   /* bad argument (null pointer, id out of range) */
#define HN_ERR_OOM       2   /* device allocation failed */
#define HN_ERR_CAPACITY  3   /* a fixed-capacity buffer would overflow */
#define HN_ERR_TIMEOUT   4   /* a bounded device wait gave up */
#define HN_ERR_CUDA      5   /* any other CUDA runtime error */
#define HN_ERR_STATE     6   /* call not valid in the object's state */

/* ---- memory kinds / flags --------------------------------------------- */
#define HN_MEM_HOST      0
#define HN_MEM_DEVICE    1

#define HN_CSR_SORTED    1u  /* adjacency lists already sorted ascending */

#define HN_DEDUP_BATCH   1u  /* removeBatchDuplicates (Hornet.cuh:107,109) */
#define HN_DEDUP_GRAPH   2u  /* removeGraphDuplicates (Hornet.cuh:107)     */

#define HN_CC_MIN_ID     0   /* label = minimum vertex id of the component  */
#define HN_CC_REFERENCE  1   /* hornetsnest CC colours: giant = 0, others
                                max(id)+1 (ConnectedComponents/CC.cu:133-156) */

#define HN_LB_BINARY_SEARCH 0 /* load_balancing::BinarySearch              */
#define HN_LB_VERTEX_BASED  1 /* load_balancing::VertexBased<VW>           */

typedef struct hn_graph hn_graph_t;
typedef struct hn_batch hn_batch_t;

/* Device view of a graph for user kernels (the C counterpart of
 * hornet::HornetDevice, hornet/include/Core/HornetDevice/HornetDevice.cuh:52-90).
 * vertex v: record vtab + 16*v = {int64 off; int32 deg; int32 cap};
 * its sorted neighbours are pool[off .. off+deg). */
typedef struct hn_device_view {
    int32_t nV;
    int32_t pad;
    int64_t nE;
    const void* vtab;
    const int32_t* pool;
} hn_device_view_t;

/* Per-call statistics of a traversal. */
typedef struct hn_bfs_stats {
    int32_t levels;          /* number of BFS levels (max distance + 1) */
    int32_t pad;
    int64_t visited;         /* vertices reached */
    int64_t edges_scanned;   /* sum of degrees of reached vertices */
} hn_bfs_stats_t;

/* ---- library ------------------------------------------------------------ */
const char* hn_last_error_string(void);
int hn_version(void);
/* Number of device kernels this library has launched in this process
 * (instrumentation for the benchmark's launch count). */
int64_t hn_kernel_launches(void);
/* Per-kernel timing: when enabled, every library kernel launch is bracketed
 * by CUDA events on its own stream.  hn_profile_enable also clears the
 * records.  hn_profile_report writes a JSON object
 * {"kernel": {"launches": n, "ms": total}, ...} (synchronises). */
int hn_profile_enable(int on);
int hn_profile_report(char* buf, int64_t len);

/* Tuning knobs (process-wide; read when a call launches, so a change takes
 * effect on the next call).  An autotuner sets them; the defaults are the
 * built-in values.  Knobs:
 *   bfs.ctas_per_sm     CTAs per SM of the BFS level kernel, 128 threads
 *                       each (1..16, 9)
 *   bfs.do_alpha        direction-optimising switch to bottom-up when the
 *                       frontier's edges exceed unexplored edges / alpha (14)
 *   bfs.do_beta         back to top-down below nV / beta frontier vertices (24)
 *   msbfs.block         batched-BFS block size: 128, 256 or 512 (256)
 *   msbfs.ctas_per_sm   batched-BFS CTAs per SM (1..8, 4)
 *   tc.warp_cap         oriented-degree bin boundary between the warp-per-
 *                       vertex and CTA-per-vertex counting kernels (32..512, 512)
 *   tc.chunk            vertices handed to a warp per atomic (1..256, 16)
 *   tc.narrow_min       candidate lists longer than this are first narrowed
 *                       to the [min, max] of N+(u) by two searches (0..1024, 0)
 *   tc.mid_cap          listed vertices (oriented degree above tc.warp_cap)
 *                       up to this go to the CTA kernel with small tables,
 *                       several CTAs per SM (32..4096, 4096)
 *   tc.cta_table_cap    table capacity of the CTA kernel for the larger
 *                       listed vertices; above it N+(u) is binary-searched
 *                       in global memory (32..16384, 16384)
 *   tc.warp_work        bound on a vertex's pairs (candidates x d+(u)) for
 *                       the warp-per-vertex kernel; above it, or with d+(u)
 *                       above tc.warp_cap, the vertex goes to CTA work
 *                       items (1024..2^30, 65536)
 *   tc.item_work        pairs bound of one CTA work item (1024..2^30, 262144)
 *   tc.flip             1: each oriented edge is counted by the endpoint
 *                       with the longer out-list (the shorter list is
 *                       probed); 0: by its tail (0..1, 1)
 *   tc.thread_du        with tc.flip: vertices with d+(u) up to this and at
 *   tc.thread_dc        most tc.thread_dc candidates run a thread each,
 *                       merging sorted lists (0 turns it off) (0..64, 16;
 *                       1..1024, 32)
 *   msbfs.bottom_up     1: batched BFS runs bottom-up levels while the
 *                       frontier is large (bfs.do_alpha / do_beta switch) (0..1, 1)
 *   tc.warp_ctas_per_sm CTAs per SM of the warp-per-vertex kernel (1..16, 8)
 *   bfs.dynamic_chunks  1: BFS CTAs take frontier chunks from a counter
 *                       instead of round-robin (0..1, 0)
 *   bfs.warp_strided    1: a warp's frontier edges are dealt to lanes
 *                       round-robin (coalesced loads) instead of 8
 *                       consecutive edges per thread (0..1, 0)
 *   bfs.host_levels     1: launch the BFS levels one by one from the host
 *                       (for per-level profiling) instead of the CUDA
 *                       graph's device-side loop (0..1, 0)
 *   bfs.kernel          BFS level kernel: 1 = independent warps on 256-edge
 *                       chunks, 0 = 128-thread CTAs on 1024-edge chunks
 *                       (bfs.ctas_per_sm, bfs.dynamic_chunks and
 *                       bfs.warp_strided apply to it) (0..1, 1)
 *   bfs.warp_ctas_per_sm  CTAs per SM of the warp-chunk level kernel, 256
 *                       threads each (1..8, 4)
 *   ktruss.device_rounds  1: the peel rounds of each K run in a CUDA graph
 *                       (WHILE node, no host round trip per round); 0: one
 *                       host round trip per round, launches sized to the
 *                       frontier (0..1, 1)
 *   update.big_min      old lists of at least this many entries (hubs) are
 *                       moved in 4096-entry chunks by their own kernel
 *                       (4..2^30, 2048)
 *   update.in_place     1: a vertex whose block class does not change is
 *                       updated inside its block, rewriting only its entries
 *                       from the first one that moves (at most 2048 of
 *                       them); 0: every touched vertex moves to a new block
 *                       (0..1, 1)
 *   update.own_sort     1: the batch keys are sorted by this library's LSD
 *                       radix sort; 0: by CUB's DeviceRadixSort (0..1, 1)
 * hn_tune_name(i) enumerates the names (NULL past the last one). */
int hn_tune_set(const char* name, int64_t value);
int hn_tune_get(const char* name, int64_t* value);
int hn_tune_reset(void);
const char* hn_tune_name(int32_t i);

/* ---- graph construction (HornetInit + gpu::Hornet(HornetInit&)) ----------
 * Replaces hornet::HornetInit(nV, nE, offsets, edges)
 * (hornet/include/Core/HornetInitialize/HornetInit.cuh:70-73) and
 * gpu::Hornet::Hornet(HornetInit&) / initialize()
 * (HornetInitialize/HornetInitialize.i.cuh:88-146).  The CSR is copied;
 * the caller keeps ownership.  `off` has nV+1 entries, `adj` nE entries.
 * Adjacency lists are stored sorted (sorted on the device unless
 * HN_CSR_SORTED says they already are). `device` = CUDA ordinal. */
int hn_graph_create_csr(int32_t nV, int64_t nE, const int32_t* off,
                        const int32_t* adj, unsigned flags, int mem,
                        int device, hn_graph_t** out);
/* Same with int64 offsets, for graphs with more than 2^31-1 edges. */
int hn_graph_create_csr64(int32_t nV, int64_t nE, const int64_t* off,
                          const int32_t* adj, unsigned flags, int mem,
                          int device, hn_graph_t** out);
/* A weighted graph: one 32-bit value per edge (an int32, a float's bits,
 * ...), the HornetInit::insertEdgeData(...) form of the reference with one
 * EdgeMetaType (hornet/include/Core/HornetInitialize/HornetInit.cuh:79-97,
 * HornetInsertTestWeighted.cu).  weights[i] belongs to adj[i] and is in
 * `mem`.  Updates carry the batch's weights (hn_batch_create_w; edges of an
 * unweighted batch get 0); BFS, TC, CC and k-truss ignore them.
 * hn_graph_reset_csr makes the graph unweighted. */
int hn_graph_create_csr_w(int32_t nV, int64_t nE, const int32_t* off, const int32_t* adj,
                          const uint32_t* weights, unsigned flags, int mem, int device,
                          hn_graph_t** out);
int hn_graph_weighted(const hn_graph_t* g, int32_t* weighted);
/* gpu::Hornet::reset(HornetInit&) (HornetInitialize.i.cuh:190-204). */
int hn_graph_reset_csr(hn_graph_t* g, int32_t nV, int64_t nE, const int32_t* off,
                       const int32_t* adj, unsigned flags, int mem);
int hn_graph_destroy(hn_graph_t* g);
/* Use `stream` (a cudaStream_t) for this graph's work; NULL = a private
 * stream created with the graph. */
int hn_graph_set_stream(hn_graph_t* g, void* stream);

/* ---- query views (no reference counterpart) ------------------------------
 * A query view shares the graph's vertex table and edge pool read-only and
 * owns its stream (`stream`, a cudaStream_t; NULL = a private one) and its
 * scratch, so read-only calls on different views of one graph -- BFS
 * (hn_bfs, hn_bfs_multi, hn_bfs_do, hn_bfs_batch), hn_tc_local, hn_tc,
 * hn_cc, the exports -- run concurrently on the device, from different
 * host threads.  The reference has one HornetGraph and synchronous calls,
 * so concurrent queries on one resident graph have no counterpart there.
 * Updates go to the graph itself; a view rejects them (HN_ERR_STATE).
 * Any handle, graph or view, serves one host thread at a time: a
 * traversal, count or update called on a handle that another thread's call
 * is using returns HN_ERR_STATE without touching it; concurrent queries
 * use one view per thread.
 * While the graph is being updated no call may run on its views; after the
 * update, hn_graph_view_refresh takes the graph's new edge count (it waits
 * for the graph's stream).  hn_graph_destroy frees a view; a view must be
 * destroyed before its graph. */
int hn_graph_view_create(hn_graph_t* g, void* stream, hn_graph_t** view);
int hn_graph_view_refresh(hn_graph_t* view);

/* out[i] = src[idx[i]] for device int32 array src (e.g. a row of BFS
 * distances) and host index / output arrays, on g's stream. */
int hn_gather_int32(hn_graph_t* g, const int32_t* src, const int64_t* idx, int64_t n,
                    int32_t* out);
/* out[i] = sum of values[off[i] .. off[i+1]) for i < nseg: device uint64
 * values and out, host ranges (nseg + 1 increasing offsets), on g's stream
 * (synchronised).  Per-graph sums of per-vertex counts for a batch of graphs
 * laid out side by side (hn_tc_owner's counts over a disjoint union). */
int hn_segment_sum_u64(hn_graph_t* g, const uint64_t* values, const int64_t* off, int64_t nseg,
                       uint64_t* out);
/* Measured read bandwidth (GB/s) of a device buffer of `bytes` (16-byte
 * aligned, at least 4 KB) read `reps` times after a first pass: a buffer that
 * fits in L2 gives the L2 read bandwidth that L2-served kernels (the
 * triangle count's list intersections) are measured against.  Diagnostic;
 * synchronises g's stream. */
int hn_read_bandwidth(hn_graph_t* g, const void* buf, int64_t bytes, int32_t reps, double* gbs);

/* ---- queries (hornet/include/Core/Hornet.cuh:113-127,
 *               HornetOperations/HornetQuery.i.cuh) ------------------------ */
int hn_graph_nv(const hn_graph_t* g, int32_t* nV);
int hn_graph_ne(const hn_graph_t* g, int64_t* nE);
/* max_degree() and max_degree_id(): lowest id among ties, as
 * thrust::max_element (HornetQuery.i.cuh:10-21,23-44). */
int hn_graph_max_degree(hn_graph_t* g, int32_t* max_degree, int32_t* max_id);
/* getCOO(true): (src,dst) sorted lexicographically, nE entries each
 * (HornetQuery.i.cuh:67-109).  Adjacency is always sorted here, so
 * `sorted` only documents intent. */
int hn_graph_export_coo(hn_graph_t* g, int sorted, int32_t* src, int32_t* dst,
                        int mem);
/* getCOO with the edge weights of a weighted graph (HornetInit::
 * insertEdgeData + getCOO, HornetInit.cuh:79-97, HornetQuery.i.cuh:67-109,
 * for one 32-bit field): weights[i] belongs to (src[i], dst[i]); equal
 * (src, dst) pairs keep their insertion order. */
int hn_graph_export_coo_w(hn_graph_t* g, int sorted, int32_t* src, int32_t* dst,
                          uint32_t* weights, int mem);
/* getCSR(true) (HornetQuery.i.cuh:111-151): off[nV+1], adj[nE]. */
int hn_graph_export_csr(hn_graph_t* g, int32_t* off, int32_t* adj, int mem);
/* Degrees of all vertices (int32[nV]). */
int hn_graph_degrees(hn_graph_t* g, int32_t* deg, int mem);
/* hornet.device() (Hornet.cuh:117): raw device view for user kernels. */
int hn_graph_device_view(hn_graph_t* g, hn_device_view_t* view);
/* Order-independent checksum of the graph's edge multiset, computed on the
 * device: the sum over stored edges (u, v) of SplitMix64((u << 32) | v),
 * modulo 2^64 (a validation aid with no reference counterpart: the
 * reference's tests compare whole sorted COO exports, HornetInsertTest.cu:
 * 42-75, which at full size means gigabytes on the host). */
int hn_graph_adjacency_hash(hn_graph_t* g, uint64_t* hash);
/* Slots held by the edge pool and by live blocks (for accounting). */
int hn_graph_memory(hn_graph_t* g, int64_t* pool_slots, int64_t* used_slots,
                    int64_t* free_list_blocks);

/* ---- batches (BatchUpdatePtr + gpu::BatchUpdate) -----------------------
 * Replaces BatchUpdatePtr<int, EMPTY, HOST|DEVICE>(n, src, dst)
 * (hornet/include/Core/BatchUpdate/BatchUpdate.cuh:91-99) and
 * gpu::BatchUpdate(ptr), which copies into owned device buffers
 * (BatchUpdate.i.cuh:154-184). */
int hn_batch_create(hn_graph_t* g, int64_t n, const int32_t* src,
                    const int32_t* dst, int mem, hn_batch_t** out);
/* Refill an existing batch (BatchUpdate::reset). */
int hn_batch_reset(hn_batch_t* b, int64_t n, const int32_t* src,
                   const int32_t* dst, int mem);
/* A batch with one 32-bit weight per edge (BatchUpdatePtr with one
 * EdgeMetaType, BatchUpdate.cuh:91-99); weights are in `mem`.  Inserted
 * edges take their batch weight; erase ignores weights. */
int hn_batch_create_w(hn_graph_t* g, int64_t n, const int32_t* src, const int32_t* dst,
                      const uint32_t* weights, int mem, hn_batch_t** out);
int hn_batch_reset_w(hn_batch_t* b, int64_t n, const int32_t* src, const int32_t* dst,
                     const uint32_t* weights, int mem);
int hn_batch_size(const hn_batch_t* b, int64_t* n);
int hn_batch_destroy(hn_batch_t* b);

/* gpu::Hornet::insert(batch, removeBatchDuplicates, removeGraphDuplicates)
 * (hornet/include/Core/HornetOperations/HornetInsert.i.cuh:12-27).
 * flags: HN_DEDUP_BATCH | HN_DEDUP_GRAPH.  Multiset semantics: without
 * flags every batch edge is added; HN_DEDUP_GRAPH drops the first copy of
 * each batch edge already in the graph.  *applied = edges added.
 * Ids outside [0,nV) -> HN_ERR_INVALID and the graph is unchanged. */
int hn_insert(hn_graph_t* g, hn_batch_t* b, unsigned flags, int64_t* applied);
/* gpu::Hornet::erase(batch, removeBatchDuplicates)
 * (HornetInsert.i.cuh:71-89): each distinct (u,v) removes
 * min(batch multiplicity, graph multiplicity) copies.  *applied = edges
 * removed. */
int hn_erase(hn_graph_t* g, hn_batch_t* b, unsigned flags, int64_t* applied);

/* Insert with both dedup flags (as hn_insert) and count the triangles the
 * insert created: *new_triangles = T(after) - T(before).  For an undirected
 * simple graph and a batch holding both directions of every edge (the
 * incremental triangle count after each insert of the dynamic-update
 * workload; the reference has no dynamic triangle counting, and
 * TriangleCounting2 (hornetsnest/src/Static/TriangleCounting/triangle2.cu)
 * recounts the whole graph). */
int hn_insert_count_triangles(hn_graph_t* g, hn_batch_t* b, int64_t* applied,
                              uint64_t* new_triangles);

/* A run of update batches applied as one: entry i inserts (ops[i] != 0) or
 * erases (ops[i] == 0) edge (src[i], dst[i]), the entries in the order the
 * batches arrived.  On a simple graph the result equals applying the
 * entries in order with insert(removeBatchDuplicates,
 * removeGraphDuplicates) and erase(removeBatchDuplicates)
 * (HornetInsert.i.cuh:12-27, HornetDelete.i.cuh:12-37): the last entry of
 * each edge decides its presence.  The net erase set is applied, then the
 * net insert set.  src/dst/ops are all in `mem`.  *inserted / *erased
 * (may be NULL) receive the edges actually added and removed. */
int hn_update_coalesced(hn_graph_t* g, int64_t n, const int32_t* src, const int32_t* dst,
                        const uint8_t* ops, int mem, int64_t* inserted, int64_t* erased);

/* ---- algorithms (hornetsnest StaticAlgorithm subclasses) -------------- */

/* BfsTopDown: set_parameters(src) + run()
 * (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:80-106).
 * dist: int32[nV], INT32_MAX when unreachable.  stats may be NULL. */
int hn_bfs(hn_graph_t* g, int32_t src, int32_t* dist, int mem,
           hn_bfs_stats_t* stats);
/* k independent BFS runs (one per source); dist is int32[k][nV]
 * row-major; stats (may be NULL) has k entries. */
int hn_bfs_multi(hn_graph_t* g, const int32_t* sources, int32_t k,
                 int32_t* dist, int mem, hn_bfs_stats_t* stats);

/* Direction-optimising BFS (top-down levels switch to bottom-up ones while
 * the frontier is large; the counterpart of hornetsnest's BottomUpBFS,
 * src/Static/BottomUpBreadthFirstSearch/BottomUpBFS.cu).  Same arguments
 * and the same distances as hn_bfs_multi; stats count the same edges
 * (sum of degrees of reached vertices), although fewer are read. */
int hn_bfs_do(hn_graph_t* g, const int32_t* sources, int32_t k, int32_t* dist,
              int mem, hn_bfs_stats_t* stats);

/* Instrumentation: per-level device time (microseconds, from the GPU's
 * global timer at each level's end inside the BFS CUDA graph) and frontier
 * edges of the latest hn_bfs / hn_bfs_multi / hn_bfs_do source on this
 * graph, for its first min(levels, max_levels, 32) levels.  us and edges
 * may be NULL.  No reference counterpart (the reference times whole runs
 * with Timer<DEVICE>, hornetsnest/test/BFSTest.cu:35-43). */
int hn_bfs_level_trace(hn_graph_t* g, int32_t max_levels, double* us, int64_t* edges,
                       int32_t* n_levels);

/* Batched BFS: up to 64 BFS "slots" traversed together, one 64-bit mask
 * per vertex, each edge read once per level for all slots on it.  Source j
 * seeds slot slots[j] (slots NULL: slot j, k <= nslots); a slot seeded by
 * several sources gets the distance to the nearest of them, which on a
 * disjoint union of graphs with one source per graph per slot is each
 * graph's own BFS.  dist is int32[nslots][nV] row-major (INT32_MAX when
 * unreachable); slot_stats (may be NULL) has nslots entries.  With one
 * source per slot the result equals hn_bfs_multi on the same sources.
 * Batches the reference's per-source BfsTopDown::run
 * (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:88-106). */
int hn_bfs_batch(hn_graph_t* g, const int32_t* sources, const int32_t* slots,
                 int32_t k, int32_t nslots, int32_t* dist, int mem,
                 hn_bfs_stats_t* slot_stats);

/* TriangleCounting2::init/run/countTriangles
 * (hornetsnest/src/Static/TriangleCounting/triangle2.cu:130-171) on the
 * graph's undirected adjacency, each triangle counted once via the
 * degree orientation of xlib/src/Graph/GraphStd.cpp:247-268.
 * per_vertex (may be NULL): uint64[nV], triangles containing each vertex.
 * per_vertex uses `mem`; *total is always host. */
int hn_tc(hn_graph_t* g, uint64_t* per_vertex, int mem, uint64_t* total);

/* Local triangle counts: counts[i] = number of triangles containing
 * seeds[i] — TriangleCounting2's per-vertex count
 * (hornetsnest/src/Static/TriangleCounting/triangle2.cu:30-59) for the
 * seeds only, without counting the rest of the graph.  The graph must be
 * simple (no self loops or repeated edges).  seeds and counts are both in
 * `mem`; counts is uint64[k]. */
int hn_tc_local(hn_graph_t* g, const int32_t* seeds, int32_t k, uint64_t* counts, int mem);
/* Owner counts: counts[v] = triangles whose lowest vertex in the degree
 * orientation is v, so each triangle is credited exactly once (sums over
 * any vertex set that contains whole triangles, e.g. one graph of a
 * disjoint union, are that set's triangle count).  Cheaper than the
 * per-vertex form of hn_tc (one atomic per vertex, not three per
 * triangle).  No reference counterpart; counts is uint64[nV] in `mem`. */
int hn_tc_owner(hn_graph_t* g, uint64_t* counts, int mem, uint64_t* total);

/* CC::run (hornetsnest/src/Static/ConnectedComponents/CC.cu:133-156).
 * mode HN_CC_MIN_ID or HN_CC_REFERENCE.  labels: int32[nV];
 * *n_components (may be NULL) is host. */
int hn_cc(hn_graph_t* g, int mode, int32_t* labels, int mem,
          int32_t* n_components);

/* KTruss::run / getMaxK (hornetsnest/src/Static/KTruss/KTruss.cu:90-174)
 * on a simple undirected graph.  edge_truss (may be NULL): int32[nE] in
 * sorted-COO order, the largest k whose k-truss holds the edge (2 if none).
 * *max_k is host. */
int hn_ktruss(hn_graph_t* g, int32_t* max_k, int32_t* edge_truss, int mem);
/* KTruss::runForKDynamic(K) (hornetsnest/src/Static/KTruss/KTruss.cu:
 * 270-295): the graph keeps only its K-truss.  Every edge whose truss
 * number is below K is erased from the dynamic graph through the update
 * pipeline (the reference peels by deleteEdgeBatch the same way).
 * *max_k (may be NULL) receives the graph's max K before the erase,
 * *removed (may be NULL) the directed edges erased. */
int hn_ktruss_keep(hn_graph_t* g, int32_t K, int32_t* max_k, int64_t* removed);

/* ---- result certificates (StaticAlgorithm::validate) --------------------
 * The reference's validate() methods return true without checking
 * (hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu:113-128,
 * ConnectedComponents/CC.cu:163-203).  These check a result on the device
 * without recomputing it; *violations = number of failed conditions (0:
 * the result is certified).  Arrays are in `mem`.
 * hn_bfs_validate: dist (int32[nV]) are the BFS distances from src iff
 *   dist[src] == 0, no edge from a reached vertex leads to an unreached one
 *   or skips a level, and every other reached vertex has an in-edge from
 *   the level before.
 * hn_cc_validate: min-id labels (int32[nV]) of an undirected graph:
 *   constant along edges, labels[v] <= v, labels[labels[v]] == labels[v],
 *   and propagating the roots' labels along edges reproduces them.
 * hn_ktruss_validate: edge truss numbers (int32[nE], sorted-COO order) of a
 *   simple undirected graph: in [2, max_k] with max_k attained, equal on
 *   both directions, and every edge numbered t >= 3 in >= t-2 triangles
 *   whose other edges are numbered >= t (the edges numbered >= t form a
 *   t-truss; maximality is not checked). */
int hn_bfs_validate(hn_graph_t* g, int32_t src, const int32_t* dist, int mem,
                    int64_t* violations);
int hn_cc_validate(hn_graph_t* g, const int32_t* labels, int mem, int64_t* violations);
int hn_ktruss_validate(hn_graph_t* g, int32_t max_k, const int32_t* edge_truss, int mem,
                       int64_t* violations);

/* ---- operator primitives with built-in operators -----------------------
 * forAllEdges(hornet, vertex_array, size, op, lb) with the BinarySearch or
 * VertexBased<vw> load balancer (primitives/Operator++.cuh:143-215,
 * LoadBalancing/BinarySearch.i.cuh:58-107, VertexBased.i.cuh:43-89) running
 * the built-in "count" operator: out[dst] += 1 for every edge (src,dst) of
 * each listed vertex (vertices == NULL: all vertices).  out: int32[nV]
 * device, accumulated.  User operators use the C++ header
 * <hornet_b200/Operator++.cuh> instead. */
int hn_for_all_edges_count(hn_graph_t* g, const int32_t* vertices, int32_t n,
                           int lb, int vw, int32_t* out);
/* forAllVertices(hornet, op) with the built-in "degree" operator:
 * out[v] = degree(v) (Operator++.i.cuh:524-540). out: int32[nV] device. */
int hn_for_all_vertices_degree(hn_graph_t* g, int32_t* out);

/* ---- on-disk formats ------------------------------------------------------
 * GraphStd binary (.bin): the reference's fast-reload format
 * (xlib/src/Graph/GraphStd.cpp:389-420 writeBinary,
 * xlib/src/Graph/GraphStdRead.cpp:212-245 readBinary) for int ids and
 * offsets.  hn_csr_read_bin with off == NULL only reports nV and nE; call
 * again with off[nV+1] and adj[nE] host buffers.  Files written with
 * in-edges (DIRECTED | ENABLE_INGOING) are read for their out-edges. */
int hn_csr_write_bin(const char* path, int32_t nV, int32_t nE, const int32_t* off,
                     const int32_t* adj);
int hn_csr_read_bin(const char* path, int32_t* nV, int32_t* nE, int32_t* off,
                    int32_t* adj);
/* Matrix Market coordinate pattern general, 1-based (the format GraphStd's
 * Market reader takes, GraphStdRead.cpp:46-61).  Host CSR. */
int hn_csr_write_mtx(const char* path, int32_t nV, int64_t nE, const int32_t* off,
                     const int32_t* adj);
/* getCSR + writeBinary / readBinary + HornetInit for a device graph. */
int hn_graph_write_bin(hn_graph_t* g, const char* path);
int hn_graph_read_bin(const char* path, int device, hn_graph_t** out);

/* ---- connected components without device allocation ---------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a host framework that owns all device memory, a service whose
 * memory budget is fixed up front, a loop that cannot afford the implicit
 * synchronisation of cudaMalloc/cudaFree): the same labels as
 * hn_cc(HN_CC_MIN_ID) computed over a caller-owned device CSR
 * (off[nV+1], adj[off[nV]]) into a caller-owned device array labels[nV],
 * with no cudaMalloc/cudaFree and no allocating library call.
 * The CSR must be undirected and symmetric (each edge stored in both
 * endpoints' lists), as hn_cc's graphs are; a one-sided CSR gives wrong
 * labels without an error.  The offsets (off[0] == 0, never decreasing) and
 * every id of adj[0, off[nV]) are checked on the device first:
 * HN_ERR_INVALID, and labels not written, when they are malformed.
 * Its only working memory is a 16 MiB static device array inside the
 * library, so nV is limited to 4,194,304 (HN_ERR_CAPACITY above that).  The
 * first call on a device resolves that array's address: make it before any
 * stream capture.  All calls share the array; calls that overlap on the GPU
 * race.  `stream` is a cudaStream_t (NULL = legacy default stream); the call
 * returns when the labels are ready.  *n_components (may be NULL) is host. */
int hn_cc_csr_noalloc(int32_t nV, const int32_t* off, const int32_t* adj,
                      int32_t* labels, int32_t* n_components, void* stream);

/* ---- synthetic inputs (not part of the reference API) --------------------
 * R-MAT edge pairs (a,b,c; d = 1-a-b-c) from a counter-based generator:
 * pair i depends only on (seed, i), so the host and device versions give
 * identical arrays.  n_vertices may be below 2^scale: endpoints >= n are
 * redrawn.  src/dst: int32[np]. */
int hn_gen_rmat_host(int32_t scale, int32_t n_vertices, int64_t np, double a,
                     double b, double c, uint64_t seed, int32_t* src,
                     int32_t* dst);
int hn_gen_rmat_device(int32_t scale, int32_t n_vertices, int64_t np, double a,
                       double b, double c, uint64_t seed, int32_t* src,
                       int32_t* dst, int device);
/* Undirected CSR on the device from an edge-pair list: mirror, drop self
 * loops, sort, dedup (the GPU counterpart of GraphStd's COOtoCSR,
 * xlib/src/Graph/GraphStd.cpp:174-206).  src/dst are device arrays of np
 * pairs.  *off_out / *adj_out receive device buffers allocated with
 * cudaMalloc (free with hn_free_device); *nE_out is the edge count. */
int hn_coo_to_csr_device(int32_t nV, int64_t np, const int32_t* src,
                         const int32_t* dst, int device, int32_t** off_out,
                         int32_t** adj_out, int64_t* nE_out);
int hn_free_device(void* p);

#ifdef __cplusplus
}
#endif
#endif /* HORNET_B200_H */
