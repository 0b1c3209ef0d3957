// Degree-oriented graph used by triangle counting.
#pragma once

#include "hn_graph.cuh"

namespace hn {

struct Oriented {
    DevBuf<long long> prefix;  // degree prefix of the undirected graph (nV+1)
    DevBuf<long long> offp;    // oriented offsets (nV+1)
    DevBuf<int32_t> fwd;       // oriented, sorted neighbour lists
    DevBuf<int32_t> feid;      // edge id of each fwd entry (when built with canon)
};

// Build N+(u) = {v in N(u) : (deg u, u) < (deg v, v)} for every vertex.
// With canon (an id per CSR position, nE entries), feid[p] = canon of the
// CSR position the oriented entry p came from.
void build_oriented(hn_graph* g, Oriented& o, const int32_t* canon = nullptr);

// Triangles of the oriented graph.  With d_counts (device array of nV
// entries): mode 1 = per-vertex counts (each triangle credited to its three
// vertices), mode 2 = owner counts (each triangle credited once, to its
// lowest vertex in the orientation).  Synchronises.
unsigned long long count_triangles(hn_graph* g, const Oriented& o,
                                   unsigned long long* d_counts, int mode = 1);

// Edge support: sup[id] += the triangles through the edge with that id, for
// the ids build_oriented(g, o, canon) recorded (sup zeroed by the caller).
// Returns the triangle total.  Synchronises.
unsigned long long edge_support(hn_graph* g, const Oriented& o, int32_t* sup);

}  // namespace hn
