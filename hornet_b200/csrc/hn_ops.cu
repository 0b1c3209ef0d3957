// Built-in operators over the operator primitives, exported through the C
// ABI.  They run the same header templates that user operators compile
// against (<hornet_b200/LoadBalancing.cuh>), so the C-ABI tests exercise
// the BinarySearch and VertexBased<VW> balancers themselves.
#include "../../include/hornet_b200/LoadBalancing.cuh"
#include "hn_graph.cuh"

namespace hn {
namespace {

// forAllEdges operator: out[dst] += 1 for every visited edge.
struct CountDst {
    int32_t* out;
    __device__ __forceinline__ void operator()(hornet::Vertex&, hornet::Edge& e) const {
        atomicAdd(out + e.dst_id(), 1);
    }
};

__global__ void k_vertex_degree(hornet::HornetDevice hd, int32_t* out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < hd.nV();
         v += (long long)gridDim.x * blockDim.x)
        out[v] = hd.vertex((int)v).degree();
}

hornet::HornetDevice view_of(hn_graph* g) {
    hn_device_view_t v;
    v.nV = g->nV;
    v.pad = 0;
    v.nE = g->nE;
    v.vtab = g->vtab;
    v.pool = g->pool;
    return hornet::HornetDevice(v);
}

template <unsigned VW>
void vertex_based(hn_graph* g, const int32_t* verts, long long n, int32_t* out) {
    hornets_nest::load_balancing::VertexBased<VW>::run(view_of(g), verts, n, CountDst{out},
                                                      g->stream);
    count_launch();
}

}  // namespace
}  // namespace hn

using namespace hn;

extern "C" int hn_for_all_edges_count(hn_graph_t* g, const int32_t* vertices, int32_t n, int lb,
                                      int vw, int32_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && out, "null argument");
    HN_REQUIRE(lb == HN_LB_BINARY_SEARCH || lb == HN_LB_VERTEX_BASED, "bad load balancer");
    HN_CUDA(cudaSetDevice(g->device));
    long long cnt = vertices ? n : g->nV;
    HN_REQUIRE(cnt >= 0, "negative vertex count");
    if (lb == HN_LB_BINARY_SEARCH) {
        hornets_nest::load_balancing::BinarySearch::run(view_of(g), vertices, cnt, CountDst{out},
                                                        g->stream);
        count_launch(2);
    } else {
        switch (vw) {
            case 1: vertex_based<1>(g, vertices, cnt, out); break;
            case 2: vertex_based<2>(g, vertices, cnt, out); break;
            case 4: vertex_based<4>(g, vertices, cnt, out); break;
            case 8: vertex_based<8>(g, vertices, cnt, out); break;
            case 16: vertex_based<16>(g, vertices, cnt, out); break;
            case 32: vertex_based<32>(g, vertices, cnt, out); break;
            default: throw Error(HN_ERR_INVALID, "vw must be a power of two in [1, 32]");
        }
    }
    HN_CUDA(cudaGetLastError());
    HN_CUDA(cudaStreamSynchronize(g->stream));
    HN_API_END
}

extern "C" int hn_for_all_vertices_degree(hn_graph_t* g, int32_t* out) {
    HN_API_BEGIN
    HN_REQUIRE(g && out, "null argument");
    HN_CUDA(cudaSetDevice(g->device));
    HN_LAUNCH(k_vertex_degree, grid_for(g, g->nV, 256), 256, 0, g->stream, view_of(g), out);
    HN_CUDA(cudaStreamSynchronize(g->stream));
    HN_API_END
}
