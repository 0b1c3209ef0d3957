// Drop-in check of the C++ shim: reference-style code (the call shapes of
// hornet/test/HornetInsertTest.cu, HornetDeleteTest.cu and
// hornetsnest/src/Static/BreadthFirstSearch/TopDown.cu) compiled for
// sm_100a against <hornet_b200/hornet.cuh> and linked with the library.
//
//   shim_test <csr_file> <batch_file> <out_prefix>
// csr_file:   int64 nV, int64 nE, int32 off[nV+1], int32 adj[nE]
// batch_file: int64 n, int32 src[n], int32 dst[n]
// Writes <out_prefix>.bfs (int32 dist[nV] from vertex 0 by a user-written
// BFS operator), <out_prefix>.deg (int32 VertexBased<4> edge counts) and
// prints PASSED / NOT PASSED for the insert and delete checks.
#include <hornet_b200/hornet.cuh>

#include <cstdio>
#include <vector>

using vert_t = int;
using HornetGPU = hornet::gpu::Hornet<vert_t>;
using UpdatePtr = hornet::BatchUpdatePtr<vert_t, hornet::EMPTY, hornet::DeviceType::HOST>;
using Update = hornet::gpu::BatchUpdate<vert_t>;
using Init = hornet::HornetInit<vert_t>;
using namespace hornets_nest;

static const int INF = 2147483647;

// the reference's BFSOperator shape (TopDown.cu:49-61), made race-free with
// atomicCAS so each vertex is enqueued once
struct BFSOperator {
    int* d_distances;
    int current_level;
    TwoLevelQueue<vert_t> queue;
    OPERATOR(Vertex& vertex, Edge& edge) {
        auto dst = edge.dst_id();
        if (d_distances[dst] == INF && atomicCAS(d_distances + dst, INF, current_level) == INF)
            queue.insert(dst);
    }
};

struct CountOp {
    int* counts;
    OPERATOR(Vertex& vertex, Edge& edge) { atomicAdd(counts + vertex.id(), 1); }
};

static bool read_file(const char* p, std::vector<char>& b) {
    FILE* f = std::fopen(p, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    b.resize(std::ftell(f));
    std::fseek(f, 0, SEEK_SET);
    bool ok = std::fread(b.data(), 1, b.size(), f) == b.size();
    std::fclose(f);
    return ok;
}

template <typename C>
static bool same(const C& a, const C& b) {
    hornet::COO<hornet::DeviceType::HOST, vert_t> x(a), y(b);
    if (x.size() != y.size()) return false;
    for (size_t i = 0; i < x.size(); i++)
        if (x.srcPtr()[i] != y.srcPtr()[i] || x.dstPtr()[i] != y.dstPtr()[i]) return false;
    return true;
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    std::vector<char> cb, bb;
    if (!read_file(argv[1], cb) || !read_file(argv[2], bb)) return 2;
    long long nV = ((long long*)cb.data())[0], nE = ((long long*)cb.data())[1];
    const int* off = (const int*)(cb.data() + 16);
    const int* adj = off + nV + 1;
    long long nb = ((long long*)bb.data())[0];
    std::vector<int> bs((int*)(bb.data() + 8), (int*)(bb.data() + 8) + nb);
    std::vector<int> bd((int*)(bb.data() + 8) + nb, (int*)(bb.data() + 8) + 2 * nb);

    Init init((int)nV, (int)nE, off, adj);
    HornetGPU hornet_gpu(init);

    // HornetInsertTest: getCOO(true) after insert == (init ∪ batch) sorted
    auto init_coo = hornet_gpu.getCOO(true);
    hornet::COO<hornet::DeviceType::HOST, vert_t> batch_coo(nb);
    for (long long i = 0; i < nb; i++) { batch_coo.srcPtr()[i] = bs[i]; batch_coo.dstPtr()[i] = bd[i]; }
    {
        Update up(UpdatePtr((int)nb, bs.data(), bd.data()));
        hornet_gpu.insert(up);
    }
    auto inst_coo = hornet_gpu.getCOO(true);
    auto expect = init_coo;
    expect.append(batch_coo);
    expect.sort();
    std::printf("insert %s\n", same(inst_coo, expect) ? "PASSED" : "NOT PASSED");

    // HornetDeleteTest: getCOO(true) after erase ∪ batch == before
    {
        Update up(batch_coo);
        hornet_gpu.erase(up);
    }
    auto del_coo = hornet_gpu.getCOO(true);
    del_coo.append(batch_coo);
    del_coo.sort();
    std::printf("erase %s\n", same(del_coo, inst_coo) ? "PASSED" : "NOT PASSED");

    // a user-written BFS over forAllEdges + TwoLevelQueue + BinarySearch
    int* d_dist = nullptr;
    cudaMalloc(&d_dist, sizeof(int) * nV);
    forAllnumV(hornet_gpu, [=] __device__(int i) { d_dist[i] = INF; });
    cudaMemset(d_dist, 0, sizeof(int));
    TwoLevelQueue<vert_t> queue(hornet_gpu);
    load_balancing::BinarySearch lb(hornet_gpu);
    queue.insert(0);
    int level = 1;
    while (queue.size() > 0) {
        forAllEdges(hornet_gpu, queue, BFSOperator{d_dist, level, queue}, lb);
        queue.swap();
        level++;
    }
    std::vector<int> dist(nV);
    cudaMemcpy(dist.data(), d_dist, sizeof(int) * nV, cudaMemcpyDeviceToHost);
    std::string p = std::string(argv[3]) + ".bfs";
    FILE* f = std::fopen(p.c_str(), "wb");
    std::fwrite(dist.data(), 4, nV, f);
    std::fclose(f);

    // forAllEdges with VertexBased<4>: per-vertex edge counts == degrees
    int* d_cnt = nullptr;
    cudaMalloc(&d_cnt, sizeof(int) * nV);
    cudaMemset(d_cnt, 0, sizeof(int) * nV);
    forAllEdges(hornet_gpu, CountOp{d_cnt}, load_balancing::VertexBased4());
    std::vector<int> cnt(nV);
    cudaMemcpy(cnt.data(), d_cnt, sizeof(int) * nV, cudaMemcpyDeviceToHost);
    p = std::string(argv[3]) + ".deg";
    f = std::fopen(p.c_str(), "wb");
    std::fwrite(cnt.data(), 4, nV, f);
    std::fclose(f);

    // StaticAlgorithm classes
    BfsTopDown bfs(hornet_gpu);
    bfs.set_parameters(0);
    bfs.run();
    std::vector<int> d2(nV);
    cudaMemcpy(d2.data(), bfs.distances(), sizeof(int) * nV, cudaMemcpyDeviceToHost);
    std::printf("bfs_class %s\n", d2 == dist ? "PASSED" : "NOT PASSED");
    CC cc(hornet_gpu);
    cc.run_min_label();
    std::printf("cc_components %d\n", cc.components());
    // KTruss on a fresh copy of the (simple, symmetric) input graph:
    // runForKDynamic(3) keeps exactly the edges whose truss number is >= 3
    {
        HornetGPU kg(init);
        KTruss kt(kg);
        kt.init();
        kt.run();
        std::printf("ktruss_validate %s\n", kt.validate() ? "PASSED" : "NOT PASSED");
        long long at_least3 = 0;
        for (int t : kt.edgeTruss()) at_least3 += t >= 3;
        const int maxk = kt.getMaxK();
        kt.runForK(3);
        std::vector<int> koff((size_t)nV + 1);
        kt.copyOffsetArrayHost(koff.data());
        const bool off_ok = koff[(size_t)nV] == at_least3;
        kt.runForKDynamic(3);
        const bool ok = off_ok && (long long)kg.nE() == at_least3 && kt.getMaxK() == maxk;
        std::printf("ktruss_max %d\nktruss_keep %s\n", maxk, ok ? "PASSED" : "NOT PASSED");
    }
    // validate() of each algorithm on the (symmetric) input graph
    {
        HornetGPU vg(init);
        BfsTopDown b2(vg);
        b2.set_parameters(0);
        b2.run();
        CC c2(vg);
        c2.run();
        TriangleCounting2 t2(vg);
        t2.init();
        t2.run();
        const bool ok = b2.validate() && c2.validate() && t2.validate();
        std::printf("validate %s\n", ok ? "PASSED" : "NOT PASSED");
    }
    cudaFree(d_dist);
    cudaFree(d_cnt);
    cudaError_t e = cudaDeviceSynchronize();
    std::printf("cuda %s\n", cudaGetErrorString(e));
    return e == cudaSuccess ? 0 : 1;
}
