// TEST INFRASTRUCTURE: times the reference's own GPU batch update
// (hornet::gpu::Hornet::insert / erase, hornet/include/Core/Hornet.cuh:107-109,
// implemented in hornet/include/Core/BatchUpdate/BatchUpdate.i.cuh) on this
// GPU.  Built by `make -C oracle ref_gpu` against the reference's headers
// where they lie; nothing of the reference is copied here.  The reference's
// own update tests (hornet/test/HornetInsertTest.cu, HornetDeleteTest.cu)
// check one batch and print no time, so this driver makes the same calls
// the way those tests do (HornetInit from a GraphStd CSR, a BatchUpdate from
// a BatchUpdatePtr, Hornet::insert / Hornet::erase) and times each call.
//
//   ref_gpu_update <graph.bin> <batch file>...
//
// A batch file is int64 n, then int32 src[n], int32 dst[n].  Each batch is
// inserted (removeBatchDuplicates and removeGraphDuplicates set) and then
// erased (removeBatchDuplicates set), in file order, as one sequence on one
// graph.  One JSON line per batch: n, the insert and erase device times
// (CUDA events around the call on the legacy default stream, which the
// reference's update path uses) and nE after each call.
#include <Hornet.hpp>

#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <vector>

using vert_t = int;
using HornetGPU = hornet::gpu::Hornet<vert_t>;
using UpdatePtr = hornet::BatchUpdatePtr<vert_t, hornet::EMPTY, hornet::DeviceType::DEVICE>;
using Update = hornet::gpu::BatchUpdate<vert_t>;
using Init = hornet::HornetInit<vert_t>;

static bool check(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    std::printf("{\"error\": \"%s: %s\"}\n", what, cudaGetErrorString(e));
    std::fflush(stdout);
    return false;
}

static bool read_batch(const char* path, std::vector<int>& src, std::vector<int>& dst) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    long long n = 0;
    bool ok = std::fread(&n, sizeof(n), 1, f) == 1 && n >= 0;
    if (ok) {
        src.resize(n);
        dst.resize(n);
        ok = std::fread(src.data(), sizeof(int), n, f) == (size_t)n &&
             std::fread(dst.data(), sizeof(int), n, f) == (size_t)n;
    }
    std::fclose(f);
    return ok;
}

int main(int argc, char* argv[]) {
    if (argc < 3) {
        std::printf("usage: %s graph.bin batch...\n", argv[0]);
        return 2;
    }
    graph::GraphStd<vert_t, vert_t> graph;
    graph.read(argv[1]);
    Init init(graph.nV(), graph.nE(), graph.csr_out_offsets(), graph.csr_out_edges());
    HornetGPU hornet(init);
    if (!check(cudaDeviceSynchronize(), "init")) return 1;
    std::printf("{\"nV\": %d, \"nE\": %lld}\n", (int)hornet.nV(), (long long)hornet.nE());
    std::fflush(stdout);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int i = 2; i < argc; i++) {
        std::vector<int> hs, hd;
        if (!read_batch(argv[i], hs, hd)) {
            std::printf("{\"error\": \"cannot read %s\"}\n", argv[i]);
            return 1;
        }
        const int n = (int)hs.size();
        int *ds = nullptr, *dd = nullptr;
        if (!check(cudaMalloc(&ds, sizeof(int) * (n ? n : 1)), "malloc") ||
            !check(cudaMalloc(&dd, sizeof(int) * (n ? n : 1)), "malloc"))
            return 1;
        cudaMemcpy(ds, hs.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
        cudaMemcpy(dd, hd.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
        float ms[2] = {0, 0};
        long long ne[2] = {0, 0};
        double wall[2] = {0, 0};
        for (int op = 0; op < 2; op++) {
            UpdatePtr ptr(n, ds, dd);
            Update update(ptr);
            if (!check(cudaDeviceSynchronize(), "batch")) return 1;
            const auto t0 = std::chrono::steady_clock::now();
            cudaEventRecord(a);
            if (op == 0)
                hornet.insert(update, true, true);
            else
                hornet.erase(update, true);
            cudaEventRecord(b);
            if (!check(cudaEventSynchronize(b), op ? "erase" : "insert")) return 1;
            wall[op] = std::chrono::duration<double, std::milli>(
                           std::chrono::steady_clock::now() - t0).count();
            cudaEventElapsedTime(&ms[op], a, b);
            ne[op] = (long long)hornet.nE();
        }
        if (!check(cudaGetLastError(), "update")) return 1;
        std::printf("{\"batch\": %d, \"insert_ms\": %.4f, \"erase_ms\": %.4f, "
                    "\"insert_wall_ms\": %.4f, \"erase_wall_ms\": %.4f, "
                    "\"nE_after_insert\": %lld, \"nE_after_erase\": %lld}\n",
                    n, ms[0], ms[1], wall[0], wall[1], ne[0], ne[1]);
        std::fflush(stdout);
        cudaFree(ds);
        cudaFree(dd);
    }
    return 0;
}
