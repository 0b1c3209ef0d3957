// hornetsnest algorithm classes over the C ABI, with the reference's names
// and methods:
//   BfsTopDown        (Static/BreadthFirstSearch/TopDown.cuh:52-70)
//   TriangleCounting2 (Static/TriangleCounting/triangle2.cuh:18-37)
//   CC                (Static/ConnectedComponents/CC.cuh:53-69)
//   KTruss            (Static/KTruss/KTruss.cuh:12-92)
// validate() certifies the last result on the device through the C ABI
// (hn_bfs_validate, hn_cc_validate, hn_ktruss_validate; TC against its two
// other counting kernels), where the reference's BFS and CC validators are
// stubs that return true (TopDown.cu:113-128, CC.cu:163-203).
#pragma once

#include <cstdint>
#include <algorithm>
#include <vector>

#include "Hornet.cuh"
#include "HornetAlg.cuh"

namespace hornets_nest {

using vid_t = int;
using dist_t = int;
using color_t = int;
using triangle_t = unsigned long long;
using HornetGraph = ::hornet::gpu::Hornet<int>;
using HornetInit = ::hornet::HornetInit<int>;

class BfsTopDown : public StaticAlgorithm<HornetGraph> {
public:
    explicit BfsTopDown(HornetGraph& h) : StaticAlgorithm(h) {
        cudaMalloc(&d_distances, sizeof(dist_t) * (size_t)(h.nV() > 0 ? h.nV() : 1));
    }
    ~BfsTopDown() override { release(); }
    void reset() override { _levels = 0; }
    void set_parameters(vid_t source) { bfs_source = source; }
    void run() override {
        hn_bfs_stats_t st;
        ::hornet::hn_check(hn_bfs(hornet.handle(), bfs_source, d_distances, HN_MEM_DEVICE, &st));
        _levels = st.levels;
    }
    void release() override {
        if (d_distances) cudaFree(d_distances);
        d_distances = nullptr;
    }
    bool validate() override {
        int64_t bad = -1;
        return _levels > 0 &&
               hn_bfs_validate(hornet.handle(), bfs_source, d_distances, HN_MEM_DEVICE, &bad) ==
                   HN_OK &&
               bad == 0;
    }
    dist_t getLevels() const { return _levels; }
    const dist_t* distances() const { return d_distances; }  // device

private:
    dist_t* d_distances = nullptr;
    vid_t bfs_source = 0;
    dist_t _levels = 0;
};

class TriangleCounting2 : public StaticAlgorithm<HornetGraph> {
public:
    explicit TriangleCounting2(HornetGraph& h) : StaticAlgorithm(h) {}
    ~TriangleCounting2() override { release(); }
    void init() {
        cudaMalloc(&triPerVertex, sizeof(triangle_t) * (size_t)(hornet.nV() > 0 ? hornet.nV() : 1));
        reset();
    }
    void reset() override { _total = 0; }
    void run() override { run(1); }
    void run(const int /*work_factor*/) {
        uint64_t t = 0;
        ::hornet::hn_check(hn_tc(hornet.handle(), (uint64_t*)triPerVertex,
                                 HN_MEM_DEVICE, &t));
        _total = t;
    }
    triangle_t countTriangles() { return _total; }
    void copyTCToHost(triangle_t* h) {
        cudaMemcpy(h, triPerVertex, sizeof(triangle_t) * hornet.nV(), cudaMemcpyDeviceToHost);
    }
    void release() override {
        if (triPerVertex) cudaFree(triPerVertex);
        triPerVertex = nullptr;
    }
    // the total against the owner counts (each triangle credited once) and
    // the per-vertex counts (three credits per triangle)
    bool validate() override {
        uint64_t owner = 0, t = 0;
        std::vector<uint64_t> pv((size_t)(hornet.nV() > 0 ? hornet.nV() : 1));
        if (hn_tc_owner(hornet.handle(), pv.data(), HN_MEM_HOST, &owner) != HN_OK) return false;
        if (hn_tc(hornet.handle(), pv.data(), HN_MEM_HOST, &t) != HN_OK) return false;
        uint64_t sum = 0;
        for (int32_t v = 0; v < hornet.nV(); v++) sum += pv[(size_t)v];
        return owner == _total && t == _total && sum == 3 * _total;
    }

private:
    triangle_t* triPerVertex = nullptr;
    triangle_t _total = 0;
};

class CC : public StaticAlgorithm<HornetGraph> {
public:
    explicit CC(HornetGraph& h) : StaticAlgorithm(h) {
        cudaMalloc(&d_colors, sizeof(color_t) * (size_t)(h.nV() > 0 ? h.nV() : 1));
    }
    ~CC() override { release(); }
    void reset() override {}
    // the reference's colouring (giant component 0, others max(id)+1)
    void run() override {
        ::hornet::hn_check(hn_cc(hornet.handle(), HN_CC_REFERENCE, d_colors, HN_MEM_DEVICE,
                                 &_ncomp));
    }
    // canonical labels (minimum vertex id per component)
    void run_min_label() {
        ::hornet::hn_check(hn_cc(hornet.handle(), HN_CC_MIN_ID, d_colors, HN_MEM_DEVICE, &_ncomp));
    }
    void release() override {
        if (d_colors) cudaFree(d_colors);
        d_colors = nullptr;
    }
    // certifies minimum-id labels (run_min_label); the reference colouring
    // of run() is certified through the min-id labels of the same graph
    bool validate() override {
        color_t* lab = nullptr;
        if (cudaMalloc(&lab, sizeof(color_t) * (size_t)(hornet.nV() > 0 ? hornet.nV() : 1)) !=
            cudaSuccess)
            return false;
        int64_t bad = -1;
        int32_t n = 0;
        bool ok = hn_cc(hornet.handle(), HN_CC_MIN_ID, lab, HN_MEM_DEVICE, &n) == HN_OK &&
                  hn_cc_validate(hornet.handle(), lab, HN_MEM_DEVICE, &bad) == HN_OK &&
                  bad == 0 && n == _ncomp;
        cudaFree(lab);
        return ok;
    }
    const color_t* colors() const { return d_colors; }  // device
    int32_t components() const { return _ncomp; }

private:
    color_t* d_colors = nullptr;
    int32_t _ncomp = 0;
};

class KTruss : public StaticAlgorithm<HornetGraph> {
public:
    explicit KTruss(HornetGraph& h) : StaticAlgorithm(h) {}
    ~KTruss() override { release(); }
    // launch-shape knobs of the reference (KTruss.cu:25-32); the sm_100a
    // implementation sizes its own launches
    void setInitParameters(int, int, int, int, int) {}
    void init() { reset(); }
    void reset() override { _maxK = 0; }
    void run() override {
        _edge_truss.resize((size_t)hornet.nE());
        ::hornet::hn_check(hn_ktruss(hornet.handle(), &_maxK,
                                     _edge_truss.empty() ? nullptr : _edge_truss.data(),
                                     HN_MEM_HOST));
    }
    vid_t getMaxK() const { return _maxK; }
    const std::vector<int32_t>& edgeTruss() const { return _edge_truss; }
    // KTruss::runForK (KTruss.cu:114-119): the K-truss of the graph, as the
    // CSR offsets (nV + 1) of its surviving edges in sorted-COO order
    // (copyOffsetArrayHost, KTruss.cu:44-47); the graph is not modified
    void runForK(int K) {
        run();
        const int32_t nV = hornet.nV();
        std::vector<int32_t> src((size_t)hornet.nE()), dst((size_t)hornet.nE());
        if (!src.empty())
            ::hornet::hn_check(hn_graph_export_coo(hornet.handle(), 1, src.data(), dst.data(),
                                                   HN_MEM_HOST));
        _offsets.assign((size_t)nV + 1, 0);
        for (size_t e = 0; e < src.size(); e++)
            if (_edge_truss[e] >= K) _offsets[(size_t)src[e] + 1]++;
        for (int32_t v = 0; v < nV; v++) _offsets[(size_t)v + 1] += _offsets[(size_t)v];
    }
    void copyOffsetArrayHost(vid_t* host_offset_array) const {
        std::copy(_offsets.begin(), _offsets.end(), host_offset_array);
    }
    // KTruss::runForKDynamic (KTruss.cu:270-295): the graph itself keeps
    // only its K-truss (edges below it are erased through the update path)
    void runForKDynamic(int max_K) {
        int64_t removed = 0;
        ::hornet::hn_check(hn_ktruss_keep(hornet.handle(), max_K, &_maxK, &removed));
    }
    void release() override {}
    bool validate() override {
        int64_t bad = -1;
        return hn_ktruss_validate(hornet.handle(), _maxK,
                                  _edge_truss.empty() ? nullptr : _edge_truss.data(),
                                  HN_MEM_HOST, &bad) == HN_OK &&
               bad == 0;
    }

private:
    int32_t _maxK = 0;
    std::vector<int32_t> _edge_truss;
    std::vector<int32_t> _offsets;
};

}  // namespace hornets_nest
