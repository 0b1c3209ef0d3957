// Host-side C++ shim with the reference's class names over the C ABI:
//   hornet::HornetInit<vid_t>            (HornetInitialize/HornetInit.cuh:56-97)
//   hornet::gpu::Hornet<vid_t>           (Core/Hornet.cuh:56-131)
//   hornet::BatchUpdatePtr<vid_t, EMPTY, DeviceType>
//   hornet::gpu::BatchUpdate<vid_t>      (BatchUpdate/BatchUpdate.cuh:77-272)
//   hornet::COO<DeviceType, vid_t>       (Static/Static.cuh:19-157, getCOO)
// for the vid_t = int, no-metadata instantiation that the hot path uses.
// Errors: the C ABI returns codes; this shim keeps the reference's
// behaviour of reporting and stopping (SafeCudaAPI.cpp:71-94) by printing
// the message and throwing std::runtime_error, which the caller may catch.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../hornet_b200.h"
#include "HornetDevice.cuh"

namespace hornet {

struct EMPTY {};
template <typename... T>
struct TypeList {};
enum class DeviceType { DEVICE, HOST };

inline void hn_check(int rc) {
    if (rc != HN_OK) throw std::runtime_error(std::string("hornet_b200: ") + hn_last_error_string());
}

template <typename vid_t = int, typename = EMPTY, typename = EMPTY, typename degree_t = int>
class HornetInit {
public:
    HornetInit(degree_t nV, degree_t nE, const degree_t* csr_offsets, const vid_t* csr_edges,
               bool sorted_adjacency = false) noexcept
        : _nV(nV), _nE(nE), _off(csr_offsets), _edges(csr_edges), _sorted(sorted_adjacency) {}
    degree_t nV() const noexcept { return _nV; }
    degree_t nE() const noexcept { return _nE; }
    const degree_t* csr_offsets() const noexcept { return _off; }
    const vid_t* csr_edges() const noexcept { return _edges; }
    bool sorted() const noexcept { return _sorted; }

private:
    degree_t _nV, _nE;
    const degree_t* _off;
    const vid_t* _edges;
    bool _sorted;
};

template <typename vid_t = int, typename = EMPTY, DeviceType device_t = DeviceType::DEVICE,
          typename degree_t = int>
class BatchUpdatePtr {
public:
    BatchUpdatePtr(degree_t nE, vid_t* src, vid_t* dst) noexcept : _n(nE), _src(src), _dst(dst) {}
    degree_t nE() const noexcept { return _n; }
    vid_t* src() const noexcept { return _src; }
    vid_t* dst() const noexcept { return _dst; }
    static constexpr DeviceType device() { return device_t; }

private:
    degree_t _n;
    vid_t* _src;
    vid_t* _dst;
};

// Sorted COO (host or device copy).
template <DeviceType device_t, typename vid_t = int, typename = EMPTY, typename degree_t = int>
class COO {
public:
    COO() = default;
    explicit COO(size_t n) { resize(n); }
    COO(const COO& o) { *this = o; }
    template <DeviceType other>
    COO(const COO<other, vid_t, EMPTY, degree_t>& o) {
        resize(o.size());
        copy_from(o.srcPtr(), o.dstPtr(), o.size(), other);
    }
    COO& operator=(const COO& o) {
        if (this != &o) {
            resize(o.size());
            copy_from(o.srcPtr(), o.dstPtr(), o.size(), device_t);
        }
        return *this;
    }
    ~COO() { release(); }

    size_t size() const noexcept { return _n; }
    vid_t* srcPtr() const noexcept { return _src; }
    vid_t* dstPtr() const noexcept { return _dst; }

    void resize(size_t n) {
        if (n == _n && _src) return;
        release();
        _n = n;
        if (!n) return;
        if (device_t == DeviceType::DEVICE) {
            hn_cuda(cudaMalloc(&_src, n * sizeof(vid_t)));
            hn_cuda(cudaMalloc(&_dst, n * sizeof(vid_t)));
        } else {
            _src = new vid_t[n];
            _dst = new vid_t[n];
        }
    }
    // append (host-side merge; used by the reference's tests)
    template <DeviceType other>
    void append(const COO<other, vid_t, EMPTY, degree_t>& o) {
        COO<DeviceType::HOST, vid_t, EMPTY, degree_t> a(*this), b(o);
        std::vector<vid_t> s(a.srcPtr(), a.srcPtr() + a.size()), d(a.dstPtr(), a.dstPtr() + a.size());
        s.insert(s.end(), b.srcPtr(), b.srcPtr() + b.size());
        d.insert(d.end(), b.dstPtr(), b.dstPtr() + b.size());
        resize(s.size());
        copy_from(s.data(), d.data(), s.size(), DeviceType::HOST);
    }
    // lexicographic (src, dst) sort
    void sort() {
        COO<DeviceType::HOST, vid_t, EMPTY, degree_t> a(*this);
        std::vector<std::pair<vid_t, vid_t>> e(a.size());
        for (size_t i = 0; i < a.size(); i++) e[i] = {a.srcPtr()[i], a.dstPtr()[i]};
        std::sort(e.begin(), e.end());
        std::vector<vid_t> s(e.size()), d(e.size());
        for (size_t i = 0; i < e.size(); i++) { s[i] = e[i].first; d[i] = e[i].second; }
        copy_from(s.data(), d.data(), s.size(), DeviceType::HOST);
    }

private:
    static void hn_cuda(cudaError_t e) {
        if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
    }
    void copy_from(const vid_t* s, const vid_t* d, size_t n, DeviceType from) {
        if (!n) return;
        cudaMemcpyKind k = from == DeviceType::HOST
                               ? (device_t == DeviceType::HOST ? cudaMemcpyHostToHost : cudaMemcpyHostToDevice)
                               : (device_t == DeviceType::HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice);
        hn_cuda(cudaMemcpy(_src, s, n * sizeof(vid_t), k));
        hn_cuda(cudaMemcpy(_dst, d, n * sizeof(vid_t), k));
    }
    void release() {
        if (device_t == DeviceType::DEVICE) {
            if (_src) cudaFree(_src);
            if (_dst) cudaFree(_dst);
        } else {
            delete[] _src;
            delete[] _dst;
        }
        _src = _dst = nullptr;
        _n = 0;
    }
    size_t _n = 0;
    vid_t* _src = nullptr;
    vid_t* _dst = nullptr;
};

namespace gpu {

template <typename vid_t = int, typename = EMPTY, typename degree_t = int>
class Hornet;

template <typename vid_t = int, typename = EMPTY, typename degree_t = int>
class BatchUpdate {
public:
    template <DeviceType device_t>
    BatchUpdate(const BatchUpdatePtr<vid_t, EMPTY, device_t, degree_t>& p) : _p_src(p.src()),
        _p_dst(p.dst()), _n(p.nE()), _mem(device_t == DeviceType::HOST ? HN_MEM_HOST : HN_MEM_DEVICE) {}
    // BatchUpdate(COO&) as the reference tests use it
    template <DeviceType device_t>
    BatchUpdate(const COO<device_t, vid_t, EMPTY, degree_t>& coo) : _p_src(coo.srcPtr()),
        _p_dst(coo.dstPtr()), _n((degree_t)coo.size()),
        _mem(device_t == DeviceType::HOST ? HN_MEM_HOST : HN_MEM_DEVICE) {}
    ~BatchUpdate() { if (_b) hn_batch_destroy(_b); }
    BatchUpdate(const BatchUpdate&) = delete;
    BatchUpdate& operator=(const BatchUpdate&) = delete;

    degree_t nE() const noexcept { return _n; }
    degree_t size() const noexcept { return _n; }

    // bind to a graph (copies the batch to the device once)
    hn_batch_t* bind(hn_graph_t* g) {
        if (!_b) hn_check(hn_batch_create(g, _n, _p_src, _p_dst, _mem, &_b));
        return _b;
    }

private:
    const vid_t* _p_src;
    const vid_t* _p_dst;
    degree_t _n;
    int _mem;
    hn_batch_t* _b = nullptr;
};

template <typename vid_t, typename Meta, typename degree_t>
class Hornet {
public:
    using VertexType = vid_t;
    using DegreeType = degree_t;
    using HornetDeviceT = ::hornet::HornetDevice;

    template <typename InitT>
    explicit Hornet(const InitT& init, int device = 0) {
        hn_check(hn_graph_create_csr(init.nV(), init.nE(), init.csr_offsets(), init.csr_edges(),
                                     init.sorted() ? HN_CSR_SORTED : 0u, HN_MEM_HOST, device, &_g));
        // the reference runs everything on the legacy default stream
        hn_check(hn_graph_set_stream(_g, (void*)cudaStreamLegacy));
    }
    ~Hornet() { if (_g) hn_graph_destroy(_g); }
    Hornet(const Hornet&) = delete;
    Hornet& operator=(const Hornet&) = delete;

    template <typename InitT>
    void reset(const InitT& init) {
        hn_check(hn_graph_reset_csr(_g, init.nV(), init.nE(), init.csr_offsets(), init.csr_edges(),
                                    init.sorted() ? HN_CSR_SORTED : 0u, HN_MEM_HOST));
    }

    void insert(BatchUpdate<vid_t, Meta, degree_t>& batch, bool removeBatchDuplicates = false,
                bool removeGraphDuplicates = false) {
        unsigned f = (removeBatchDuplicates ? HN_DEDUP_BATCH : 0u) |
                     (removeGraphDuplicates ? HN_DEDUP_GRAPH : 0u);
        int64_t applied = 0;
        hn_check(hn_insert(_g, batch.bind(_g), f, &applied));
    }

    void erase(BatchUpdate<vid_t, Meta, degree_t>& batch, bool removeBatchDuplicates = false) {
        int64_t applied = 0;
        hn_check(hn_erase(_g, batch.bind(_g), removeBatchDuplicates ? HN_DEDUP_BATCH : 0u,
                          &applied));
    }

    degree_t nV() const noexcept { int32_t v = 0; hn_graph_nv(_g, &v); return v; }
    degree_t nE() const noexcept { int64_t e = 0; hn_graph_ne(_g, &e); return (degree_t)e; }

    vid_t max_degree_id() const {
        int32_t d = 0, id = 0;
        hn_check(hn_graph_max_degree(_g, &d, &id));
        return id;
    }
    degree_t max_degree() const {
        int32_t d = 0, id = 0;
        hn_check(hn_graph_max_degree(_g, &d, &id));
        return d;
    }

    HornetDeviceT device() const {
        hn_device_view_t v;
        hn_check(hn_graph_device_view(_g, &v));
        return HornetDeviceT(v);
    }

    COO<DeviceType::DEVICE, vid_t, EMPTY, degree_t> getCOO(bool sortAdjacencyList = false) const {
        COO<DeviceType::DEVICE, vid_t, EMPTY, degree_t> coo((size_t)nE());
        if (coo.size())
            hn_check(hn_graph_export_coo(_g, sortAdjacencyList, coo.srcPtr(), coo.dstPtr(),
                                         HN_MEM_DEVICE));
        return coo;
    }

    // stream / synchronisation used by the operator templates
    cudaStream_t stream() const {
        return cudaStreamLegacy;
    }
    void sync() const { cudaStreamSynchronize(cudaStreamLegacy); }
    hn_graph_t* handle() const noexcept { return _g; }

private:
    hn_graph_t* _g = nullptr;
};

}  // namespace gpu
}  // namespace hornet
