// On-disk graph formats (host code).
//
// * GraphStd binary (.bin), the reference's fast-reload format
//   (xlib/src/Graph/GraphStd.cpp:389-420 writeBinary,
//    xlib/src/Graph/GraphStdRead.cpp:212-245 readBinary), for the
//   vid_t = eoff_t = int instantiation:
//     "intint"  (the demangled type names of vid_t and eoff_t)
//     int32 nV, int32 nE
//     16-byte structure record: 8 zero bytes, int32 flags, 4 zero bytes
//       (flags 1 = DIRECTED, 1|4 = DIRECTED|ENABLE_INGOING)
//     int32 out_offsets[nV+1], [int32 in_offsets[nV+1]],
//     int32 out_edges[nE],     [int32 in_edges[nE]]
//   The bracketed in-edge arrays exist only with ENABLE_INGOING; the reader
//   skips them.
// * Matrix Market coordinate/pattern/general export with 1-based ids, the
//   format GraphStd's Market reader takes (GraphStdRead.cpp:46-61).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "hn_graph.cuh"

namespace {

const char kClassId[] = "intint";
constexpr int kDirected = 1;
constexpr int kIngoing = 4;

struct File {
    FILE* f = nullptr;
    File(const char* p, const char* m) : f(std::fopen(p, m)) {}
    ~File() { if (f) std::fclose(f); }
};

void write_all(FILE* f, const void* p, size_t bytes) {
    if (bytes && std::fwrite(p, 1, bytes, f) != bytes)
        throw hn::Error(HN_ERR_INVALID, "short write");
}

void read_all(FILE* f, void* p, size_t bytes) {
    if (bytes && std::fread(p, 1, bytes, f) != bytes)
        throw hn::Error(HN_ERR_INVALID, "truncated .bin file");
}

void write_bin(const char* path, int32_t nV, int32_t nE, const int32_t* off, const int32_t* adj) {
    File f(path, "wb");
    if (!f.f) throw hn::Error(HN_ERR_INVALID, std::string("cannot open ") + path);
    write_all(f.f, kClassId, sizeof(kClassId) - 1);
    write_all(f.f, &nV, 4);
    write_all(f.f, &nE, 4);
    unsigned char rec[16] = {0};
    int flags = kDirected;
    std::memcpy(rec + 8, &flags, 4);
    write_all(f.f, rec, 16);
    write_all(f.f, off, sizeof(int32_t) * ((size_t)nV + 1));
    write_all(f.f, adj, sizeof(int32_t) * (size_t)nE);
}

}  // namespace

using namespace hn;

extern "C" {

int hn_csr_write_bin(const char* path, int32_t nV, int32_t nE, const int32_t* off,
                     const int32_t* adj) {
    HN_API_BEGIN
    HN_REQUIRE(path && off && (adj || nE == 0) && nV >= 0 && nE >= 0, "bad arguments");
    write_bin(path, nV, nE, off, adj);
    HN_API_END
}

int hn_csr_read_bin(const char* path, int32_t* nV, int32_t* nE, int32_t* off, int32_t* adj) {
    HN_API_BEGIN
    HN_REQUIRE(path && nV && nE, "bad arguments");
    File f(path, "rb");
    if (!f.f) throw Error(HN_ERR_INVALID, std::string("cannot open ") + path);
    char cid[sizeof(kClassId) - 1];
    read_all(f.f, cid, sizeof(cid));
    if (std::memcmp(cid, kClassId, sizeof(cid)) != 0)
        throw Error(HN_ERR_INVALID, "not an int/int GraphStd binary file");
    int32_t v = 0, e = 0;
    read_all(f.f, &v, 4);
    read_all(f.f, &e, 4);
    unsigned char rec[16];
    read_all(f.f, rec, 16);
    int flags = 0;
    std::memcpy(&flags, rec + 8, 4);
    if (v < 0 || e < 0) throw Error(HN_ERR_INVALID, "negative sizes in .bin header");
    *nV = v;
    *nE = e;
    if (!off) return HN_OK;  // size query
    HN_REQUIRE(adj || e == 0, "null edge buffer");
    const bool twice = (flags & kIngoing) != 0;
    read_all(f.f, off, sizeof(int32_t) * ((size_t)v + 1));
    if (twice) std::fseek(f.f, (long)(sizeof(int32_t) * ((size_t)v + 1)), SEEK_CUR);
    read_all(f.f, adj, sizeof(int32_t) * (size_t)e);
    HN_API_END
}

int hn_csr_write_mtx(const char* path, int32_t nV, int64_t nE, const int32_t* off,
                     const int32_t* adj) {
    HN_API_BEGIN
    HN_REQUIRE(path && off && (adj || nE == 0) && nV >= 0 && nE >= 0, "bad arguments");
    File f(path, "w");
    if (!f.f) throw Error(HN_ERR_INVALID, std::string("cannot open ") + path);
    std::fprintf(f.f, "%%%%MatrixMarket matrix coordinate pattern general\n");
    std::fprintf(f.f, "%d %d %lld\n", nV, nV, (long long)nE);
    for (int32_t u = 0; u < nV; u++)
        for (int32_t i = off[u]; i < off[u + 1]; i++)
            std::fprintf(f.f, "%d %d\n", u + 1, adj[i] + 1);
    HN_API_END
}

int hn_graph_write_bin(hn_graph_t* g, const char* path) {
    HN_API_BEGIN
    HN_REQUIRE(g && path, "null argument");
    HN_REQUIRE(g->nE <= 0x7FFFFFFF, "the .bin format holds int32 offsets");
    std::vector<int32_t> off((size_t)g->nV + 1), adj((size_t)g->nE);
    int rc = hn_graph_export_csr(g, off.data(), adj.data(), HN_MEM_HOST);
    if (rc != HN_OK) return rc;
    write_bin(path, g->nV, (int32_t)g->nE, off.data(), adj.data());
    HN_API_END
}

int hn_graph_read_bin(const char* path, int device, hn_graph_t** out) {
    HN_API_BEGIN
    HN_REQUIRE(path && out, "null argument");
    *out = nullptr;
    int32_t nV = 0, nE = 0;
    int rc = hn_csr_read_bin(path, &nV, &nE, nullptr, nullptr);
    if (rc != HN_OK) return rc;
    std::vector<int32_t> off((size_t)nV + 1), adj((size_t)nE + 1);
    rc = hn_csr_read_bin(path, &nV, &nE, off.data(), adj.data());
    if (rc != HN_OK) return rc;
    return hn_graph_create_csr(nV, nE, off.data(), adj.data(), 0, HN_MEM_HOST, device, out);
    HN_API_END
}

}  // extern "C"
