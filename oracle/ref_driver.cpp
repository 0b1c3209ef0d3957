// Test infrastructure only: a command-line driver around the reference's own
// host-side graph code (xlib/src/Graph/{GraphStd,BFS,WCC}.cpp), compiled from
// the reference sources by oracle/Makefile into oracle/_ref/ref_driver.
//
// It is the "reference" arm of the oracle: the CPU BFS and WCC verifiers and
// the GraphStd Matrix Market reader (symmetrise + dedup + DIRECTED_BY_DEGREE
// orientation) run unmodified on CSR files that the tests and the bench write.
//
// graph::WCC::run() may only run once per process (WCC.cpp:56-58, a static
// flag), which is why this is a process per call rather than a library.
//
// CSR file format (little-endian): int64 nV, int64 nE, int32 off[nV+1],
// int32 adj[nE].  Result files are raw int32 arrays of length nV.
#include <Graph/BFS.hpp>
#include <Graph/GraphStd.hpp>
#include <Graph/WCC.hpp>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <limits>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct Csr {
    int64_t nV = 0, nE = 0;
    std::vector<int32_t> off, adj;
};

bool read_csr(const char* path, Csr& g) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    bool ok = std::fread(&g.nV, 8, 1, f) == 1 && std::fread(&g.nE, 8, 1, f) == 1;
    if (ok) {
        g.off.resize(g.nV + 1);
        g.adj.resize(g.nE);
        ok = std::fread(g.off.data(), 4, g.nV + 1, f) == size_t(g.nV + 1) &&
             std::fread(g.adj.data(), 4, g.nE, f) == size_t(g.nE);
    }
    std::fclose(f);
    return ok;
}

bool write_csr(const char* path, int64_t nV, int64_t nE, const int32_t* off,
               const int32_t* adj) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(&nV, 8, 1, f) == 1 && std::fwrite(&nE, 8, 1, f) == 1 &&
              std::fwrite(off, 4, nV + 1, f) == size_t(nV + 1) &&
              std::fwrite(adj, 4, nE, f) == size_t(nE);
    std::fclose(f);
    return ok;
}

bool write_i32(const char* path, const int32_t* p, int64_t n) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(p, 4, n, f) == size_t(n);
    std::fclose(f);
    return ok;
}

double now_s() {
    return std::chrono::duration<double>(
               std::chrono::steady_clock::now().time_since_epoch()).count();
}

int usage() {
    std::fprintf(stderr,
        "usage:\n"
        "  ref_driver bfs <csr> <out_dist> <src> [<src> ...]   (out: k*nV int32)\n"
        "  ref_driver wcc <csr> <out_color>\n"
        "  ref_driver read_mtx <mtx> <undirected|directed> <by_degree 0|1> <out_csr>\n"
        "  ref_driver time_bfs <csr> <src> [<src> ...]   (prints seconds, visited edges)\n");
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) return usage();
    const std::string cmd = argv[1];

    if (cmd == "bfs" || cmd == "time_bfs") {
        const bool timing = cmd == "time_bfs";
        if (argc < (timing ? 4 : 5)) return usage();
        Csr g;
        if (!read_csr(argv[2], g)) { std::perror("read csr"); return 1; }
        graph::GraphStd<int, int> gs(g.off.data(), int(g.nV), g.adj.data(), int(g.nE));
        graph::BFS<int, int> bfs(gs);
        std::vector<int32_t> out;
        double t = 0;
        long long edges = 0;
        for (int a = timing ? 3 : 4; a < argc; a++) {
            int src = std::atoi(argv[a]);
            bfs.reset();
            double t0 = now_s();
            bfs.run(src);
            t += now_s() - t0;
            // edges scanned = sum of the degrees of the reached vertices,
            // counted here from the CSR (graph::BFS::visited_edges reads
            // GraphStd's _out_degrees, which the CSR constructor used here
            // does not fill)
            {
                const int* d = bfs.result();
                for (int64_t v = 0; v < g.nV; v++)
                    if (d[v] != std::numeric_limits<int>::max()) edges += g.off[v + 1] - g.off[v];
            }
            if (!timing) {
                const int* d = bfs.result();
                out.insert(out.end(), d, d + g.nV);
            }
        }
        if (timing) {
            std::printf("%.9f %lld\n", t, edges);
            return 0;
        }
        if (!write_i32(argv[3], out.data(), int64_t(out.size()))) { std::perror("write"); return 1; }
        return 0;
    }
    if (cmd == "wcc") {
        if (argc != 4) return usage();
        Csr g;
        if (!read_csr(argv[2], g)) { std::perror("read csr"); return 1; }
        graph::GraphStd<int, int> gs(g.off.data(), int(g.nV), g.adj.data(), int(g.nE));
        graph::WCC<int, int> wcc(gs);
        double t0 = now_s();
        wcc.run();
        double t = now_s() - t0;
        std::vector<int32_t> col(wcc.result(), wcc.result() + g.nV);
        if (!write_i32(argv[3], col.data(), g.nV)) { std::perror("write"); return 1; }
        std::printf("%.9f %d\n", t, int(wcc.size()));
        return 0;
    }
    if (cmd == "read_mtx") {
        if (argc != 6) return usage();
        using namespace graph;
        const bool undirected = std::strcmp(argv[3], "undirected") == 0;
        const bool by_degree = std::atoi(argv[4]) != 0;
        ParsingProp prop = parsing_prop::NONE;
        if (by_degree) prop = parsing_prop::DIRECTED_BY_DEGREE | parsing_prop::SORT;
        GraphStd<int, int> gs(undirected ? structure_prop::UNDIRECTED
                                         : structure_prop::DIRECTED,
                              argv[2], prop);
        if (!write_csr(argv[5], gs.nV(), gs.nE(), gs.csr_out_offsets(),
                       gs.csr_out_edges())) {
            std::perror("write csr");
            return 1;
        }
        return 0;
    }
    return usage();
}
