// Test-only driver (oracle): exposes the reference's own header-only host logic --
// Round::up (src/Round.hpp:20-49), Pattern (src/Pattern.hpp:15-100) and
// Graph::computeVertexCover (src/Graph.hpp:49-91) -- through a C ABI so the tests can compare
// the product's host library against the reference code itself.  The headers are included
// from the reference tree at build time (see oracle/Makefile); nothing of them is copied.
#include <cassert>
#include <cctype>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "throwf.hpp"
#include "Round.hpp"
#include "Pattern.hpp"
#include "Graph.hpp"

extern "C" {

int ref_round_up_235(int n, int c) { return Round::up<2, 3, 5>(n, c); }
int ref_round_up_2(int n, int c) { return Round::up<2>(n, c); }

// Fills match[] for every (i0..i3) in [1,n]^4 in lexicographic order; returns 0, or 1 with
// the exception message in err (size >= 256).
int ref_pattern_enumerate(const char* desc, int n, int holes, uint8_t* match, char* err) {
    try {
        Pattern p(desc, holes);
        size_t k = 0;
        for (int a = 1; a <= n; ++a)
            for (int b = 1; b <= n; ++b)
                for (int c = 1; c <= n; ++c)
                    for (int d = 1; d <= n; ++d) match[k++] = p.match(a, b, c, d) ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        std::strncpy(err, e.what(), 255);
        err[255] = 0;
        return 1;
    }
}

void ref_vertex_cover(int nv, int ne, const int32_t* edges, uint8_t* out) {
    Graph g(nv);
    for (int i = 0; i < ne; ++i) g.addEdge(edges[2 * i], edges[2 * i + 1]);
    auto cover = g.computeVertexCover();
    std::memset(out, 0, (size_t)nv);
    for (int v : cover) out[v] = 1;
}
}
