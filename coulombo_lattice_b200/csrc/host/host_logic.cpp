// Host-side logic of the integral path; see host_logic.hpp.
#include "host_logic.hpp"

#include <algorithm>
#include <cstdint>
#include <cctype>
#include <cmath>
#include <limits>
#include <map>

#include "status.hpp"

namespace cl {

// ---------------------------------------------------------------------------------------
// src/Round.hpp:20-49 -- the same two-level recursion over the prime list {2, 3, 5}.
// ---------------------------------------------------------------------------------------
namespace {
int64_t up_single(int64_t n, int64_t c, int p) {
    while (c < n) c *= p;
    return c;
}
int64_t up_list(int64_t n, int64_t c, const int* primes, int count) {
    if (count == 1) return up_single(n, c, primes[0]);
    int64_t best = up_list(n, c, primes + 1, count - 1);
    while (c < n) {
        c *= primes[0];
        best = std::min(best, up_list(n, c, primes + 1, count - 1));
    }
    return best;
}
}  // namespace

int round_up_235(int n, int c) {
    if (c < 1) fail(CL_ERR_ARGUMENT, "round_up_235: c must be >= 1");
    static const int primes[3] = {2, 3, 5};
    int64_t r = up_list(n, c, primes, 3);
    if (r > std::numeric_limits<int>::max()) fail(CL_ERR_ARGUMENT, "round_up_235: result overflows int");
    return static_cast<int>(r);
}

// ---------------------------------------------------------------------------------------
// src/Broadcaster.cpp:8-22 (float GCD) and :24-43 (per-axis grid).
// ---------------------------------------------------------------------------------------
namespace {
double float_gcd(double a, double b) {
    if (a < b) std::swap(a, b);
    while (true) {
        double r = std::fmod(a, b);
        if (r < 1.0e-10) return b;
        if (r < 1.0e-2) return 0.0;
        a = b;
        b = r;
    }
}

void compute_axis(const double* pos, int64_t n, int d, int& size, double& origin, double& step) {
    std::vector<double> buf(static_cast<size_t>(n));
    for (int64_t a = 0; a < n; ++a) buf[a] = pos[3 * a + d];
    std::sort(buf.begin(), buf.end());
    step = std::numeric_limits<double>::quiet_NaN();
    for (int64_t a = 1; a < n; ++a) {
        double next = buf[a] - buf[a - 1];
        if (next > 1.0e-10) {
            step = std::isnan(step) ? next : float_gcd(step, next);
            if (step == 0) fail(CL_ERR_ARGUMENT, "could not find common grid step");
        }
    }
    origin = buf[0];
    if (std::isnan(step)) {
        // All atoms share this coordinate.  The reference divides by NaN here; one grid
        // point with a unit step is the well-defined equivalent (G at distance >= 1 step
        // never enters an aperiodic convolution of a 1-point axis).
        size = 1;
        step = 1.0;
        return;
    }
    double extent = (buf[n - 1] - buf[0]) / step;
    if (!(extent < 1.0e9)) fail(CL_ERR_ARGUMENT, "grid is too large");
    size = static_cast<int>(std::lrint(extent)) + 1;
}
}  // namespace

Grid detect_grid(const double* pos, int64_t n_atoms, int64_t* cells) {
    if (n_atoms <= 0) fail(CL_ERR_ARGUMENT, "no atoms");
    Grid g;
    for (int d = 0; d < 3; ++d) compute_axis(pos, n_atoms, d, g.raw[d], g.origin[d], g.step[d]);
    for (int d = 0; d < 3; ++d) g.pad[d] = round_up_235(g.raw[d], 1);
    if (cells) {
        for (int64_t a = 0; a < n_atoms; ++a) {
            int64_t ix = std::lrint((pos[3 * a + 0] - g.origin[0]) / g.step[0]);
            int64_t iy = std::lrint((pos[3 * a + 1] - g.origin[1]) / g.step[1]);
            int64_t iz = std::lrint((pos[3 * a + 2] - g.origin[2]) / g.step[2]);
            cells[a] = (iz * g.pad[1] + iy) * g.pad[0] + ix;
        }
    }
    return g;
}

// ---------------------------------------------------------------------------------------
// src/Pattern.hpp:15-100
// ---------------------------------------------------------------------------------------
Pattern::Pattern(const std::string& description, int hole_count) : hole_count_(hole_count) {
    std::string::size_type start = 0, comma;
    auto add = [this](const std::string& p) {
        if (p.empty()) fail(CL_ERR_ARGUMENT, "invalid empty pattern");
        for (char c : p) {
            unsigned char u = static_cast<unsigned char>(c);
            bool valid = (c == '*') || (u < 128 && std::isalnum(u) && c != '0');
            if (!valid) fail(CL_ERR_ARGUMENT, "invalid character '%c' in pattern", c);
        }
        patterns_.push_back(p);
    };
    while ((comma = description.find(',', start)) != std::string::npos) {
        add(description.substr(start, comma - start));
        start = comma + 1;
    }
    add(description.substr(start));
}

bool Pattern::match_one(const std::string& p, const int idx[4]) const {
    int assignments[256] = {0};
    for (int pos = 0; pos < 4; ++pos) {
        // Characters past the end read as '\0', which then acts as one more tied letter
        // (Pattern.hpp:90-93 indexes pattern[0..3] of shorter strings).
        char c = pos < static_cast<int>(p.size()) ? p[pos] : '\0';
        int i = idx[pos];
        bool ok;
        if (c == '*') {
            ok = true;
        } else if (c >= '1' && c <= '9') {
            ok = (i == c - '0');
        } else if (c == 'h') {
            ok = (i <= hole_count_);
        } else if (c == 'e') {
            ok = (i > hole_count_);
        } else {
            int& a = assignments[static_cast<unsigned char>(c)];
            if (a) {
                ok = (i == a);
            } else {
                a = i;
                ok = true;
            }
        }
        if (!ok) return false;
    }
    return true;
}

bool Pattern::match(int i0, int i1, int i2, int i3) const {
    const int idx[4] = {i0, i1, i2, i3};
    for (const auto& p : patterns_)
        if (match_one(p, idx)) return true;
    return false;
}

std::vector<std::array<int16_t, 4>> enumerate_integrals(const Pattern& pattern, int n) {
    if (n < 0 || n >= std::numeric_limits<short>::max()) fail(CL_ERR_ARGUMENT, "too many input files");
    std::vector<std::array<int16_t, 4>> out;
    for (int i1 = 1; i1 <= n; ++i1)
        for (int i2 = 1; i2 <= n; ++i2)
            for (int i3 = 1; i3 <= n; ++i3)
                for (int i4 = 1; i4 <= n; ++i4)
                    if (pattern.match(i1, i2, i3, i4))
                        out.push_back({(int16_t)i1, (int16_t)i2, (int16_t)i3, (int16_t)i4});
    return out;
}

// ---------------------------------------------------------------------------------------
// src/Planner.hpp:134-144 and the product order of src/FunctionCollection.cpp:91-105
// ---------------------------------------------------------------------------------------
ProductRef product_of(int l, int r) {
    uint8_t conj = 0;
    if (l < r) {
        conj = 1;
        std::swap(l, r);
    }
    return ProductRef{l * (l - 1) / 2 + r - 1, conj};
}

void product_states(int p, int* fl, int* fr) {
    int l = static_cast<int>((1.0 + std::sqrt(1.0 + 8.0 * p)) / 2.0);
    while (l > 1 && l * (l - 1) / 2 > p) --l;
    while ((l + 1) * l / 2 <= p) ++l;
    *fl = l;
    *fr = p - l * (l - 1) / 2 + 1;
}

// ---------------------------------------------------------------------------------------
// src/Graph.hpp:49-91 -- loops are forced into the cover; then repeatedly take the vertex
// of smallest (degree, index): if it is a leaf its neighbour joins the cover, otherwise the
// vertex of largest (degree, index) does.
// ---------------------------------------------------------------------------------------
std::set<int> vertex_cover(int vertex_count, const std::vector<std::pair<int, int>>& edge_list) {
    // the distinct edges, in the set order of the reference (sorted pairs): through a bitmap
    // over the vertex pairs when it is small (one pass, no sort), else by sorting
    std::vector<std::pair<int, int>> edges;
    const size_t vc = (size_t)std::max(vertex_count, 0);
    if (vc * vc <= (size_t{1} << 28)) {
        std::vector<uint64_t> seen((vc * vc + 63) / 64, 0);
        for (const auto& e : edge_list) {
            if (e.first < 0 || e.second < 0 || e.first >= vertex_count || e.second >= vertex_count)
                fail(CL_ERR_ARGUMENT, "edge vertex out of range");
            const size_t bit = (size_t)e.first * vc + (size_t)e.second;
            seen[bit >> 6] |= uint64_t{1} << (bit & 63);
        }
        for (size_t w = 0; w < seen.size(); ++w)
            for (uint64_t m = seen[w]; m; m &= m - 1) {
                const size_t bit = w * 64 + (size_t)__builtin_ctzll(m);
                edges.push_back({(int)(bit / vc), (int)(bit % vc)});
            }
    } else {
        edges = edge_list;
        std::sort(edges.begin(), edges.end());
        edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    }
    std::set<int> cover;
    for (const auto& e : edges)
        if (e.first == e.second) cover.insert(e.first);
    std::vector<std::set<int>> nb(vertex_count);
    for (const auto& e : edges) {
        if (e.first != e.second && !cover.count(e.first) && !cover.count(e.second)) {
            nb[e.first].insert(e.second);
            nb[e.second].insert(e.first);
        }
    }
    // ordered by (degree, index); degrees only change while a vertex is out of the set
    std::set<std::pair<size_t, int>> queue;
    for (int v = 0; v < vertex_count; ++v)
        if (!nb[v].empty()) queue.insert({nb[v].size(), v});
    while (!queue.empty()) {
        int v = queue.begin()->second;
        if (nb[v].size() == 1) {
            v = *nb[v].begin();
        } else {
            v = queue.rbegin()->second;
        }
        queue.erase({nb[v].size(), v});
        cover.insert(v);
        for (int w : nb[v]) {
            if (queue.erase({nb[w].size(), w})) {
                nb[w].erase(v);
                if (!nb[w].empty()) queue.insert({nb[w].size(), w});
            }
        }
    }
    return cover;
}

// ---------------------------------------------------------------------------------------
// src/Planner.hpp:71-104
// ---------------------------------------------------------------------------------------
std::vector<PlanStep> orient_steps(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs) {
    if (specs.size() > static_cast<size_t>(std::numeric_limits<int>::max()))
        fail(CL_ERR_ARGUMENT, "too many integrals to compute");
    const int product_count = n_inputs * (n_inputs + 1) / 2;
    std::vector<PlanStep> steps;
    steps.reserve(specs.size());
    std::vector<std::pair<int, int>> edges;
    edges.reserve(specs.size());
    for (size_t id = 0; id < specs.size(); ++id) {
        const auto& s = specs[id];
        for (int k = 0; k < 4; ++k)
            if (s[k] < 1 || s[k] > n_inputs) fail(CL_ERR_ARGUMENT, "integral index out of range");
        PlanStep st{static_cast<int>(id), product_of(s[0], s[3]), product_of(s[1], s[2])};
        steps.push_back(st);
        edges.push_back({st.left.product, st.right.product});
    }
    const auto cover = vertex_cover(product_count, edges);
    std::vector<char> in_cover(product_count, 0);
    for (int v : cover) in_cover[v] = 1;
    for (auto& st : steps)
        if (!in_cover[st.left.product]) std::swap(st.left, st.right);
    return steps;
}

std::vector<PlanStep> compute_plan(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs) {
    if (specs.size() > static_cast<size_t>(std::numeric_limits<int>::max()))
        fail(CL_ERR_ARGUMENT, "too many integrals to compute");
    const int product_count = n_inputs * (n_inputs + 1) / 2;
    std::vector<PlanStep> steps;
    steps.reserve(specs.size());
    std::vector<std::pair<int, int>> edges;
    edges.reserve(specs.size());
    for (size_t id = 0; id < specs.size(); ++id) {
        const auto& s = specs[id];
        for (int k = 0; k < 4; ++k)
            if (s[k] < 1 || s[k] > n_inputs) fail(CL_ERR_ARGUMENT, "integral index out of range");
        PlanStep st{static_cast<int>(id), product_of(s[0], s[3]), product_of(s[1], s[2])};
        steps.push_back(st);
        edges.push_back({st.left.product, st.right.product});
    }
    auto cover = vertex_cover(product_count, edges);
    for (auto& st : steps)
        if (!cover.count(st.left.product)) std::swap(st.left, st.right);
    std::stable_sort(steps.begin(), steps.end(), [](const PlanStep& a, const PlanStep& b) {
        if (a.left.product != b.left.product) return a.left.product < b.left.product;
        if (a.right.product != b.right.product) return a.right.product < b.right.product;
        return (a.left.conjugate == a.right.conjugate) && (b.left.conjugate != b.right.conjugate);
    });
    return steps;
}

}  // namespace cl
