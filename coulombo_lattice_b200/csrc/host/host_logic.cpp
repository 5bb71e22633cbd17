// Host-side logic of the integral path; see host_logic.hpp.
#include "host_logic.hpp"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <thread>

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
namespace {

// Greedy vertex cover on a dense bitmap adjacency (vertex counts up to 16,384): the same rule
// and the same order of choices as the set-based form below -- self-loops force their vertex
// in; then, repeatedly, the queued vertex of least (degree, index) gives way to its single
// neighbour if it is a leaf, else the vertex of greatest (degree, index) is taken -- with
// degrees kept as counters and neighbourhoods as bit rows.
std::set<int> vertex_cover_dense(int vertex_count, const std::vector<std::pair<int, int>>& edge_list) {
    const size_t vc = (size_t)vertex_count;
    const size_t words = (vc + 63) / 64;
    std::vector<uint8_t> in_cover(vc, 0);
    for (const auto& e : edge_list) {
        if (e.first < 0 || e.second < 0 || e.first >= vertex_count || e.second >= vertex_count)
            fail(CL_ERR_ARGUMENT, "edge vertex out of range");
        if (e.first == e.second) in_cover[(size_t)e.first] = 1;
    }
    std::vector<uint64_t> adj(vc * words, 0);
    for (const auto& e : edge_list) {
        const size_t a = (size_t)e.first, b = (size_t)e.second;
        if (a == b || in_cover[a] || in_cover[b]) continue;
        adj[a * words + (b >> 6)] |= uint64_t{1} << (b & 63);
        adj[b * words + (a >> 6)] |= uint64_t{1} << (a & 63);
    }
    std::vector<int> degree(vc, 0);
    for (size_t v = 0; v < vc; ++v)
        for (size_t w = 0; w < words; ++w) degree[v] += __builtin_popcountll(adj[v * words + w]);
    std::set<std::pair<int, int>> queue;
    std::vector<uint8_t> queued(vc, 0);
    for (size_t v = 0; v < vc; ++v)
        if (degree[v] > 0) {
            queue.insert({degree[v], (int)v});
            queued[v] = 1;
        }
    std::set<int> cover;
    for (size_t v = 0; v < vc; ++v)
        if (in_cover[v]) cover.insert((int)v);
    while (!queue.empty()) {
        int v = queue.begin()->second;
        if (degree[v] == 1) {
            const uint64_t* row = &adj[(size_t)v * words];
            for (size_t w = 0; w < words; ++w)
                if (row[w]) {
                    v = (int)(w * 64 + (size_t)__builtin_ctzll(row[w]));
                    break;
                }
        } else {
            v = queue.rbegin()->second;
        }
        queue.erase({degree[v], v});
        queued[(size_t)v] = 0;
        cover.insert(v);
        const uint64_t* row = &adj[(size_t)v * words];
        for (size_t w = 0; w < words; ++w)
            for (uint64_t m = row[w]; m; m &= m - 1) {
                const size_t u = w * 64 + (size_t)__builtin_ctzll(m);
                if (!queued[u]) continue;
                queue.erase({degree[u], (int)u});
                adj[u * words + ((size_t)v >> 6)] &= ~(uint64_t{1} << (v & 63));
                if (--degree[u] > 0)
                    queue.insert({degree[u], (int)u});
                else
                    queued[u] = 0;
            }
    }
    return cover;
}

}  // namespace

std::set<int> vertex_cover(int vertex_count, const std::vector<std::pair<int, int>>& edge_list) {
    if (vertex_count > 0 && vertex_count <= 16384) return vertex_cover_dense(vertex_count, edge_list);
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
namespace {

// Runs f(begin, end) over [0, n) on up to hardware_concurrency threads (one when n is small).
template <typename F>
void parallel_ranges(size_t n, F&& f) {
    const size_t hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>(std::min<size_t>(hw, 32), n / 65536 + 1);
    if (nt <= 1) {
        f(size_t{0}, n);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t t = 0; t < nt; ++t) pool.emplace_back([&, t] { f(n * t / nt, n * (t + 1) / nt); });
    for (auto& th : pool) th.join();
}

// The steps of the integral list (id, left and right products) and their graph edges.
void build_steps(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs, std::vector<PlanStep>& steps,
                 std::vector<std::pair<int, int>>& edges) {
    if (specs.size() > static_cast<size_t>(std::numeric_limits<int>::max()))
        fail(CL_ERR_ARGUMENT, "too many integrals to compute");
    steps.resize(specs.size());
    edges.resize(specs.size());
    std::atomic<bool> bad{false};
    parallel_ranges(specs.size(), [&](size_t i0, size_t i1) {
        for (size_t id = i0; id < i1; ++id) {
            const auto& s = specs[id];
            for (int k = 0; k < 4; ++k)
                if (s[k] < 1 || s[k] > n_inputs) bad = true;
            const PlanStep st{static_cast<int>(id), product_of(s[0], s[3]), product_of(s[1], s[2])};
            steps[id] = st;
            edges[id] = {st.left.product, st.right.product};
        }
    });
    if (bad) fail(CL_ERR_ARGUMENT, "integral index out of range");
}

}  // namespace

std::vector<PlanStep> orient_steps(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs) {
    const int product_count = n_inputs * (n_inputs + 1) / 2;
    std::vector<PlanStep> steps;
    std::vector<std::pair<int, int>> edges;
    build_steps(n_inputs, specs, steps, edges);
    const auto cover = vertex_cover(product_count, edges);
    std::vector<char> in_cover(product_count, 0);
    for (int v : cover) in_cover[v] = 1;
    parallel_ranges(steps.size(), [&](size_t i0, size_t i1) {
        for (size_t i = i0; i < i1; ++i)
            if (!in_cover[steps[i].left.product]) std::swap(steps[i].left, steps[i].right);
    });
    return steps;
}

std::vector<PlanStep> compute_plan(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs) {
    const int product_count = n_inputs * (n_inputs + 1) / 2;
    std::vector<PlanStep> steps;
    std::vector<std::pair<int, int>> edges;
    build_steps(n_inputs, specs, steps, edges);
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
