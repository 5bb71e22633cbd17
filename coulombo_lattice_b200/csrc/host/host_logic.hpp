// Host-side logic of the integral path: size rounding, lattice-grid detection, the
// --integrals pattern language, product indexing, the greedy vertex cover and the step plan.
// Each piece restates the behaviour of the reference file cited beside it.
#pragma once

#include <array>
#include <cstdint>
#include <set>
#include <string>
#include <vector>

namespace cl {

// Smallest c * 2^i * 3^j * 5^k >= n (src/Round.hpp:20-49).
int round_up_235(int n, int c = 1);

// Lattice grid of a set of atom positions (src/Broadcaster.cpp:8-43, 76-87, 136-143).
struct Grid {
    int raw[3];
    int pad[3];
    double origin[3];
    double step[3];
};
// pos is [atom][3]; cells (optional) receives (iz*Ny + iy)*Nx + ix on the padded grid.
Grid detect_grid(const double* pos, int64_t n_atoms, int64_t* cells);

// --integrals matcher (src/Pattern.hpp:15-100).
class Pattern {
public:
    Pattern(const std::string& description, int hole_count);
    bool match(int i0, int i1, int i2, int i3) const;

private:
    int hole_count_;
    std::vector<std::string> patterns_;
    bool match_one(const std::string& p, const int idx[4]) const;
};

// All (i1..i4) in [1,n]^4 matching, lexicographic (coulombo.cpp:135-148).
std::vector<std::array<int16_t, 4>> enumerate_integrals(const Pattern& pattern, int n_inputs);

// Product of a (left, right) state pair (src/Planner.hpp:134-144).
struct ProductRef {
    int product;
    uint8_t conjugate;
};
ProductRef product_of(int i_left, int i_right);
// Inverse for the creation order of FunctionCollection::createProducts
// (src/FunctionCollection.cpp:91-105): product p -> 1-based (fL >= fR).
void product_states(int p, int* f_left, int* f_right);

// Greedy vertex cover (src/Graph.hpp:49-91).
std::set<int> vertex_cover(int vertex_count, const std::vector<std::pair<int, int>>& edges);

// MasterPlanner::addIntegral + computePlan (src/Planner.hpp:71-104).
struct PlanStep {
    int id;
    ProductRef left, right;
};
std::vector<PlanStep> compute_plan(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs);

// The same steps with the reference's orientation (which product is prepared) but in input
// order: the GPU computes every step at once, so the execution order of
// Planner.hpp:94-101 does not matter to the values.
std::vector<PlanStep> orient_steps(int n_inputs, const std::vector<std::array<int16_t, 4>>& specs);

}  // namespace cl
