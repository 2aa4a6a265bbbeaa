// Host-side model of the spectral workload: shapes, the radial two-thirds
// retained-mode set, K^2 grouping, order hashes, vertical operator families,
// fixtures, twiddle tables and the per-column tables the kernels read.
//
// Follows include/skbench/skbench.hpp:15-124 and src/model.cpp of the
// reference so that mode order, grouping and layouts are identical.

#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace skb {

struct Workload {
    std::uint64_t nx = 0, ny = 0, nz = 0, fields = 0;
    double lx = 1.0, ly = 1.0;
    bool antialias = true;

    std::uint64_t planes() const { return nz * fields; }                 // skbench.hpp:32
    std::uint64_t nxHalf() const { return nx / 2 + 1; }                  // model.cpp:114
    std::uint64_t realElements() const { return nx * ny * planes(); }    // model.cpp:120
    std::uint64_t spectrumElements() const { return nxHalf() * ny * planes(); }
    std::uint64_t nj() const { return nz < 2 ? 0 : 2 * (nz - 1) / 3; }  // model.cpp:124-127
};

void validate_workload(const Workload& w);  // throws std::invalid_argument

struct RetainedMode {
    std::int64_t k = 0, l = 0;
    std::uint64_t kx = 0, ky = 0;  // stored half-spectrum position
    bool conj = false;             // stored value is the conjugate
    double radial = 0.0;
};

struct ModeGroup {
    std::uint64_t key = 0, first = 0, count = 0;
};

// model.cpp:129-167.
std::vector<RetainedMode> retained_modes(const Workload& w);
// model.cpp:169-207.
std::vector<ModeGroup> squared_wavenumber_groups(const std::vector<RetainedMode>& modes);
// model.cpp:209-217, 462-487 ("fnv1a64:%016x").
std::string mode_order_hash(const std::vector<RetainedMode>& modes);
std::string group_order_hash(const std::vector<ModeGroup>& groups);
std::string wvm_order_hash(const Workload& w);

// Vertical operators: forward[g][j][z] (Nj x Nz) and inverse[g][z][j].
struct VerticalFamily {
    std::string id;
    std::uint64_t nz = 0, nj = 0, groups = 0;
    std::vector<double> forward, inverse;
};
// model.cpp:489-506 truncated orthonormal DCT-II, one group.
VerticalFamily orthonormal_family(std::uint64_t nz, std::uint64_t nj);
// model.cpp:523-565 K^2 pair-rotation family.
VerticalFamily k2_rotation_family(const Workload& w, const std::vector<ModeGroup>& groups);
// Seeded Sturm-Liouville family: per K^2 group the eigenvectors of the
// discretised -d/dz (1/N^2(z)) d/dz + K^2 operator (Neumann ends) with an
// exponential N^2(z) profile, lowest Nj modes, orthonormal rows.
VerticalFamily sturm_liouville_family(const Workload& w, const std::vector<ModeGroup>& groups, std::uint64_t seed);

// model.cpp:618-661 makeFixture; kind 0 impulse, 1 sinusoid, 2 random, 3 dc, 4 nyquist.
std::vector<double> make_fixture(const Workload& w, int kind, std::uint64_t seed);

// exp(-2 pi i k / n) for k in [0, n), as interleaved (re, im) doubles, from
// long double evaluation on [0, pi/4] and exact octant symmetry.
std::vector<double> twiddle_table(std::uint64_t n);

// Column tables for the fused gather / embed (see horizontal.hpp ModeTables).
struct ColumnTables {
    std::uint64_t activeKx = 0;
    std::vector<int> cellMap;   // activeKx * ny
    std::vector<int> gatherMap;  // activeKx * ny: stored cells only (no kx = 0 partners)
    std::vector<int> colStart;  // activeKx + 1
    std::vector<int> colKy, colMode;
    std::vector<int> modeKx, modeKy;
    std::vector<unsigned char> modeConj;
};
ColumnTables column_tables(const Workload& w, const std::vector<RetainedMode>& modes, std::uint64_t columns);

}  // namespace skb
