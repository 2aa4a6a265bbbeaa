// Prepared spectral-flux fixtures (the authoritative WVM boundary) for the
// command line: the little-endian "SKFXP001" file the reference's
// loadPreparedSpectralFluxFixture reads (src/spectral_flux_fixture.cpp:150-411;
// layout in skb_cuda/fixture.py), checked as the reference checks it before
// any timing and returned in this library's order (modes as
// retainedHorizontalModes orders them, operator groups as runs of modes that
// share a file group, matrices forward[g][j][z] / inverse[g][z][j]).

#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "skb_cuda.h"

namespace skbh {

struct PreparedFixture {
    std::uint64_t nx = 0, ny = 0, nz = 0, nj = 0;
    double lx = 0, ly = 0, lz = 0, latitude = 0, pointwiseScale = 0;
    std::string fixtureId, repository, commit, generator, fixtureHash, normalization, modeMapping,
        derivativeConvention;
    std::vector<std::uint64_t> groupModes;            // operator groups, retained-mode order
    std::array<std::vector<double>, 2> forward, inverse;
    std::array<std::uint32_t, 15> inputFamily{};
    std::array<std::uint32_t, 4> targetFamily{};
    std::vector<std::complex<double>> modalInputs;    // [mode][15][j]
    std::vector<std::complex<double>> expectedTargets;  // [mode][4][j]
    std::uint64_t sourceGroups = 0;                   // groups declared in the file
};

// Throws std::runtime_error with the reason when the file is not a valid
// prepared fixture; `modes` are the retained modes of its grid.
PreparedFixture load_prepared_fixture(const std::string& path, const std::vector<skb_retained_mode>& modes);

}  // namespace skbh
