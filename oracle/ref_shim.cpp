// Test infrastructure only: a C shim over the reference's own CPU functions.
//
// This file is compiled together with the reference sources where they lie
// (src/model.cpp, src/pointwise_advection.cpp, src/json.cpp and
// src/spectral_flux_fixture.cpp of
// JeffreyEarly/spectral-kernel-benchmarks) by oracle/Makefile into
// oracle/_ref/libskbref.so.  Nothing in the product links it.  It exists so
// that tests/golden/make_golden.py can pin the oracle restatement
// (oracle/skb_oracle.cpp) and the CUDA provider against outputs of the
// reference's own arithmetic.
//
// Every entry point returns 0 on success and a negative value when the
// reference threw; the message is kept for skbref_last_error().

#include "skbench/skbench.hpp"
#include "pointwise_advection.hpp"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <random>
#include <string>
#include <vector>

namespace skbench {
// benchmark.cpp:1068-1073 defines median(); benchmark.cpp needs FFTW and is not
// compiled here, so json.cpp's dependency is satisfied with the same definition
// of a median (middle element, or mean of the two middle elements).
double median(std::vector<double> values) {
    if (values.empty()) return 0.0;
    std::sort(values.begin(), values.end());
    const auto middle = values.size() / 2;
    return values.size() % 2 == 0 ? 0.5 * (values[middle - 1] + values[middle]) : values[middle];
}
}  // namespace skbench

namespace {
thread_local std::string lastError;

skbench::Workload makeWorkload(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields) {
    skbench::Workload workload;
    workload.nx = nx;
    workload.ny = ny;
    workload.nz = nz;
    workload.fields = fields;
    return workload;
}

template <typename Body>
int guarded(Body body) {
    try {
        body();
        return 0;
    } catch (const std::exception& error) {
        lastError = error.what();
        return -1;
    }
}

skbench::VerticalOperators groupSlice(const skbench::GroupedVerticalOperators& family, std::size_t group) {
    skbench::VerticalOperators ops;
    ops.id = family.id;
    ops.nz = family.nz;
    ops.nj = family.nj;
    const auto elements = family.nz * family.nj;
    ops.forward.assign(family.forward.begin() + static_cast<std::ptrdiff_t>(group * elements),
                       family.forward.begin() + static_cast<std::ptrdiff_t>((group + 1) * elements));
    ops.inverse.assign(family.inverse.begin() + static_cast<std::ptrdiff_t>(group * elements),
                       family.inverse.begin() + static_cast<std::ptrdiff_t>((group + 1) * elements));
    return ops;
}
}  // namespace

extern "C" {

const char* skbref_last_error() { return lastError.c_str(); }

// Retained modes (model.cpp:129-167). Arrays must hold halfRows entries.
int skbref_retained_modes(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                          std::int64_t* k, std::int64_t* l, std::uint64_t* storedKx, std::uint64_t* storedKy,
                          std::uint8_t* conj, double* radial, std::uint64_t* count) {
    return guarded([&] {
        const auto modes = skbench::retainedHorizontalModes(makeWorkload(nx, ny, nz, fields));
        for (std::size_t i = 0; i < modes.size(); ++i) {
            k[i] = modes[i].k;
            l[i] = modes[i].l;
            storedKx[i] = modes[i].storedKx;
            storedKy[i] = modes[i].storedKy;
            conj[i] = modes[i].conjugatesStoredValue ? 1 : 0;
            radial[i] = modes[i].radialMode;
        }
        *count = modes.size();
    });
}

// K^2 groups (model.cpp:169-207) and the three order hashes (model.cpp:209-217, 462-487).
int skbref_groups_and_hashes(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                             std::uint64_t* keys, std::uint64_t* first, std::uint64_t* counts,
                             std::uint64_t* groupCount, char* modeHash, char* groupHash, char* wvmHash) {
    return guarded([&] {
        const auto workload = makeWorkload(nx, ny, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        const auto groups = skbench::squaredWavenumberGroups(modes);
        for (std::size_t g = 0; g < groups.size(); ++g) {
            keys[g] = groups[g].squaredModeKey;
            first[g] = groups[g].firstMode;
            counts[g] = groups[g].modeCount;
        }
        *groupCount = groups.size();
        std::strncpy(modeHash, skbench::modeOrderHash(modes).c_str(), 63);
        std::strncpy(groupHash, skbench::verticalModeGroupHash(groups).c_str(), 63);
        std::strncpy(wvmHash, skbench::wvmSpectrumOrderHash(workload).c_str(), 63);
    });
}

// Fixtures (model.cpp:618-661): kind 0 impulse, 1 sinusoid, 2 random, 3 dc, 4 nyquist.
int skbref_make_fixture(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                        int kind, std::uint64_t seed, double* out) {
    return guarded([&] {
        const auto values = skbench::makeFixture(makeWorkload(nx, ny, nz, fields),
                                                 static_cast<skbench::FixtureKind>(kind), seed);
        std::memcpy(out, values.data(), values.size() * sizeof(double));
    });
}

// Direct O(N^4) DFT oracles (model.cpp:663-716).
int skbref_direct_r2c(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                      const double* input, double* wvmSpectrum) {
    return guarded([&] {
        skbench::directR2C(makeWorkload(nx, ny, nz, fields), input,
                           reinterpret_cast<skbench::Complex*>(wvmSpectrum));
    });
}

int skbref_direct_c2r(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                      const double* wvmSpectrum, double* output) {
    return guarded([&] {
        skbench::directC2R(makeWorkload(nx, ny, nz, fields),
                           reinterpret_cast<const skbench::Complex*>(wvmSpectrum), output);
    });
}

// Retention and embedding (model.cpp:310-339).
int skbref_gather_retained(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                           const double* wvmSpectrum, double* retained) {
    return guarded([&] {
        const auto workload = makeWorkload(nx, ny, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        skbench::gatherRetained(workload, modes, reinterpret_cast<const skbench::Complex*>(wvmSpectrum),
                                reinterpret_cast<skbench::Complex*>(retained));
    });
}

int skbref_embed_retained(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                          const double* retained, double* wvmSpectrum) {
    return guarded([&] {
        const auto workload = makeWorkload(nx, ny, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        skbench::embedRetained(workload, modes, reinterpret_cast<const skbench::Complex*>(retained),
                               reinterpret_cast<skbench::Complex*>(wvmSpectrum));
    });
}

// Vertical fixtures (model.cpp:489-565). Arrays hold groups*nj*nz entries.
int skbref_k2_vertical_fixture(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                               double* forward, double* inverse, std::uint64_t* nj, char* id) {
    return guarded([&] {
        const auto workload = makeWorkload(nx, ny, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        const auto family = skbench::squaredWavenumberVerticalFixture(workload, modes);
        std::memcpy(forward, family.forward.data(), family.forward.size() * sizeof(double));
        std::memcpy(inverse, family.inverse.data(), family.inverse.size() * sizeof(double));
        *nj = family.nj;
        std::strncpy(id, family.id.c_str(), 127);
    });
}

int skbref_orthonormal_vertical_fixture(std::uint64_t nz, std::uint64_t nj, double* forward, double* inverse) {
    return guarded([&] {
        const auto ops = skbench::orthonormalVerticalFixture(nz, nj);
        std::memcpy(forward, ops.forward.data(), ops.forward.size() * sizeof(double));
        std::memcpy(inverse, ops.inverse.data(), ops.inverse.size() * sizeof(double));
    });
}

// Scalar vertical projections (model.cpp:567-605), applied group by group over the
// K^2 family so each group's columns see that group's matrix.  direction 0 = forward
// (physical [mode][field][z] -> modal [mode][field][j]), 1 = inverse.
int skbref_grouped_vertical(std::uint64_t nx, std::uint64_t ny, std::uint64_t nz, std::uint64_t fields,
                            int direction, const double* input, double* output) {
    return guarded([&] {
        const auto workload = makeWorkload(nx, ny, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        const auto family = skbench::squaredWavenumberVerticalFixture(workload, modes);
        const auto nj = family.nj;
        const auto* in = reinterpret_cast<const skbench::Complex*>(input);
        auto* out = reinterpret_cast<skbench::Complex*>(output);
        for (std::size_t g = 0; g < family.groups.size(); ++g) {
            const auto ops = groupSlice(family, g);
            const auto first = family.groups[g].firstMode;
            const auto count = family.groups[g].modeCount;
            if (direction == 0) {
                skbench::verticalForward(workload, count, ops, in + first * fields * nz, out + first * fields * nj);
            } else {
                skbench::verticalInverse(workload, count, ops, in + first * fields * nj, out + first * fields * nz);
            }
        }
    });
}

// The spectral-pipeline round trip in the order of runSpectralPipelineBenchmark's
// reference computation (benchmark.cpp:3072-3110), composed from model.cpp with
// the direct DFTs in place of FFTW: makeFixture(random, seed) -> directR2C ->
// gatherRetained -> per-group verticalForward -> applySyntheticModalWorkInterleaved
// (syntheticModalWorkWeights) -> per-group verticalInverse -> embedRetained ->
// directC2R (unnormalised).  input: nx*ny*nz*fields doubles; weights:
// modes*fields*nj doubles; output: like input.
int skbref_spectral_pipeline(std::uint64_t n, std::uint64_t nz, std::uint64_t fields, std::uint64_t seed,
                             double* input, double* weights, double* output) {
    return guarded([&] {
        const auto workload = makeWorkload(n, n, nz, fields);
        const auto modes = skbench::retainedHorizontalModes(workload);
        const auto family = skbench::squaredWavenumberVerticalFixture(workload, modes);
        const auto nj = family.nj;
        const auto real = skbench::makeFixture(workload, skbench::FixtureKind::random, seed);
        std::memcpy(input, real.data(), real.size() * sizeof(double));
        std::vector<skbench::Complex> spectrum(workload.spectrumElements());
        skbench::directR2C(workload, real.data(), spectrum.data());
        std::vector<skbench::Complex> retained(modes.size() * workload.planes());
        skbench::gatherRetained(workload, modes, spectrum.data(), retained.data());
        std::vector<skbench::Complex> modal(modes.size() * fields * nj), worked(modal.size());
        for (std::size_t g = 0; g < family.groups.size(); ++g) {
            const auto ops = groupSlice(family, g);
            const auto first = family.groups[g].firstMode;
            skbench::verticalForward(workload, family.groups[g].modeCount, ops, retained.data() + first * fields * nz,
                                     modal.data() + first * fields * nj);
        }
        const auto w = skbench::syntheticModalWorkWeights(workload, modes);
        std::memcpy(weights, w.data(), w.size() * sizeof(double));
        skbench::applySyntheticModalWorkInterleaved(modal.size(), w.data(), modal.data(), worked.data());
        for (std::size_t g = 0; g < family.groups.size(); ++g) {
            const auto ops = groupSlice(family, g);
            const auto first = family.groups[g].firstMode;
            skbench::verticalInverse(workload, family.groups[g].modeCount, ops, worked.data() + first * fields * nj,
                                     retained.data() + first * fields * nz);
        }
        skbench::embedRetained(workload, modes, retained.data(), spectrum.data());
        std::vector<double> back(workload.realElements());
        skbench::directC2R(workload, spectrum.data(), back.data());
        std::memcpy(output, back.data(), back.size() * sizeof(double));
    });
}

// PointwiseAdvectionExecutor (pointwise_advection.cpp:152-240); policy 0 serial,
// 1 vector-serial, 2 spatial-static.
int skbref_pointwise(int policy, std::uint64_t workers, std::uint64_t volume, double scale,
                     const double* shared, const double* derivative, double* target) {
    return guarded([&] {
        skbench::PointwiseAdvectionExecutor executor(static_cast<skbench::PointwiseAdvectionPolicy>(policy),
                                                     workers, volume, scale);
        executor.execute(shared, derivative, target);
    });
}

// Error metrics (model.cpp:718-751).
double skbref_max_rel_error_complex(const double* actual, const double* expected, std::uint64_t count) {
    return skbench::maximumRelativeError(reinterpret_cast<const skbench::Complex*>(actual),
                                         reinterpret_cast<const skbench::Complex*>(expected), count);
}

double skbref_max_rel_error_real(const double* actual, const double* expected, std::uint64_t count, double scale) {
    return skbench::maximumRelativeError(actual, expected, count, scale);
}

double skbref_rel_l2_error(const double* actual, const double* expected, std::uint64_t count) {
    return skbench::relativeL2Error(reinterpret_cast<const skbench::Complex*>(actual),
                                    reinterpret_cast<const skbench::Complex*>(expected), count);
}

// The 15 -> 4 synthetic flux at a small square size, composed from the reference's
// own functions in the order of runProductionLifetimeFluxBenchmark's independent
// oracle (benchmark.cpp:4182-4241), with the direct DFTs standing in for FFTW
// ESTIMATE plans (same unnormalised transforms).  Inputs are drawn as in
// benchmark.cpp:4045-4058.  modalIn holds modes*15*nj complex, modalOut modes*4*nj.
int skbref_flux_direct(std::uint64_t n, std::uint64_t nz, std::uint64_t seed, double* modalIn, double* modalOut) {
    return guarded([&] {
        using skbench::Complex;
        skbench::Workload out = makeWorkload(n, n, nz, 4);
        skbench::Workload in = makeWorkload(n, n, nz, 15);
        skbench::Workload triple = makeWorkload(n, n, nz, 3);
        skbench::Workload target = makeWorkload(n, n, nz, 1);
        const auto modes = skbench::retainedHorizontalModes(out);
        const auto H = modes.size();
        const auto nj = out.retainedVerticalModes();
        const auto plane = n * n;
        const auto volume = plane * nz;
        const double scale = 1.0 / static_cast<double>(plane * plane);
        const auto family = skbench::squaredWavenumberVerticalFixture(out, modes);

        std::mt19937_64 generator(seed);
        std::uniform_real_distribution<double> distribution(-0.125, 0.125);
        std::vector<Complex> inputModal(H * nj * 15);
        for (std::size_t m = 0; m < H; ++m) {
            const bool dc = modes[m].k == 0 && modes[m].l == 0;
            for (std::size_t f = 0; f < 15; ++f) {
                for (std::size_t j = 0; j < nj; ++j) {
                    auto& value = inputModal[skbench::modalSpectrumIndex(in, m, j, f)];
                    value.real = distribution(generator);
                    value.imag = dc ? 0.0 : distribution(generator);
                }
            }
        }
        std::memcpy(modalIn, inputModal.data(), inputModal.size() * sizeof(Complex));

        std::vector<Complex> physicalIn(H * nz * 15);
        for (std::size_t g = 0; g < family.groups.size(); ++g) {
            const auto ops = groupSlice(family, g);
            const auto first = family.groups[g].firstMode;
            skbench::verticalInverse(in, family.groups[g].modeCount, ops, inputModal.data() + first * 15 * nj,
                                     physicalIn.data() + first * 15 * nz);
        }
        std::vector<Complex> compactTriple(H * nz * 3), compactTarget(H * nz), physicalOut(H * nz * 4);
        std::vector<Complex> tripleSpectrum(triple.spectrumElements()), targetSpectrum(target.spectrumElements());
        std::vector<double> shared(triple.realElements()), derivative(triple.realElements()),
            targetVolume(target.realElements());
        auto copyTriple = [&](std::size_t firstField) {
            for (std::size_t m = 0; m < H; ++m)
                for (std::size_t f = 0; f < 3; ++f)
                    for (std::size_t z = 0; z < nz; ++z)
                        compactTriple[skbench::retainedSpectrumIndex(triple, m, z, f)] =
                            physicalIn[skbench::retainedSpectrumIndex(in, m, z, firstField + f)];
        };
        copyTriple(0);
        skbench::embedRetained(triple, modes, compactTriple.data(), tripleSpectrum.data());
        skbench::directC2R(triple, tripleSpectrum.data(), shared.data());
        skbench::PointwiseAdvectionExecutor pointwise(skbench::PointwiseAdvectionPolicy::serial, 1, volume, scale);
        for (std::size_t t = 0; t < 4; ++t) {
            copyTriple(3 + 3 * t);
            skbench::embedRetained(triple, modes, compactTriple.data(), tripleSpectrum.data());
            skbench::directC2R(triple, tripleSpectrum.data(), derivative.data());
            pointwise.execute(shared.data(), derivative.data(), targetVolume.data());
            skbench::directR2C(target, targetVolume.data(), targetSpectrum.data());
            skbench::gatherRetained(target, modes, targetSpectrum.data(), compactTarget.data());
            for (std::size_t m = 0; m < H; ++m)
                for (std::size_t z = 0; z < nz; ++z)
                    physicalOut[skbench::retainedSpectrumIndex(out, m, z, t)] =
                        compactTarget[skbench::retainedSpectrumIndex(target, m, z, 0)];
        }
        auto* result = reinterpret_cast<Complex*>(modalOut);
        for (std::size_t g = 0; g < family.groups.size(); ++g) {
            const auto ops = groupSlice(family, g);
            const auto first = family.groups[g].firstMode;
            skbench::verticalForward(out, family.groups[g].modeCount, ops, physicalOut.data() + first * 4 * nz,
                                     result + first * 4 * nj);
        }
    });
}

// A prepared spectral-flux fixture (SKFXP001) read by the reference's own loader,
// loadPreparedSpectralFluxFixture (spectral_flux_fixture.cpp:150-411), reported
// in the loader's order: modes as retainedHorizontalModes orders them, operator
// groups (first mode, mode count, key, matrix source group) of family 0 (both
// families share them), matrices per family and source group as the loader
// stores them (forward [j][z], inverse [z][j]), modal inputs [mode][15][j] and
// the file's expected targets [mode][4][j].  dims receives Nx, Nz, modes, Nj,
// operator groups and source groups; with null arrays only dims is written.
int skbref_load_flux_fixture(const char* path, std::uint64_t* dims, std::int64_t* k, std::int64_t* l,
                             std::uint64_t* groupFirst, std::uint64_t* groupCount, std::uint64_t* groupKey,
                             std::uint64_t* matrixSource, double* forward, double* inverse, double* modalIn,
                             double* expected) {
    return guarded([&] {
        const auto fixture = skbench::loadPreparedSpectralFluxFixture(path);
        const auto& fam0 = fixture.operatorFamilies[0];
        const std::size_t sources = fixture.groupKeys.size();
        dims[0] = fixture.workload.nx;
        dims[1] = fixture.workload.nz;
        dims[2] = fixture.modes.size();
        dims[3] = fam0.nj;
        dims[4] = fam0.groups.size();
        dims[5] = sources;
        if (k == nullptr) return;
        for (std::size_t m = 0; m < fixture.modes.size(); ++m) {
            k[m] = fixture.modes[m].k;
            l[m] = fixture.modes[m].l;
        }
        for (std::size_t g = 0; g < fam0.groups.size(); ++g) {
            groupFirst[g] = fam0.groups[g].firstMode;
            groupCount[g] = fam0.groups[g].modeCount;
            groupKey[g] = fam0.groups[g].squaredModeKey;
            matrixSource[g] = fam0.matrixSourceGroups[g];
        }
        const std::size_t per = fam0.nz * fam0.nj * sources;
        for (std::size_t f = 0; f < 2; ++f) {
            std::memcpy(forward + f * per, fixture.operatorFamilies[f].forward.data(), per * sizeof(double));
            std::memcpy(inverse + f * per, fixture.operatorFamilies[f].inverse.data(), per * sizeof(double));
        }
        std::memcpy(modalIn, fixture.modalInputs.data(), fixture.modalInputs.size() * sizeof(skbench::Complex));
        std::memcpy(expected, fixture.expectedModalTargets.data(),
                    fixture.expectedModalTargets.size() * sizeof(skbench::Complex));
    });
}

// The authoritative two-family 15 -> 4 flux of a prepared fixture, composed from
// the reference's own functions: the fixture read by its loader, each input slot
// and target taken through verticalInverse / verticalForward (model.cpp:567-605)
// with the operator matrices of its family (the fixture's field-to-family maps,
// authoritative_spectral_flux.cpp:193-216, 340-440) and operator group, then the
// streamed order of skbref_flux_direct: embedRetained + directC2R of U,V,W, per
// target the derivative triple, PointwiseAdvectionExecutor with the fixture's
// pointwise scale, directR2C + gatherRetained.  The direct DFTs stand in for the
// FFTW plans (same unnormalised transforms), so keep Nx small.  modalOut holds
// modes*4*nj complex in the loader's mode order.
int skbref_two_family_flux_direct(const char* path, double* modalOut) {
    return guarded([&] {
        using skbench::Complex;
        const auto fixture = skbench::loadPreparedSpectralFluxFixture(path);
        const auto n = fixture.workload.nx, nz = fixture.workload.nz;
        skbench::Workload out = fixture.workload;
        out.fields = 4;
        skbench::Workload in = fixture.workload;
        in.fields = 15;
        skbench::Workload triple = fixture.workload;
        triple.fields = 3;
        skbench::Workload single = fixture.workload;
        single.fields = 1;
        const auto& modes = fixture.modes;
        const auto H = modes.size();
        const auto nj = out.retainedVerticalModes();
        const auto volume = n * n * nz;
        auto slice = [&](std::size_t family, std::size_t group) {
            const auto& ops = fixture.operatorFamilies[family];
            return groupSlice(ops, ops.matrixSourceGroups[group]);
        };
        const auto& groups = fixture.operatorFamilies[0].groups;

        // Inverse vertical transform, one slot at a time with its family's matrices.
        std::vector<Complex> physicalIn(H * nz * 15);
        for (std::size_t f = 0; f < 15; ++f) {
            const auto family = fixture.inputFieldFamilies[f];
            for (std::size_t g = 0; g < groups.size(); ++g) {
                const auto first = groups[g].firstMode, count = groups[g].modeCount;
                std::vector<Complex> modal(count * nj), phys(count * nz);
                for (std::size_t m = 0; m < count; ++m)
                    for (std::size_t j = 0; j < nj; ++j)
                        modal[skbench::modalSpectrumIndex(single, m, j, 0)] =
                            fixture.modalInputs[skbench::modalSpectrumIndex(in, first + m, j, f)];
                skbench::verticalInverse(single, count, slice(family, g), modal.data(), phys.data());
                for (std::size_t m = 0; m < count; ++m)
                    for (std::size_t z = 0; z < nz; ++z)
                        physicalIn[skbench::retainedSpectrumIndex(in, first + m, z, f)] =
                            phys[skbench::retainedSpectrumIndex(single, m, z, 0)];
            }
        }

        std::vector<Complex> compactTriple(H * nz * 3), compactTarget(H * nz), physicalOut(H * nz * 4);
        std::vector<Complex> tripleSpectrum(triple.spectrumElements()), targetSpectrum(single.spectrumElements());
        std::vector<double> shared(triple.realElements()), derivative(triple.realElements()),
            targetVolume(single.realElements());
        auto copyTriple = [&](std::size_t firstField) {
            for (std::size_t m = 0; m < H; ++m)
                for (std::size_t f = 0; f < 3; ++f)
                    for (std::size_t z = 0; z < nz; ++z)
                        compactTriple[skbench::retainedSpectrumIndex(triple, m, z, f)] =
                            physicalIn[skbench::retainedSpectrumIndex(in, m, z, firstField + f)];
        };
        copyTriple(0);
        skbench::embedRetained(triple, modes, compactTriple.data(), tripleSpectrum.data());
        skbench::directC2R(triple, tripleSpectrum.data(), shared.data());
        skbench::PointwiseAdvectionExecutor pointwise(skbench::PointwiseAdvectionPolicy::serial, 1, volume,
                                                      fixture.pointwiseScale);
        for (std::size_t t = 0; t < 4; ++t) {
            copyTriple(3 + 3 * t);
            skbench::embedRetained(triple, modes, compactTriple.data(), tripleSpectrum.data());
            skbench::directC2R(triple, tripleSpectrum.data(), derivative.data());
            pointwise.execute(shared.data(), derivative.data(), targetVolume.data());
            skbench::directR2C(single, targetVolume.data(), targetSpectrum.data());
            skbench::gatherRetained(single, modes, targetSpectrum.data(), compactTarget.data());
            for (std::size_t m = 0; m < H; ++m)
                for (std::size_t z = 0; z < nz; ++z)
                    physicalOut[skbench::retainedSpectrumIndex(out, m, z, t)] =
                        compactTarget[skbench::retainedSpectrumIndex(single, m, z, 0)];
        }

        // Forward vertical transform, one target at a time with its family's matrices.
        auto* result = reinterpret_cast<Complex*>(modalOut);
        for (std::size_t t = 0; t < 4; ++t) {
            const auto family = fixture.targetFieldFamilies[t];
            for (std::size_t g = 0; g < groups.size(); ++g) {
                const auto first = groups[g].firstMode, count = groups[g].modeCount;
                std::vector<Complex> phys(count * nz), modal(count * nj);
                for (std::size_t m = 0; m < count; ++m)
                    for (std::size_t z = 0; z < nz; ++z)
                        phys[skbench::retainedSpectrumIndex(single, m, z, 0)] =
                            physicalOut[skbench::retainedSpectrumIndex(out, first + m, z, t)];
                skbench::verticalForward(single, count, slice(family, g), phys.data(), modal.data());
                for (std::size_t m = 0; m < count; ++m)
                    for (std::size_t j = 0; j < nj; ++j)
                        result[skbench::modalSpectrumIndex(out, first + m, j, t)] =
                            modal[skbench::modalSpectrumIndex(single, m, j, 0)];
            }
        }
    });
}

// Writes the reference's own JSON/CSV report for a minimal filled report, so the
// schema tests can compare key sets with the CUDA harness's output.
int skbref_write_schema_sample(const char* jsonPath, const char* csvPath) {
    return guarded([&] {
        skbench::BenchmarkReport report;
        report.status = "passed";
        report.runId = "schema-sample";
        report.profile = "smoke";
        report.workload = makeWorkload(8, 8, 7, 2);
        skbench::ProviderRecord provider;
        provider.id = "sample";
        provider.ledger.push_back({"stage", skbench::StageState::executed, "detail"});
        provider.timings.push_back({"primitive", "stage", "forward", skbench::StageState::executed, 8, {1.0, 2.0}});
        provider.correctness.push_back({"metric", 0.0, 1.0e-12, true, 0.0});
        report.providers.push_back(provider);
        skbench::writeJson(report, jsonPath);
        skbench::writeCsv(report, csvPath);
    });
}

}  // extern "C"
