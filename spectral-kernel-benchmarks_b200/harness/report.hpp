// Benchmark report records and their JSON / CSV writers.
//
// The records and the key order of the JSON follow the reference's
// spectral-kernel-benchmark-v1 report (include/skbench/skbench.hpp:700-920,
// src/json.cpp:120-310, schema/spectral-kernel-benchmark-v1.schema.json), and
// the CSV has the reference's nine columns, one row per timing sample, so the
// reference's campaign tools and `compare` read either unchanged.

#pragma once

#include <cstdint>
#include <ostream>
#include <string>
#include <vector>

namespace skbh {

enum class StageState { executed, fused, elided, setupOnly, unsupported };
const char* stage_state_name(StageState s);

struct Timing {
    std::string scope, stage, direction;
    StageState state = StageState::executed;
    std::uint64_t bytesMoved = 0;
    std::vector<double> seconds;
};

struct LedgerEntry {
    std::string stage;
    StageState state = StageState::executed;
    std::string detail;
};

struct Metric {
    std::string name;
    double maximumRelativeError = 0.0;
    double relativeL2Error = 0.0;
    double tolerance = 1e-12;
    bool passed = false;
};

struct DirectionContract {
    std::string nativePlacement, adapterPlacement;
    bool destroysNativeInput = false, adapterPreservesCallerInput = true;
    bool requiresPreservationCopyForRepeatedExecution = false;
    bool preservationIncludedInPrimitiveTiming = false, preservationIncludedInAdapterTiming = false;
    std::string nativeInputRepresentationId, nativeOutputRepresentationId;
    std::string adapterInputRepresentationId, adapterOutputRepresentationId;
    std::string physicalExtents, stridesElements;
    std::uint64_t paddingElements = 0, minimumAlignmentBytes = 256;
    std::string aliasing = "inputs, outputs and provider scratch do not overlap";
    std::uint64_t reusableWorkBytes = 0;
    bool outputCanFeedOppositeDirection = true;
};

struct ProviderRecord {
    std::string id = "cuda", version, libraryIdentity, algorithmId, nativeRepresentationId, modeOrderId,
                schedulingId = "one CUDA stream per provider handle";
    std::string sourceIdentity, sourceSha256, configureFlags, compilerFlags, planningConfiguration;
    std::uint64_t workers = 1, internalWorkers = 1, outerWorkers = 1, gemmCallsPerExecution = 0;
    DirectionContract forward, inverse;
    double otherSetupSeconds = 0, allocationSeconds = 0, planningSeconds = 0;
    std::uint64_t planningBytes = 0, persistentBytes = 0, scratchBytes = 0;
    bool opaqueProviderMemory = false;
    std::vector<LedgerEntry> ledger;
    std::vector<Timing> timings;
    std::vector<Metric> correctness;
};

struct Environment {
    std::string timestampUtc, hostname, operatingSystem, machineModel, cpuBrand;
    std::uint64_t totalCores = 0, performanceCores = 0, efficiencyCores = 0, physicalMemoryBytes = 0;
    std::string compiler, compilerVersion, compilerFlags, buildType, gitCommit;
    bool gitDirty = false;
};

struct Report {
    std::string schema = "spectral-kernel-benchmark-v1";
    std::string status = "passed";
    std::string scalarTypeId = "float64";
    std::uint64_t scalarBits = 64;
    std::string runId, profile;
    std::uint64_t seed = 0, warmups = 0, samples = 0;
    std::uint64_t nx = 0, ny = 0, nz = 0, fields = 0, nkl = 0, nj = 0;
    bool antialias = true;
    std::string verticalMatrixFamilyId = "orthonormal-dct2-truncated-v1";
    std::uint64_t verticalGroupCount = 0, minGroupModes = 0, maxGroupModes = 0, minGroupColumns = 0,
                  maxGroupColumns = 0;
    double medianGroupModes = 0, medianGroupColumns = 0;
    std::string verticalGroupOrderHash, retainedModeOrderHash, wvmFullSpectrumOrderHash;
    std::uint64_t realBytes = 0, fullSpectrumBytes = 0, retainedSpectrumBytes = 0, modalSpectrumBytes = 0,
                  verticalMatrixFamilySourceBytes = 0, verticalPeakBytes = 0, orderingPeakBytes = 0,
                  pipelinePeakBytes = 0;
    Environment environment;
    std::vector<ProviderRecord> providers;
};

double median(std::vector<double> values);
void write_json(const Report& r, std::ostream& out);
void write_csv(const Report& r, std::ostream& out);
// `compare`: median milliseconds per (provider, scope, stage, direction) of a
// report CSV; returns 1 when it holds no timed rows.
int compare_csv(std::istream& in, std::ostream& out);

}  // namespace skbh
