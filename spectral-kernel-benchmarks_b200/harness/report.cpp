// JSON / CSV writers for the spectral-kernel-benchmark-v1 report.

#include "report.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iomanip>
#include <map>
#include <sstream>
#include <stdexcept>
#include <istream>
#include <tuple>

namespace skbh {

const char* stage_state_name(StageState s) {
    switch (s) {
        case StageState::executed: return "executed";
        case StageState::fused: return "fused";
        case StageState::elided: return "elided";
        case StageState::setupOnly: return "setup-only";
        case StageState::unsupported: return "unsupported";
    }
    return "unsupported";
}

double median(std::vector<double> v) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t m = v.size() / 2;
    return v.size() % 2 ? v[m] : 0.5 * (v[m - 1] + v[m]);
}

namespace {

// Minimal streaming JSON emitter: objects and arrays track whether a comma
// is due; keys are written in the order the caller gives them.
class Json {
public:
    explicit Json(std::ostream& out) : out_(out) {}
    Json& begin(const char* key = nullptr, char open = '{') {
        sep(key);
        out_ << open;
        first_.push_back(true);
        return *this;
    }
    Json& end(char close = '}') {
        first_.pop_back();
        if (newline_) {
            out_ << '\n';
            newline_ = false;
        }
        out_ << close;
        return *this;
    }
    Json& str(const char* key, const std::string& v) {
        sep(key);
        quote(v);
        return *this;
    }
    Json& u64(const char* key, std::uint64_t v) {
        sep(key);
        out_ << v;
        return *this;
    }
    Json& num(const char* key, double v) {
        sep(key);
        number(v);
        return *this;
    }
    Json& boolean(const char* key, bool v) {
        sep(key);
        out_ << (v ? "true" : "false");
        return *this;
    }
    // The next item starts on a new line.
    Json& raw_newline() {
        newline_ = true;
        return *this;
    }
    void number(double v) {
        if (!std::isfinite(v)) {
            out_ << "null";
            return;
        }
        std::ostringstream s;
        s << std::setprecision(17) << v;
        out_ << s.str();
    }

private:
    void sep(const char* key) {
        if (!first_.empty()) {
            if (!first_.back()) out_ << ',';
            first_.back() = false;
        }
        if (newline_) {
            out_ << '\n';
            newline_ = false;
        }
        if (key) {
            quote(key);
            out_ << ':';
        }
    }
    void quote(const std::string& v) {
        out_ << '"';
        for (const char c : v) {
            switch (c) {
                case '"': out_ << "\\\""; break;
                case '\\': out_ << "\\\\"; break;
                case '\n': out_ << "\\n"; break;
                case '\r': out_ << "\\r"; break;
                case '\t': out_ << "\\t"; break;
                default:
                    if (static_cast<unsigned char>(c) < 0x20) {
                        char buf[8];
                        std::snprintf(buf, sizeof buf, "\\u%04x", c);
                        out_ << buf;
                    } else {
                        out_ << c;
                    }
            }
        }
        out_ << '"';
    }
    std::ostream& out_;
    std::vector<bool> first_;
    bool newline_ = false;
};

void direction(Json& j, const char* key, const DirectionContract& c) {
    j.begin(key)
        .str("nativePlacement", c.nativePlacement)
        .str("adapterPlacement", c.adapterPlacement)
        .boolean("destroysNativeInput", c.destroysNativeInput)
        .boolean("adapterPreservesCallerInput", c.adapterPreservesCallerInput)
        .boolean("requiresPreservationCopyForRepeatedExecution", c.requiresPreservationCopyForRepeatedExecution)
        .boolean("preservationIncludedInPrimitiveTiming", c.preservationIncludedInPrimitiveTiming)
        .boolean("preservationIncludedInAdapterTiming", c.preservationIncludedInAdapterTiming)
        .str("nativeInputRepresentationId", c.nativeInputRepresentationId)
        .str("nativeOutputRepresentationId", c.nativeOutputRepresentationId)
        .str("adapterInputRepresentationId", c.adapterInputRepresentationId)
        .str("adapterOutputRepresentationId", c.adapterOutputRepresentationId)
        .str("physicalExtents", c.physicalExtents)
        .str("stridesElements", c.stridesElements)
        .u64("paddingElements", c.paddingElements)
        .u64("minimumAlignmentBytes", c.minimumAlignmentBytes)
        .str("aliasing", c.aliasing)
        .u64("reusableWorkBytes", c.reusableWorkBytes)
        .boolean("outputCanFeedOppositeDirection", c.outputCanFeedOppositeDirection)
        .end();
}

void csv_field(std::ostream& out, const std::string& v) {
    if (v.find_first_of(",\"\n") == std::string::npos) {
        out << v;
        return;
    }
    out << '"';
    for (const char c : v) {
        if (c == '"') out << '"';
        out << c;
    }
    out << '"';
}

std::vector<std::string> split_csv(const std::string& line) {
    std::vector<std::string> fields(1);
    bool quoted = false;
    for (size_t i = 0; i < line.size(); ++i) {
        const char c = line[i];
        if (quoted) {
            if (c == '"' && i + 1 < line.size() && line[i + 1] == '"') {
                fields.back() += '"';
                ++i;
            } else if (c == '"') {
                quoted = false;
            } else {
                fields.back() += c;
            }
        } else if (c == '"') {
            quoted = true;
        } else if (c == ',') {
            fields.emplace_back();
        } else {
            fields.back() += c;
        }
    }
    return fields;
}

}  // namespace

void write_json(const Report& r, std::ostream& out) {
    Json j(out);
    const double verticalFraction = r.nz > 1 ? double(r.nj) / double(r.nz - 1) : 0.0;
    const std::uint64_t nxHalf = r.nx / 2 + 1, planes = r.nz * r.fields;
    j.begin();
    j.raw_newline().str("schema", r.schema);
    j.raw_newline().str("status", r.status);
    j.raw_newline().begin("numericType").str("id", r.scalarTypeId).u64("scalarBits", r.scalarBits).end();
    j.raw_newline()
        .begin("run")
        .str("id", r.runId)
        .str("profile", r.profile)
        .u64("seed", r.seed)
        .u64("warmups", r.warmups)
        .u64("samples", r.samples)
        .end();
    j.raw_newline()
        .begin("provenance")
        .str("benchmarkRepository", "JeffreyEarly/spectral-kernel-benchmarks")
        .str("waveVortexModelRepository", "JeffreyEarly/wave-vortex-model")
        .u64("waveVortexModelIssue", 129)
        .str("auditedProductionBaselineCommit", "be0f78995c49a2bfe4c43d75827856e3812ac278")
        .str("historicalHarnessCommit", "b63fef8f6a9e400c6ec560205906578b763d8298")
        .str("historicalDecisionCommit", "34797085d1b642b9d9c822f30a6b5c18e139c2bf")
        .end();
    j.raw_newline()
        .begin("logicalOperators")
        .str("horizontalForward", "T_h^+=P_h F_xy")
        .str("horizontalInverse", "T_h^-=F_xy^-1 E_h")
        .str("verticalForward", "T_z^+=V_f")
        .str("verticalInverse", "T_z^-=V_i")
        .str("verticalFixtureId", r.verticalMatrixFamilyId)
        .str("resultKey", "(k,l,j,field)")
        .end();
    j.raw_newline().begin("workload");
    j.u64("Nx", r.nx).u64("Ny", r.ny).u64("Nz", r.nz).u64("fields", r.fields);
    j.u64("H", r.ny * nxHalf).u64("Nkl", r.nkl).u64("Nj", r.nj).u64("planes", planes);
    j.begin("antialias")
        .boolean("enabled", r.antialias)
        .str("horizontalPolicy", "radial-two-thirds")
        .num("horizontalCutoffFraction", 2.0 / 3.0)
        .str("verticalPolicy", "floor(2*(Nz-1)/3)")
        .num("verticalRetainedFraction", verticalFraction)
        .end();
    j.begin("grouping")
        .str("realPlaneOrder", "x-fastest,y,z,field")
        .str("fullSpectrumOrder", "z-fastest,field,kx,ky")
        .str("retainedOrder", "z-fastest,field,radial-mode")
        .str("verticalColumnOrder", "field-fastest-within-radial-mode")
        .str("verticalMatrixFamilyId", r.verticalMatrixFamilyId)
        .u64("verticalGroupCount", r.verticalGroupCount);
    j.begin("verticalGroupModes")
        .u64("minimum", r.minGroupModes)
        .num("median", r.medianGroupModes)
        .u64("maximum", r.maxGroupModes)
        .end();
    j.begin("verticalGroupColumns")
        .u64("minimum", r.minGroupColumns)
        .num("median", r.medianGroupColumns)
        .u64("maximum", r.maxGroupColumns)
        .end();
    j.str("verticalGroupOrderHash", r.verticalGroupOrderHash).end();
    j.begin("stridesElements");
    j.begin("real").u64("x", 1).u64("y", r.nx).u64("z", r.nx * r.ny).u64("field", r.nx * r.ny * r.nz).end();
    j.begin("fullSpectrum").u64("z", 1).u64("field", r.nz).u64("kx", planes).u64("ky", planes * nxHalf).end();
    j.begin("retainedSpectrum").u64("z", 1).u64("field", r.nz).u64("mode", planes).end();
    j.begin("modalSpectrum").u64("j", 1).u64("field", r.nj).u64("mode", r.nj * r.fields).end();
    j.end();
    j.begin("bytes")
        .u64("real", r.realBytes)
        .u64("fullSpectrum", r.fullSpectrumBytes)
        .u64("retainedSpectrum", r.retainedSpectrumBytes)
        .u64("modalSpectrum", r.modalSpectrumBytes)
        .u64("verticalMatrixFamilySource", r.verticalMatrixFamilySourceBytes)
        .u64("verticalBenchmarkEstimatedExplicitPeak", r.verticalPeakBytes)
        .u64("orderingPackingEstimatedExplicitPeak", r.orderingPeakBytes)
        .u64("spectralPipelineEstimatedExplicitPeak", r.pipelinePeakBytes)
        .end();
    j.begin("permutationHashes")
        .str("retainedModeOrder", r.retainedModeOrderHash)
        .str("wvmFullSpectrumOrder", r.wvmFullSpectrumOrderHash)
        .end();
    j.end();
    const auto& e = r.environment;
    j.raw_newline()
        .begin("environment")
        .str("timestampUtc", e.timestampUtc)
        .str("hostname", e.hostname)
        .str("operatingSystem", e.operatingSystem)
        .str("machineModel", e.machineModel)
        .str("cpuBrand", e.cpuBrand)
        .u64("totalCores", e.totalCores)
        .u64("performanceCores", e.performanceCores)
        .u64("efficiencyCores", e.efficiencyCores)
        .u64("physicalMemoryBytes", e.physicalMemoryBytes)
        .str("compiler", e.compiler)
        .str("compilerVersion", e.compilerVersion)
        .str("compilerFlags", e.compilerFlags)
        .str("buildType", e.buildType)
        .str("gitCommit", e.gitCommit)
        .boolean("gitDirty", e.gitDirty)
        .end();
    j.raw_newline().begin("providers", '[');
    for (const auto& p : r.providers) {
        j.raw_newline().begin();
        j.str("id", p.id)
            .str("version", p.version)
            .str("libraryIdentity", p.libraryIdentity)
            .str("algorithmId", p.algorithmId)
            .str("nativeRepresentationId", p.nativeRepresentationId)
            .str("modeOrderId", p.modeOrderId)
            .str("schedulingId", p.schedulingId);
        j.begin("providerBuild")
            .str("sourceIdentity", p.sourceIdentity)
            .str("sourceSha256", p.sourceSha256)
            .str("configureFlags", p.configureFlags)
            .str("compilerFlags", p.compilerFlags)
            .end();
        j.u64("workers", p.workers);
        j.begin("scheduling")
            .u64("internalWorkers", p.internalWorkers)
            .u64("outerWorkers", p.outerWorkers)
            .u64("totalLogicalWorkers", p.workers)
            .end();
        j.u64("gemmCallsPerExecution", p.gemmCallsPerExecution);
        j.begin("executionContract");
        direction(j, "forward", p.forward);
        direction(j, "inverse", p.inverse);
        j.end();
        j.begin("setup")
            .num("totalSeconds", p.otherSetupSeconds + p.allocationSeconds + p.planningSeconds)
            .num("otherSeconds", p.otherSetupSeconds)
            .num("allocationSeconds", p.allocationSeconds)
            .num("wisdomGenerationSeconds", 0.0)
            .num("wisdomImportSeconds", 0.0)
            .end();
        j.begin("planning")
            .num("seconds", p.planningSeconds)
            .str("configuration", p.planningConfiguration)
            .u64("temporaryBytes", p.planningBytes)
            .u64("wisdomBytes", 0)
            .num("timeLimitSeconds", 0.0)
            .boolean("budgetExhausted", false)
            .end();
        j.begin("memory")
            .u64("persistentBytes", p.persistentBytes)
            .u64("scratchBytes", p.scratchBytes)
            .boolean("opaqueProviderMemory", p.opaqueProviderMemory)
            .end();
        j.begin("componentLedger", '[');
        for (const auto& l : p.ledger)
            j.begin().str("stage", l.stage).str("state", stage_state_name(l.state)).str("detail", l.detail).end();
        j.end(']');
        j.begin("timings", '[');
        for (const auto& t : p.timings) {
            j.begin()
                .str("scope", t.scope)
                .str("stage", t.stage)
                .str("direction", t.direction)
                .str("state", stage_state_name(t.state))
                .u64("bytesMoved", t.bytesMoved)
                .num("medianSeconds", median(t.seconds));
            j.begin("samplesSeconds", '[');
            for (const double s : t.seconds) j.num(nullptr, s);
            j.end(']').end();
        }
        j.end(']');
        j.begin("correctness", '[');
        for (const auto& m : p.correctness)
            j.begin()
                .str("name", m.name)
                .num("maximumRelativeError", m.maximumRelativeError)
                .num("relativeL2Error", m.relativeL2Error)
                .num("tolerance", m.tolerance)
                .boolean("passed", m.passed)
                .end();
        j.end(']');
        j.end();
    }
    j.raw_newline().end(']');
    j.raw_newline().end();
    out << '\n';
}

void write_csv(const Report& r, std::ostream& out) {
    out << "run_id,provider,scope,stage,direction,state,bytes_moved,sample_index,seconds\n";
    for (const auto& p : r.providers) {
        for (const auto& t : p.timings) {
            auto prefix = [&] {
                csv_field(out, r.runId);
                out << ',';
                csv_field(out, p.id);
                out << ',';
                csv_field(out, t.scope);
                out << ',';
                csv_field(out, t.stage);
                out << ',';
                csv_field(out, t.direction);
                out << ',';
                csv_field(out, stage_state_name(t.state));
                out << ',' << t.bytesMoved << ',';
            };
            if (t.seconds.empty()) {
                prefix();
                out << ",\n";
                continue;
            }
            for (size_t i = 0; i < t.seconds.size(); ++i) {
                prefix();
                out << i << ',' << std::setprecision(17) << t.seconds[i] << '\n';
            }
        }
    }
}

int compare_csv(std::istream& in, std::ostream& out) {
    std::string line;
    if (!std::getline(in, line)) throw std::runtime_error("CSV result is empty.");
    std::map<std::tuple<std::string, std::string, std::string, std::string>, std::vector<double>> groups;
    while (std::getline(in, line)) {
        const auto f = split_csv(line);
        if (f.size() != 9 || f[8].empty()) continue;
        groups[{f[1], f[2], f[3], f[4]}].push_back(std::stod(f[8]));
    }
    out << "provider\tscope\tstage\tdirection\tmedian_ms\tsamples\n";
    for (const auto& [key, values] : groups) {
        out << std::get<0>(key) << '\t' << std::get<1>(key) << '\t' << std::get<2>(key) << '\t' << std::get<3>(key)
            << '\t' << std::fixed << std::setprecision(6) << 1000.0 * median(values) << '\t' << values.size() << '\n';
    }
    return groups.empty() ? 1 : 0;
}

}  // namespace skbh
