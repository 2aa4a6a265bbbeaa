// Prepared spectral-flux fixture reader (see fixture.hpp).

#include "fixture.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <stdexcept>
#include <type_traits>
#include <utility>

namespace skbh {
namespace {

class Reader {
public:
    explicit Reader(const std::string& path) {
        std::ifstream in(path, std::ios::binary);
        if (!in) throw std::runtime_error("Unable to open prepared spectral-flux fixture: " + path);
        data_.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
    }
    void take(void* out, std::size_t bytes, const char* label) {
        if (bytes > data_.size() - at_)
            throw std::runtime_error(std::string("Prepared spectral-flux fixture is truncated at ") + label + '.');
        std::memcpy(out, data_.data() + at_, bytes);
        at_ += bytes;
    }
    template <typename T>
    T value(const char* label) {
        T v{};
        take(&v, sizeof v, label);
        return v;
    }
    template <typename T>
    std::vector<T> values(std::uint64_t count, const char* label) {
        if (count > (data_.size() - at_) / sizeof(T))
            throw std::runtime_error(std::string("Prepared spectral-flux fixture is truncated at ") + label + '.');
        std::vector<T> v(count);
        take(v.data(), count * sizeof(T), label);
        return v;
    }
    std::string string(const char* label) {
        const auto n = value<std::uint64_t>(label);
        if (n > data_.size() - at_)
            throw std::runtime_error(std::string("Prepared spectral-flux fixture is truncated at ") + label + '.');
        std::string s(data_.data() + at_, data_.data() + at_ + n);
        at_ += n;
        if (s.find('\0') != std::string::npos) throw std::runtime_error(std::string(label) + " contains NUL bytes.");
        return s;
    }
    bool finished() const { return at_ == data_.size(); }

private:
    std::vector<char> data_;
    std::size_t at_ = 0;
};

void require(bool ok, const char* message) {
    if (!ok) throw std::runtime_error(message);
}

template <typename T>
void require_finite(const std::vector<T>& v, const char* message) {
    for (const auto& x : v)
        if constexpr (std::is_same_v<T, double>) {
            require(std::isfinite(x), message);
        } else {
            require(std::isfinite(x.real()) && std::isfinite(x.imag()), message);
        }
}

}  // namespace

PreparedFixture load_prepared_fixture(const std::string& path, const std::vector<skb_retained_mode>& modes) {
    Reader r(path);
    char magic[8];
    r.take(magic, 8, "magic");
    require(std::memcmp(magic, "SKFXP001", 8) == 0, "Prepared spectral-flux fixture has the wrong magic.");
    require(r.value<std::uint32_t>("version") == 1, "Prepared spectral-flux fixture has an unsupported version.");
    require(r.value<std::uint32_t>("byte order") == 0x01020304u, "Prepared spectral-flux fixture has the wrong byte order.");
    require(r.value<std::uint32_t>("authoritative flag") == 1, "Prepared spectral-flux fixture is not authoritative.");
    require(r.value<std::uint32_t>("reserved word") == 0, "Prepared spectral-flux fixture reserved header word is nonzero.");
    PreparedFixture f;
    f.nx = r.value<std::uint64_t>("Nx");
    f.ny = r.value<std::uint64_t>("Ny");
    f.nz = r.value<std::uint64_t>("Nz");
    const auto nkl = r.value<std::uint64_t>("Nkl");
    f.nj = r.value<std::uint64_t>("Nj");
    const auto groups = r.value<std::uint64_t>("group count");
    const auto families = r.value<std::uint64_t>("family count");
    const auto inputs = r.value<std::uint64_t>("input count");
    const auto targets = r.value<std::uint64_t>("target count");
    require(f.nx > 0 && f.ny > 0 && f.nz > 0 && nkl > 0 && f.nj > 0 && groups > 0, "Invalid fixture dimension.");
    require(families == 2, "Spectral-flux fixture must contain wave-f and wave-g.");
    require(inputs == 15, "Spectral-flux fixture must contain 15 input fields.");
    require(targets == 4, "Spectral-flux fixture must contain four targets.");
    f.lx = r.value<double>("Lx");
    f.ly = r.value<double>("Ly");
    f.lz = r.value<double>("Lz");
    f.latitude = r.value<double>("latitude");
    f.pointwiseScale = r.value<double>("pointwise scale");
    require(f.nx == f.ny && f.nx % 2 == 0, "The authoritative path requires an even square horizontal grid.");
    require(f.lx == f.ly, "The authoritative path requires a square horizontal domain.");
    require(std::isfinite(f.lx) && f.lx > 0 && std::isfinite(f.lz) && f.lz > 0 && std::isfinite(f.latitude) &&
                std::isfinite(f.pointwiseScale) && f.pointwiseScale > 0,
            "Spectral-flux fixture contains invalid physical metadata.");
    const double cells = static_cast<double>(f.nx * f.ny);
    require(f.pointwiseScale == 1.0 / (cells * cells), "Spectral-flux fixture pointwise normalization is inconsistent.");
    require(f.nj == 2 * (f.nz - 1) / 3, "Spectral-flux fixture Nj violates floor(2*(Nz-1)/3).");
    f.fixtureId = r.string("fixture id");
    f.repository = r.string("WVM repository");
    f.commit = r.string("WVM commit");
    f.generator = r.string("generator identity");
    f.fixtureHash = r.string("fixture hash");
    f.normalization = r.string("normalization");
    f.modeMapping = r.string("mode mapping");
    f.derivativeConvention = r.string("derivative convention");
    require(!f.fixtureId.empty(), "Spectral-flux fixture id is empty.");
    require(f.repository == "JeffreyEarly/wave-vortex-model", "Spectral-flux fixture identifies the wrong WVM repository.");
    require(f.commit.size() == 40, "Spectral-flux fixture WVM commit is not a full object id.");
    require(f.fixtureHash.rfind("sha256:", 0) == 0 && f.fixtureHash.size() == 71,
            "Spectral-flux fixture identity is not SHA-256.");
    const auto keys = r.values<std::int32_t>(2 * nkl, "mode keys");
    const auto vertical = r.values<std::int32_t>(f.nj, "vertical mode keys");
    const auto groupOf = r.values<std::uint32_t>(nkl, "mode group indices");
    const auto groupKeys = r.values<std::uint64_t>(groups, "group keys");
    const auto inFam = r.values<std::uint32_t>(15, "input field families");
    const auto outFam = r.values<std::uint32_t>(4, "target field families");
    const std::uint64_t perGroup = f.nz * f.nj;
    const auto inverseRaw = r.values<double>(groups * 2 * perGroup, "inverse operator matrices");
    const auto forwardRaw = r.values<double>(groups * 2 * perGroup, "forward operator matrices");
    auto in = r.values<std::complex<double>>(nkl * 15 * f.nj, "modal inputs");
    auto out = r.values<std::complex<double>>(nkl * 4 * f.nj, "modal targets");
    require(r.finished(), "Prepared spectral-flux fixture contains trailing bytes.");

    for (std::uint64_t j = 0; j < f.nj; ++j)
        require(vertical[j] == static_cast<std::int32_t>(j), "Spectral-flux fixture vertical mode keys are not j=0..Nj-1.");
    std::map<std::pair<std::int64_t, std::int64_t>, std::uint64_t> source;
    for (std::uint64_t m = 0; m < nkl; ++m)
        require(source.emplace(std::make_pair<std::int64_t, std::int64_t>(keys[2 * m], keys[2 * m + 1]), m).second,
                "Spectral-flux fixture horizontal mode keys are not unique.");
    require(modes.size() == nkl, "Spectral-flux fixture retained horizontal mode count is inconsistent.");
    std::vector<std::uint64_t> order(nkl);
    for (std::uint64_t m = 0; m < nkl; ++m) {
        const auto it = source.find({modes[m].k, modes[m].l});
        require(it != source.end(), "Spectral-flux fixture is missing a retained horizontal mode key.");
        order[m] = it->second;
    }
    std::vector<bool> used(groups, false);
    for (std::uint64_t m = 0; m < nkl; ++m) {
        require(groupOf[m] < groups, "Spectral-flux fixture mode group index is out of range.");
        require(m == 0 || groupOf[m] >= groupOf[m - 1], "Spectral-flux fixture mode groups are not contiguous.");
        const std::int64_t k = keys[2 * m], l = keys[2 * m + 1];
        require(groupKeys[groupOf[m]] == static_cast<std::uint64_t>(k * k + l * l),
                "Spectral-flux fixture group diagnostic key is inconsistent.");
        used[groupOf[m]] = true;
    }
    for (std::uint64_t g = 0; g < groups; ++g) {
        require(used[g], "Spectral-flux fixture does not use every declared mode group.");
        require(g == 0 || groupKeys[g] >= groupKeys[g - 1], "Spectral-flux fixture group diagnostic keys are not nondecreasing.");
    }
    const std::uint32_t wantIn[15] = {0, 0, 1, 0, 0, 1, 0, 0, 1, 1, 1, 0, 1, 1, 0};
    const std::uint32_t wantOut[4] = {0, 0, 1, 1};
    require(std::equal(inFam.begin(), inFam.end(), wantIn), "Spectral-flux fixture input field-to-operator map is inconsistent.");
    require(std::equal(outFam.begin(), outFam.end(), wantOut),
            "Spectral-flux fixture target-to-operator map is inconsistent.");
    require_finite(inverseRaw, "Inverse operator payload contains a non-finite value.");
    require_finite(forwardRaw, "Forward operator payload contains a non-finite value.");
    require_finite(in, "Modal input payload contains a non-finite value.");
    require_finite(out, "Modal target payload contains a non-finite value.");

    // Retained-mode order, operator groups as runs of one file group.
    f.modalInputs.resize(in.size());
    f.expectedTargets.resize(out.size());
    std::vector<std::uint32_t> runGroup;
    for (std::uint64_t m = 0; m < nkl; ++m) {
        const auto s = order[m];
        std::copy_n(in.begin() + s * 15 * f.nj, 15 * f.nj, f.modalInputs.begin() + m * 15 * f.nj);
        std::copy_n(out.begin() + s * 4 * f.nj, 4 * f.nj, f.expectedTargets.begin() + m * 4 * f.nj);
        const auto g = groupOf[s];
        if (runGroup.empty() || runGroup.back() != g) {
            runGroup.push_back(g);
            f.groupModes.push_back(1);
        } else {
            ++f.groupModes.back();
        }
    }
    for (std::uint64_t j = 0; j < 15 * f.nj; ++j)
        require(f.modalInputs[j].imag() == 0.0, "Spectral-flux fixture DC modal inputs must be real.");
    for (int fam = 0; fam < 2; ++fam) {
        f.forward[fam].resize(runGroup.size() * perGroup);
        f.inverse[fam].resize(runGroup.size() * perGroup);
        for (std::size_t g = 0; g < runGroup.size(); ++g) {
            const double* inv = inverseRaw.data() + (runGroup[g] * 2 + fam) * perGroup;  // (z, j) at z + Nz j
            const double* fwd = forwardRaw.data() + (runGroup[g] * 2 + fam) * perGroup;  // (j, z) at j + Nj z
            for (std::uint64_t z = 0; z < f.nz; ++z)
                for (std::uint64_t j = 0; j < f.nj; ++j) {
                    f.inverse[fam][g * perGroup + z * f.nj + j] = inv[z + f.nz * j];
                    f.forward[fam][g * perGroup + j * f.nz + z] = fwd[j + f.nj * z];
                }
        }
    }
    for (int i = 0; i < 15; ++i) f.inputFamily[i] = inFam[i];
    for (int i = 0; i < 4; ++i) f.targetFamily[i] = outFam[i];
    f.sourceGroups = groups;
    return f;
}

}  // namespace skbh
