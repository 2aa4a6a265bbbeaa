#include "model.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <limits>
#include <random>
#include <set>
#include <stdexcept>
#include <thread>

namespace skb {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

std::vector<std::int64_t> dft_order(std::uint64_t n) {
    std::vector<std::int64_t> out;
    out.reserve(n);
    for (std::uint64_t v = 0; v < (n + 1) / 2; ++v) out.push_back(static_cast<std::int64_t>(v));
    for (std::uint64_t v = n / 2; v > 0; --v) out.push_back(-static_cast<std::int64_t>(v));
    return out;
}

bool self_conjugate(std::int64_t m, std::uint64_t n) {
    return m == 0 || (n % 2 == 0 && m == -static_cast<std::int64_t>(n / 2));
}

std::uint64_t wrap(std::int64_t m, std::uint64_t n) {
    return static_cast<std::uint64_t>(m >= 0 ? m : static_cast<std::int64_t>(n) + m);
}

std::uint64_t magnitude(std::int64_t v) {
    return v < 0 ? static_cast<std::uint64_t>(-(v + 1)) + 1 : static_cast<std::uint64_t>(v);
}

struct Fnv {
    std::uint64_t h = UINT64_C(14695981039346656037);
    template <typename T>
    void add(T value) {
        using U = std::make_unsigned_t<T>;
        const auto bits = static_cast<U>(value);
        for (std::size_t b = 0; b < sizeof(T); ++b) {
            h ^= static_cast<std::uint8_t>((bits >> (8 * b)) & 0xffu);
            h *= UINT64_C(1099511628211);
        }
    }
    std::string str() const {
        char buf[32];
        std::snprintf(buf, sizeof buf, "fnv1a64:%016llx", static_cast<unsigned long long>(h));
        return buf;
    }
};

}  // namespace

void validate_workload(const Workload& w) {
    if (w.nx < 2 || w.ny < 2 || w.nz < 1 || w.fields < 1)
        throw std::invalid_argument("workload: need Nx >= 2, Ny >= 2, Nz >= 1 and fields >= 1");
    if (!(w.lx > 0.0) || !(w.ly > 0.0)) throw std::invalid_argument("workload: Lx and Ly must be greater than zero");
}

std::vector<RetainedMode> retained_modes(const Workload& w) {
    validate_workload(w);
    const auto ks = dft_order(w.nx);
    const auto ls = dft_order(w.ny);
    const double maxK = 2.0 * kPi * (static_cast<double>(w.nx / 2) / w.lx);
    std::vector<RetainedMode> modes;
    modes.reserve(w.nxHalf() * w.ny);
    for (const auto l : ls) {
        for (const auto k : ks) {
            const bool primary = l > 0 || (self_conjugate(l, w.ny) && (k > 0 || self_conjugate(k, w.nx)));
            const bool nyquist = (w.nx % 2 == 0 && k == -static_cast<std::int64_t>(w.nx / 2)) ||
                                 (w.ny % 2 == 0 && l == -static_cast<std::int64_t>(w.ny / 2));
            if (!primary || nyquist) continue;
            const double pk = 2.0 * kPi * static_cast<double>(k) / w.lx;
            const double pl = 2.0 * kPi * static_cast<double>(l) / w.ly;
            // Stored through volatile: the radius bits must not depend on FMA contraction.
            volatile double pk2 = pk * pk;
            volatile double pl2 = pl * pl;
            const double radial = std::sqrt(pk2 + pl2);
            if (w.antialias && radial > 2.0 * maxK / 3.0) continue;
            RetainedMode m;
            m.k = k;
            m.l = l;
            m.radial = radial;
            if (k >= 0) {
                m.kx = static_cast<std::uint64_t>(k);
                m.ky = wrap(l, w.ny);
            } else {
                m.kx = static_cast<std::uint64_t>(-k);
                m.ky = wrap(-l, w.ny);
                m.conj = true;
            }
            modes.push_back(m);
        }
    }
    std::stable_sort(modes.begin(), modes.end(), [](const RetainedMode& a, const RetainedMode& b) {
        if (a.radial != b.radial) return a.radial < b.radial;
        if (a.k != b.k) return a.k < b.k;
        return a.l < b.l;
    });
    return modes;
}

std::vector<ModeGroup> squared_wavenumber_groups(const std::vector<RetainedMode>& modes) {
    if (modes.empty()) throw std::invalid_argument("K^2 grouping: the retained-mode list is empty");
    std::vector<ModeGroup> groups;
    std::set<std::uint64_t> closed;
    for (std::uint64_t i = 0; i < modes.size(); ++i) {
        const auto k = magnitude(modes[i].k);
        const auto l = magnitude(modes[i].l);
        const auto key = k * k + l * l;
        if (groups.empty() || groups.back().key != key) {
            if (closed.count(key))
                throw std::invalid_argument("K^2 grouping: a K^2 key reappears after its group closed (modes with one key must be adjacent)");
            if (!groups.empty()) closed.insert(groups.back().key);
            groups.push_back({key, i, 1});
        } else {
            ++groups.back().count;
        }
    }
    return groups;
}

std::string mode_order_hash(const std::vector<RetainedMode>& modes) {
    Fnv f;
    for (const auto& m : modes) {
        f.add(m.k);
        f.add(m.l);
    }
    return f.str();
}

std::string group_order_hash(const std::vector<ModeGroup>& groups) {
    Fnv f;
    for (const auto& g : groups) {
        f.add(g.key);
        f.add(g.first);
        f.add(g.count);
    }
    return f.str();
}

std::string wvm_order_hash(const Workload& w) {
    Fnv f;
    for (std::uint64_t ky = 0; ky < w.ny; ++ky) {
        const std::int64_t signedKy = ky <= w.ny / 2 ? static_cast<std::int64_t>(ky)
                                                     : static_cast<std::int64_t>(ky) - static_cast<std::int64_t>(w.ny);
        for (std::uint64_t kx = 0; kx < w.nxHalf(); ++kx)
            for (std::uint64_t field = 0; field < w.fields; ++field)
                for (std::uint64_t z = 0; z < w.nz; ++z) {
                    f.add(static_cast<std::int64_t>(kx));
                    f.add(signedKy);
                    f.add(z);
                    f.add(field);
                }
    }
    return f.str();
}

VerticalFamily orthonormal_family(std::uint64_t nz, std::uint64_t nj) {
    if (nz == 0 || nj == 0 || nj > nz) throw std::invalid_argument("Vertical fixture requires 1 <= Nj <= Nz.");
    VerticalFamily fam;
    fam.id = "orthonormal-dct2-truncated-v1";
    fam.nz = nz;
    fam.nj = nj;
    fam.groups = 1;
    fam.forward.resize(nj * nz);
    fam.inverse.resize(nz * nj);
    for (std::uint64_t j = 0; j < nj; ++j) {
        const double norm = j == 0 ? std::sqrt(1.0 / static_cast<double>(nz)) : std::sqrt(2.0 / static_cast<double>(nz));
        for (std::uint64_t z = 0; z < nz; ++z) {
            const double v = norm * std::cos(kPi * (static_cast<double>(z) + 0.5) * static_cast<double>(j) /
                                             static_cast<double>(nz));
            fam.forward[j * nz + z] = v;
            fam.inverse[z * nj + j] = v;
        }
    }
    return fam;
}

VerticalFamily k2_rotation_family(const Workload& w, const std::vector<ModeGroup>& groups) {
    if (w.lx != w.ly)
        throw std::invalid_argument("The exact integer K-squared fixture currently requires a square horizontal domain.");
    const auto base = orthonormal_family(w.nz, w.nj());
    VerticalFamily fam;
    fam.id = "synthetic-k2-grouped-orthonormal-dct2-pair-rotation-v1";
    fam.nz = base.nz;
    fam.nj = base.nj;
    fam.groups = groups.size();
    const auto elems = fam.nz * fam.nj;
    fam.forward.resize(fam.groups * elems);
    fam.inverse.resize(fam.groups * elems);
    for (std::uint64_t g = 0; g < fam.groups; ++g) {
        const auto key = groups[g].key;
        const double phase = static_cast<double>((key % UINT64_C(4093)) + 1) / 4094.0;
        const double c = std::cos(0.5 * kPi * phase);
        const double s = std::sin(0.5 * kPi * phase);
        double* F = fam.forward.data() + g * elems;
        double* I = fam.inverse.data() + g * elems;
        for (std::uint64_t j = 0; j < fam.nj; j += 2) {
            for (std::uint64_t z = 0; z < fam.nz; ++z) {
                const double a = base.forward[j * fam.nz + z];
                double ar = a;
                if (j + 1 < fam.nj) {
                    const double b = base.forward[(j + 1) * fam.nz + z];
                    ar = c * a + s * b;
                    const double br = -s * a + c * b;
                    F[(j + 1) * fam.nz + z] = br;
                    I[z * fam.nj + j + 1] = br;
                } else if ((key & 1U) != 0) {
                    ar = -a;
                }
                F[j * fam.nz + z] = ar;
                I[z * fam.nj + j] = ar;
            }
        }
    }
    return fam;
}

namespace {

// Symmetric tridiagonal eigen-decomposition by implicit QL with Wilkinson
// shifts (the textbook tql2 iteration).  d: diagonal (out: eigenvalues),
// e: sub-diagonal in e[1..n-1], z: n x n row-major, in: identity, out: columns
// are eigenvectors.
void tridiagonal_eigen(std::vector<double>& d, std::vector<double>& e, std::vector<double>& z, int n) {
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    double f = 0.0, tst1 = 0.0;
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        int m = l;
        while (m < n && std::fabs(e[m]) > eps * tst1) ++m;
        if (m > l) {
            int iter = 0;
            do {
                if (++iter > 60) throw std::runtime_error("tridiagonal eigen-solver did not converge");
                double g = d[l];
                double p = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(p, 1.0);
                if (p < 0) r = -r;
                d[l] = e[l] / (p + r);
                d[l + 1] = e[l] * (p + r);
                const double dl1 = d[l + 1];
                double h = g - d[l];
                for (int i = l + 2; i < n; ++i) d[i] -= h;
                f += h;
                p = d[m];
                double c = 1.0, c2 = c, c3 = c, el1 = e[l + 1], s = 0.0, s2 = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * e[i];
                    h = c * p;
                    r = std::hypot(p, e[i]);
                    e[i + 1] = s * r;
                    s = e[i] / r;
                    c = p / r;
                    p = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; ++k) {
                        h = z[k * n + i + 1];
                        z[k * n + i + 1] = s * z[k * n + i] + c * h;
                        z[k * n + i] = c * z[k * n + i] - s * h;
                    }
                }
                p = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * p;
                d[l] = c * p;
            } while (std::fabs(e[l]) > eps * tst1);
        }
        d[l] += f;
        e[l] = 0.0;
    }
}

}  // namespace

VerticalFamily sturm_liouville_family(const Workload& w, const std::vector<ModeGroup>& groups, std::uint64_t seed) {
    const int nz = static_cast<int>(w.nz);
    const auto nj = w.nj();
    if (nz < 2 || nj == 0) throw std::invalid_argument("Sturm-Liouville family requires Nz >= 2.");
    VerticalFamily fam;
    fam.id = "seeded-sturm-liouville-exponential-n2-v1";
    fam.nz = w.nz;
    fam.nj = nj;
    fam.groups = groups.size();
    const auto elems = fam.nz * fam.nj;
    fam.forward.resize(fam.groups * elems);
    fam.inverse.resize(fam.groups * elems);
    // Seeded stratification: N^2(z) = N0^2 exp((z - top)/h) on a unit-depth grid.
    std::mt19937_64 gen(seed);
    std::uniform_real_distribution<double> scaleHeight(0.1, 0.3);
    const double h = scaleHeight(gen);
    const double dz = 1.0 / static_cast<double>(nz);
    std::vector<double> inv(nz + 1);  // 1/N^2 at cell interfaces
    for (int i = 0; i <= nz; ++i) inv[i] = std::exp(-(static_cast<double>(i) * dz - 1.0) / h);
    // Groups are independent: split them over the host threads (set-up time
    // only; 7,486 groups of Nz = 129 take about 30 s on one thread).
    auto group_range = [&](std::uint64_t g0, std::uint64_t g1) {
        for (std::uint64_t g = g0; g < g1; ++g) {
            const double k2 = 4.0 * kPi * kPi * static_cast<double>(groups[g].key);
            std::vector<double> d(nz), e(nz, 0.0), z(static_cast<std::size_t>(nz) * nz, 0.0);
            for (int i = 0; i < nz; ++i) {
                const double up = i + 1 < nz ? inv[i + 1] : 0.0;  // Neumann top
                const double dn = i > 0 ? inv[i] : 0.0;           // Neumann bottom
                // K^2 enters weighted by 1/N^2, so the eigenvectors depend on the group.
                d[i] = (up + dn) / (dz * dz) + 1e-3 * k2 * 0.5 * (inv[i] + inv[i + 1]);
                if (i > 0) e[i] = -inv[i] / (dz * dz);
                z[static_cast<std::size_t>(i) * nz + i] = 1.0;
            }
            tridiagonal_eigen(d, e, z, nz);
            std::vector<int> order(nz);
            for (int i = 0; i < nz; ++i) order[i] = i;
            std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] < d[b]; });
            double* F = fam.forward.data() + g * elems;
            double* I = fam.inverse.data() + g * elems;
            for (std::uint64_t j = 0; j < nj; ++j) {
                const int col = order[j];
                // Sign convention: first nonzero entry positive.
                double sign = 1.0;
                for (int r = 0; r < nz; ++r) {
                    if (std::fabs(z[static_cast<std::size_t>(r) * nz + col]) > 1e-12) {
                        sign = z[static_cast<std::size_t>(r) * nz + col] < 0 ? -1.0 : 1.0;
                        break;
                    }
                }
                for (int r = 0; r < nz; ++r) {
                    const double v = sign * z[static_cast<std::size_t>(r) * nz + col];
                    F[j * fam.nz + r] = v;
                    I[r * fam.nj + j] = v;
                }
            }
        }
    };
    const std::uint64_t threads =
        std::min<std::uint64_t>(std::max(1u, std::thread::hardware_concurrency()), (fam.groups + 63) / 64);
    if (threads <= 1) {
        group_range(0, fam.groups);
        return fam;
    }
    std::vector<std::thread> pool;
    const std::uint64_t per = (fam.groups + threads - 1) / threads;
    for (std::uint64_t t = 0; t < threads; ++t) {
        const std::uint64_t g0 = t * per, g1 = std::min(fam.groups, g0 + per);
        if (g0 < g1) pool.emplace_back(group_range, g0, g1);
    }
    for (auto& th : pool) th.join();
    return fam;
}

std::vector<double> make_fixture(const Workload& w, int kind, std::uint64_t seed) {
    validate_workload(w);
    std::vector<double> values(w.realElements(), 0.0);
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> normal;
    for (std::uint64_t f = 0; f < w.fields; ++f) {
        for (std::uint64_t z = 0; z < w.nz; ++z) {
            const auto plane = z + w.nz * f;
            const double amp = 1.0 + 0.125 * static_cast<double>(plane);
            double* p = values.data() + plane * w.nx * w.ny;
            if (kind == 0) {
                p[(1 + plane) % w.nx + w.nx * ((2 + 3 * plane) % w.ny)] = amp;
                continue;
            }
            for (std::uint64_t y = 0; y < w.ny; ++y) {
                for (std::uint64_t x = 0; x < w.nx; ++x) {
                    double v = 0.0;
                    switch (kind) {
                        case 1: {
                            const double phase = 0.17 * static_cast<double>(plane);
                            v = amp * std::cos(2.0 * kPi *
                                                   (static_cast<double>(x) / static_cast<double>(w.nx) +
                                                    2.0 * static_cast<double>(y) / static_cast<double>(w.ny)) +
                                               phase);
                            break;
                        }
                        case 2: v = normal(gen); break;
                        case 3: v = amp; break;
                        case 4: v = amp * (((x + y) % 2 == 0) ? 1.0 : -1.0); break;
                        default: break;
                    }
                    p[x + w.nx * y] = v;
                }
            }
        }
    }
    return values;
}

std::vector<double> twiddle_table(std::uint64_t n) {
    std::vector<double> out(2 * n);
    const long double twoPi = 6.283185307179586476925286766559005768L;
    for (std::uint64_t k = 0; k < n; ++k) {
        // Reduce k/n to the first octant so every value is a long double
        // cos/sin of an angle in [0, pi/4], then place it by symmetry.
        std::uint64_t octant = (8 * k) / n;  // 0..7
        long double c, s;
        const std::uint64_t kk = 8 * k - octant * n;  // position inside the octant, times 8
        auto eval = [&](long double numer) {  // angle = 2 pi numer / (8 n)
            const long double a = twoPi * numer / (8.0L * static_cast<long double>(n));
            c = std::cos(a);
            s = std::sin(a);
        };
        double re, im;  // exp(-i theta), theta = 2 pi k / n
        if (octant % 2 == 0) {
            eval(static_cast<long double>(kk));
        } else {
            eval(static_cast<long double>(n - kk));
        }
        // Octant mapping of (cos theta, sin theta) from (c, s) of the reduced angle.
        double ct, st;
        const double cd = static_cast<double>(c), sd = static_cast<double>(s);
        switch (octant) {
            case 0: ct = cd; st = sd; break;
            case 1: ct = sd; st = cd; break;
            case 2: ct = -sd; st = cd; break;
            case 3: ct = -cd; st = sd; break;
            case 4: ct = -cd; st = -sd; break;
            case 5: ct = -sd; st = -cd; break;
            case 6: ct = sd; st = -cd; break;
            default: ct = cd; st = -sd; break;
        }
        re = ct;
        im = -st;
        out[2 * k] = re;
        out[2 * k + 1] = im;
    }
    return out;
}

ColumnTables column_tables(const Workload& w, const std::vector<RetainedMode>& modes, std::uint64_t columns) {
    ColumnTables t;
    t.activeKx = columns;
    t.cellMap.assign(columns * w.ny, -1);
    t.gatherMap.assign(columns * w.ny, -1);
    std::vector<std::vector<std::pair<int, int>>> perColumn(columns);
    t.modeKx.resize(modes.size());
    t.modeKy.resize(modes.size());
    t.modeConj.resize(modes.size());
    for (std::uint64_t m = 0; m < modes.size(); ++m) {
        const auto& mode = modes[m];
        if (mode.kx >= columns || mode.ky >= w.ny) throw std::invalid_argument("retained mode outside the column band");
        const int code = static_cast<int>(m << 1) | (mode.conj ? 1 : 0);
        t.cellMap[mode.kx * w.ny + mode.ky] = code;
        t.gatherMap[mode.kx * w.ny + mode.ky] = code;
        perColumn[mode.kx].push_back({static_cast<int>(mode.ky), code});
        t.modeKx[m] = static_cast<int>(mode.kx);
        t.modeKy[m] = static_cast<int>(mode.ky);
        t.modeConj[m] = mode.conj ? 1 : 0;
    }
    // kx = 0 Hermitian partners (model.cpp:332-335): (0, Ny - ky) holds the
    // conjugate of the stored value.
    for (std::uint64_t m = 0; m < modes.size(); ++m) {
        const auto& mode = modes[m];
        if (mode.kx == 0 && mode.ky != 0 && 2 * mode.ky != w.ny) {
            const auto partner = (w.ny - mode.ky) % w.ny;
            t.cellMap[partner] = static_cast<int>(m << 1) | (mode.conj ? 0 : 1);
        }
    }
    t.colStart.assign(columns + 1, 0);
    for (std::uint64_t c = 0; c < columns; ++c) {
        std::sort(perColumn[c].begin(), perColumn[c].end());
        t.colStart[c + 1] = t.colStart[c] + static_cast<int>(perColumn[c].size());
        for (const auto& [ky, code] : perColumn[c]) {
            t.colKy.push_back(ky);
            t.colMode.push_back(code);
        }
    }
    return t;
}

}  // namespace skb
