// Separable direct DFTs in long double for validation.

#include "direct.hpp"

#include <algorithm>
#include <cmath>

namespace skbh {

std::vector<lcplx> unit_roots(std::uint64_t n, int sign) {
    std::vector<lcplx> out(n);
    const long double twoPi = 6.283185307179586476925286766559005768L;
    for (std::uint64_t k = 0; k < n; ++k) {
        const long double a = twoPi * static_cast<long double>(k) / static_cast<long double>(n);
        out[k] = lcplx(std::cos(a), sign * std::sin(a));
    }
    return out;
}

std::vector<cplx> direct_r2c(const skb_workload& w, const double* real) {
    const std::uint64_t nx = w.nx, ny = w.ny, nz = w.nz, planes = w.nz * w.fields, half = w.nx / 2 + 1;
    const auto rx = unit_roots(nx, -1), ry = unit_roots(ny, -1);
    std::vector<cplx> out(ny * half * planes);
    std::vector<lcplx> rows(ny * half);
    for (std::uint64_t p = 0; p < planes; ++p) {
        const double* f = real + p * nx * ny;
        for (std::uint64_t y = 0; y < ny; ++y)
            for (std::uint64_t kx = 0; kx < half; ++kx) {
                lcplx s = 0;
                for (std::uint64_t x = 0; x < nx; ++x) s += static_cast<long double>(f[y * nx + x]) * rx[(kx * x) % nx];
                rows[y * half + kx] = s;
            }
        const std::uint64_t field = p / nz, z = p % nz;
        for (std::uint64_t ky = 0; ky < ny; ++ky)
            for (std::uint64_t kx = 0; kx < half; ++kx) {
                lcplx s = 0;
                for (std::uint64_t y = 0; y < ny; ++y) s += rows[y * half + kx] * ry[(ky * y) % ny];
                out[((ky * half + kx) * w.fields + field) * nz + z] = cplx(double(s.real()), double(s.imag()));
            }
    }
    return out;
}

std::vector<double> direct_c2r(const skb_workload& w, const cplx* spectrum) {
    const std::uint64_t nx = w.nx, ny = w.ny, nz = w.nz, planes = w.nz * w.fields, half = w.nx / 2 + 1;
    const auto rx = unit_roots(nx, +1), ry = unit_roots(ny, +1);
    std::vector<double> out(nx * ny * planes);
    std::vector<lcplx> cols(ny * half);
    for (std::uint64_t p = 0; p < planes; ++p) {
        const std::uint64_t field = p / nz, z = p % nz;
        for (std::uint64_t y = 0; y < ny; ++y)
            for (std::uint64_t kx = 0; kx < half; ++kx) {
                lcplx s = 0;
                for (std::uint64_t ky = 0; ky < ny; ++ky) {
                    const cplx v = spectrum[((ky * half + kx) * w.fields + field) * nz + z];
                    s += lcplx(v.real(), v.imag()) * ry[(ky * y) % ny];
                }
                cols[y * half + kx] = s;
            }
        for (std::uint64_t y = 0; y < ny; ++y)
            for (std::uint64_t x = 0; x < nx; ++x) {
                long double s = cols[y * half].real();
                if (nx % 2 == 0 && nx > 1) s += ((x % 2) ? -1.0L : 1.0L) * cols[y * half + nx / 2].real();
                const std::uint64_t interior = (nx % 2 == 0) ? nx / 2 : half;
                for (std::uint64_t kx = 1; kx < interior; ++kx)
                    s += 2.0L * (cols[y * half + kx] * rx[(kx * x) % nx]).real();
                out[p * nx * ny + y * nx + x] = double(s);
            }
    }
    return out;
}

std::vector<cplx> gather(const skb_workload& w, const std::vector<skb_retained_mode>& modes, const cplx* spectrum,
                         double scale) {
    const std::uint64_t planes = w.nz * w.fields, half = w.nx / 2 + 1;
    std::vector<cplx> out(modes.size() * planes);
    for (std::size_t m = 0; m < modes.size(); ++m) {
        const auto& md = modes[m];
        for (std::uint64_t p = 0; p < planes; ++p) {
            cplx v = spectrum[(md.stored_ky * half + md.stored_kx) * planes + p];
            if (md.conjugates_stored_value) v = std::conj(v);
            out[m * planes + p] = scale * v;
        }
    }
    return out;
}

std::vector<cplx> embed(const skb_workload& w, const std::vector<skb_retained_mode>& modes, const cplx* retained) {
    const std::uint64_t planes = w.nz * w.fields, half = w.nx / 2 + 1;
    std::vector<cplx> out(w.ny * half * planes, cplx(0, 0));
    for (std::size_t m = 0; m < modes.size(); ++m) {
        const auto& md = modes[m];
        for (std::uint64_t p = 0; p < planes; ++p) {
            cplx v = retained[m * planes + p];
            if (md.conjugates_stored_value) v = std::conj(v);
            out[(md.stored_ky * half + md.stored_kx) * planes + p] = v;
            if (md.stored_kx == 0 && md.stored_ky != 0 && 2 * md.stored_ky != w.ny)
                out[((w.ny - md.stored_ky) * half) * planes + p] = std::conj(v);
        }
    }
    return out;
}

double max_relative_error(const cplx* a, const cplx* e, std::size_t n) {
    double num = 0, den = 0;
    for (std::size_t i = 0; i < n; ++i) {
        num = std::max(num, std::abs(a[i] - e[i]));
        den = std::max(den, std::abs(e[i]));
    }
    return num / std::max(den, 1.0);
}

double max_relative_error(const double* a, const double* e, std::size_t n, double scale) {
    double num = 0, den = 0;
    for (std::size_t i = 0; i < n; ++i) {
        num = std::max(num, std::abs(scale * a[i] - e[i]));
        den = std::max(den, std::abs(e[i]));
    }
    return num / std::max(den, 1.0);
}

double relative_l2_error(const cplx* a, const cplx* e, std::size_t n) {
    long double err = 0, ref = 0;
    for (std::size_t i = 0; i < n; ++i) {
        const long double dr = (long double)a[i].real() - e[i].real(), di = (long double)a[i].imag() - e[i].imag();
        err += dr * dr + di * di;
        ref += (long double)e[i].real() * e[i].real() + (long double)e[i].imag() * e[i].imag();
    }
    return ref == 0 ? double(std::sqrt(err)) : double(std::sqrt(err / ref));
}

double relative_l2_error(const double* a, const double* e, std::size_t n, double scale) {
    long double err = 0, ref = 0;
    for (std::size_t i = 0; i < n; ++i) {
        const long double d = (long double)scale * a[i] - e[i];
        err += d * d;
        ref += (long double)e[i] * e[i];
    }
    return ref == 0 ? double(std::sqrt(err)) : double(std::sqrt(err / ref));
}

}  // namespace skbh
