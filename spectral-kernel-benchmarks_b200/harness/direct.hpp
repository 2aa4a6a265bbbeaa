// Direct (O(N^3) separable, long double) transforms the `validate` command and
// the `run` correctness probes compare the GPU provider against, as the
// reference's validate compares its providers against directR2C / directC2R /
// directRetained (src/benchmark.cpp:4898-4996).

#pragma once

#include <complex>
#include <cstdint>
#include <vector>

#include "skb_cuda.h"

namespace skbh {

using cplx = std::complex<double>;
using lcplx = std::complex<long double>;

// exp(sign * 2 pi i * k / n) for k in [0, n), in long double.
std::vector<lcplx> unit_roots(std::uint64_t n, int sign);

// Real [field][z][y][x] -> WVM spectrum [ky][kx][field][z] (unnormalised).
std::vector<cplx> direct_r2c(const skb_workload& w, const double* real);
// WVM spectrum -> real, with FFTW's c2r semantics: the y transform first, then
// the x transform that ignores the imaginary parts of the kx = 0 and
// kx = Nx/2 bins.  Unnormalised (Nx*Ny times the input of a forward).
std::vector<double> direct_c2r(const skb_workload& w, const cplx* spectrum);
// Retained [mode][field][z] from a WVM spectrum (conjugated where the mode's
// stored value is its conjugate partner), times `scale`.
std::vector<cplx> gather(const skb_workload& w, const std::vector<skb_retained_mode>& modes, const cplx* spectrum,
                         double scale = 1.0);
// WVM spectrum holding only the retained modes, with the kx = 0 Hermitian
// partner (0, Ny - ky) written for ky != 0, 2 ky != Ny.
std::vector<cplx> embed(const skb_workload& w, const std::vector<skb_retained_mode>& modes, const cplx* retained);

// max |a - e| / max(max |e|, 1) and ||a - e|| / ||e|| (the reference's
// metrics, src/model.cpp:718-751).
double max_relative_error(const cplx* a, const cplx* e, std::size_t n);
double max_relative_error(const double* a, const double* e, std::size_t n, double scale = 1.0);
double relative_l2_error(const cplx* a, const cplx* e, std::size_t n);
double relative_l2_error(const double* a, const double* e, std::size_t n, double scale = 1.0);

}  // namespace skbh
