// Type-I vertical transforms of the constant-stratification kernel.
//
// In place on complex arrays data[row][storageChannels][nz] (z adjacent, re/im
// interleaved; T = double or float).  Channels first .. first+channels-1 of
// every row are transformed; bit c of dstMask selects the sine transform for
// channel first+c, otherwise the cosine one:
//   DCT-I (FFTW REDFT00, all nz points)
//     Y_k = x_0 + (-1)^k x_M + 2 sum_{z=1}^{M-1} x_z cos(pi k z / M),  M = nz-1
//   DST-I (FFTW RODFT00 on the nz-2 interior points, endpoints untouched)
//     Y_k = 2 sum_{z=1}^{M-1} x_z sin(pi k z / M),  k = 1 .. M-1
// With `normalize` the WVM forward normalisation of the reference
// (src/constant_stratification.cpp:199-231) follows in the same pass: DCT
// values times 1/(nz-1) with the last one halved, DST interior values times
// 1/(nz-1) and both endpoints set to zero.

#pragma once

#include <cuda_runtime.h>

namespace skb {

// tw: L = 2(nz-1) complex twiddles exp(-2 pi i m / L), m in [0, L), of the
// handle's precision.
cudaError_t launch_type1(bool f64, void* data, long long rows, int nz, int storageChannels, int first, int channels,
                         unsigned dstMask, bool normalize, const void* tw, cudaStream_t s);
// The normalisation alone (the reference's separate adapter pass).
cudaError_t launch_type1_normalize(bool f64, void* data, long long rows, int nz, int storageChannels, int first,
                                   int channels, unsigned dstMask, cudaStream_t s);
// True when the transform runs as a 2(nz-1)-point warp FFT of the symmetric
// extension; other lengths use a direct O(nz^2) sum per column.
bool type1_uses_fft(int nz);

}  // namespace skb
