// host_fft.hpp -- double-precision FFTs for the host-side preparation of the
// search inputs (micrograph whitening, template spectrum, pixel-size
// resampling).  Conventions of the reference's Image class
// (src/core/image.cpp:5085-5113): unnormalised transforms, half spectra of
// nx/2+1 complex values per row, c2r ignoring the imaginary parts of the DC
// and Nyquist terms.
#pragma once
#include <complex>
#include <vector>

namespace tmhost {

using cplx = std::complex<double>;

// in-place complex transform of length n (sign -1 forward, +1 inverse)
void fft1(std::vector<cplx>& x, int sign);

// 2-D r2c: in ny*nx reals, out ny*(nx/2+1) complex
void rfft2(int nx, int ny, const double* in, cplx* out);
// 2-D c2r: in ny*(nx/2+1) complex, out ny*nx reals (input preserved)
void irfft2(int nx, int ny, const cplx* in, double* out);
// 3-D r2c: in nz*ny*nx reals, out nz*ny*(nx/2+1) complex
void rfft3(int nx, int ny, int nz, const double* in, cplx* out);
// 3-D c2r (input preserved)
void irfft3(int nx, int ny, int nz, const cplx* in, double* out);

}  // namespace tmhost
