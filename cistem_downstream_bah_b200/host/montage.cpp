// montage.cpp -- the projection montage of the found peaks (see peaks.hpp).
#include <algorithm>
#include <cmath>
#include <complex>

#include "host_fft.hpp"
#include "peaks.hpp"
#include "prep.hpp"

namespace tmhost {

namespace {
constexpr float kPif = 3.14159265359f;

float deg2rad(float d) { return (float)((double)(d * kPif) / 180.); }

// RotationMatrix::SetToEulerRotation (matrix.cpp:490-510), the two columns used
void euler_columns(float phi, float theta, float psi, float* m) {
    const float cphi = cosf(deg2rad(phi)), sphi = sinf(deg2rad(phi));
    const float cth = cosf(deg2rad(theta)), sth = sinf(deg2rad(theta));
    const float cpsi = cosf(deg2rad(psi)), spsi = sinf(deg2rad(psi));
    m[0] = cphi * cth * cpsi - sphi * spsi;
    m[1] = -cphi * cth * spsi - sphi * cpsi;
    m[2] = sphi * cth * cpsi + cphi * spsi;
    m[3] = -sphi * cth * spsi + cphi * cpsi;
    m[4] = -sth * cpsi;
    m[5] = sth * spsi;
}

// Image::ReturnLinearInterpolatedFourier (image.cpp:2899-3020) on a T^3 half spectrum
std::complex<float> interp_fourier(const std::vector<std::complex<float>>& vol, int T, float x, float y, float z) {
    const int TP = T / 2 + 1, lb = -(T / 2), ub = T / 2 - 1;
    std::complex<float> acc(0.f, 0.f);
    const int i0 = (int)floorf(x), j0 = (int)floorf(y), k0 = (int)floorf(z);
    if (j0 < lb || j0 + 1 > ub || k0 < lb || k0 + 1 > ub) return acc;
    const float wx1 = x - (float)i0, wx0 = 1.f - wx1;
    if (x >= 0.f) {
        if (i0 + 1 > T / 2) return acc;
        for (int dk = 0; dk < 2; dk++) {
            const int k = k0 + dk, pz = k >= 0 ? k : T + k;
            const float wz = 1.f - fabsf(z - (float)k);
            for (int dj = 0; dj < 2; dj++) {
                const int j = j0 + dj, py = j >= 0 ? j : T + j;
                const float w = wz * (1.f - fabsf(y - (float)j));
                const std::complex<float>* row = vol.data() + ((size_t)pz * T + py) * TP;
                acc += row[i0] * (w * wx0) + row[i0 + 1] * (w * wx1);
            }
        }
    } else {
        if (i0 < -(T / 2)) return acc;
        for (int dk = 0; dk < 2; dk++) {
            const int k = k0 + dk, pz = k > 0 ? T - k : -k;
            const float wz = 1.f - fabsf(z - (float)k);
            for (int dj = 0; dj < 2; dj++) {
                const int j = j0 + dj, py = j > 0 ? T - j : -j;
                const float w = wz * (1.f - fabsf(y - (float)j));
                const std::complex<float>* row = vol.data() + ((size_t)pz * T + py) * TP;
                acc += std::conj(row[-i0]) * (w * wx0) + std::conj(row[-i0 - 1]) * (w * wx1);
            }
        }
    }
    return acc;
}
}  // namespace

std::vector<float> projection_montage(const std::vector<float>& volume, int T, const std::vector<PeakInfo>& peaks,
                                      int nx, int ny) {
    const int TP = T / 2 + 1, c = T / 2;
    // ReturnAverageOfMaxN(100): voxels on the three central planes
    std::vector<float> plane_vals;
    for (int k = 0; k < T; k++)
        for (int j = 0; j < T; j++)
            for (int i = 0; i < T; i++)
                if (i == c || j == c || k == c) plane_vals.push_back(volume[((size_t)k * T + j) * T + i]);
    std::sort(plane_vals.begin(), plane_vals.end());
    const size_t first = plane_vals.size() > 100 ? plane_vals.size() - 100 : 0;
    float max_density = 0.f;
    for (size_t i = first; i < plane_vals.size(); i++) max_density += plane_vals[i];
    max_density /= (float)(plane_vals.size() - first);
    // the volume's spectrum (ForwardFFT scaled 1/T^3), x sqrt(T*T*sqrt(T)), DC zeroed, quadrants swapped
    std::vector<float> vol(volume.size());
    for (size_t i = 0; i < vol.size(); i++) vol[i] = volume[i] / max_density;
    std::vector<std::complex<float>> spec = template_spectrum(vol, T, 1.0f);
    const float scale = sqrtf((float)T * (float)T * sqrtf((float)T));
    for (auto& v : spec) v *= scale;
    spec[0] = 0;   // already zero; the scaling keeps it so
    std::vector<float> out((size_t)nx * ny, 0.f);
    std::vector<cplx> slice((size_t)T * TP);
    std::vector<double> proj((size_t)T * T);
    for (const PeakInfo& p : peaks) {
        float m[6];
        euler_columns(p.phi, p.theta, p.psi, m);
        // ExtractSlice (image.cpp:2450-2607) without a resolution limit, DC zero
        for (int y = 0; y < T; y++) {
            const int j = y < T / 2 ? y : y - T;
            for (int i = 0; i < TP; i++) {
                std::complex<float> val(0.f, 0.f);
                if (i == 0) {
                    if (j != 0) {
                        const int jj = (j > 0 || j == -(T / 2)) ? j : -j;
                        val = interp_fourier(spec, T, m[1] * (float)jj, m[3] * (float)jj, m[5] * (float)jj);
                        if (jj != j) val = std::conj(val);
                    }
                } else {
                    const float fx = (float)i, fy = (float)j;
                    val = interp_fourier(spec, T, m[0] * fx + m[1] * fy, m[2] * fx + m[3] * fy, m[4] * fx + m[5] * fy);
                }
                // SwapRealSpaceQuadrants (even T: (-1)^(i+j)) and x sqrt(T*T)
                const float sgn = ((i + j) & 1) ? -1.f : 1.f;
                slice[(size_t)y * TP + i] = cplx(val * (sgn * (float)T));
            }
        }
        irfft2(T, T, slice.data(), proj.data());
        Image2 pimg;
        pimg.nx = pimg.ny = T;
        pimg.v.assign(proj.begin(), proj.end());
        const float e = edge_mean(pimg);
        // InsertOtherImageAtSpecifiedPosition with threshold 0 at the peak
        const int ox = nx / 2 + (p.x - nx / 2) - T / 2, oy = ny / 2 + (p.y - ny / 2) - T / 2;
        for (int jj = 0; jj < T; jj++)
            for (int ii = 0; ii < T; ii++) {
                const int x = ox + ii, y = oy + jj;
                const float v = pimg.v[(size_t)jj * T + ii] - e;
                if (x >= 0 && x < nx && y >= 0 && y < ny && v > 0.f) out[(size_t)y * nx + x] += v;
            }
    }
    return out;
}

}  // namespace tmhost
