// peaks.cpp -- see peaks.hpp.
#include "peaks.hpp"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>

namespace tmhost {

namespace {
int myroundint(float a) { return a > 0 ? (int)(a + 0.5f) : (int)(a - 0.5f); }
}  // namespace

std::vector<PeakInfo> find_peaks(int nx, int ny, std::vector<float>& mip, const float* psi, const float* theta,
                                 const float* phi, const float* defocus, const float* pixel, float threshold,
                                 int min_peak_radius, int template_size, float pixel_size, int max_peaks) {
    std::vector<PeakInfo> out;
    const int edge = template_size / 4 + 1;
    const int i_min = edge, i_max = nx - edge, j_min = edge, j_max = ny - edge;
    const float r2 = powf((float)min_peak_radius, 2);
    while ((int)out.size() < max_peaks) {
        // FindPeakWithIntegerCoordinates(0, FLT_MAX, edge): first maximum in scan order
        float best = -FLT_MAX;
        int bi = 0, bj = 0;
        bool found = false;
        for (int j = j_min; j <= j_max && j < ny; j++)
            for (int i = i_min; i <= i_max && i < nx; i++) {
                const float v = mip[(size_t)j * nx + i];
                if (v > best) {
                    best = v;
                    bi = i;
                    bj = j;
                    found = true;
                }
            }
        if (!found || best < threshold) break;
        PeakInfo p{};
        const float cx = (float)bi, cy = (float)bj;   // peak + box centre = pixel coordinate
        p.x = bi;
        p.y = bj;
        p.x_pos = cx * pixel_size;
        p.y_pos = cy * pixel_size;
        for (int j = std::max(myroundint(cy) - min_peak_radius, 0); j < std::min(myroundint(cy) + min_peak_radius, ny); j++) {
            const float dy = ((float)j - cy) * ((float)j - cy);
            for (int i = std::max(myroundint(cx) - min_peak_radius, 0); i < std::min(myroundint(cx) + min_peak_radius, nx); i++) {
                const float dx = ((float)i - cx) * ((float)i - cx);
                const size_t a = (size_t)j * nx + i;
                if (dx == 0 && dy == 0) {
                    p.phi = phi[a];
                    p.theta = theta[a];
                    p.psi = psi[a];
                    p.defocus = defocus[a];
                    p.pixel_size = pixel[a];
                    p.peak_height = mip[a];
                }
                if (dx + dy <= r2) mip[a] = -FLT_MAX;
            }
        }
        out.push_back(p);
    }
    return out;
}

std::string write_peak_records(const std::string& result_file, const std::vector<PeakInfo>& peaks, float threshold,
                               int min_peak_radius) {
    std::string base = result_file;
    if (base.size() > 4 && base.compare(base.size() - 4, 4, ".mrc") == 0) base.resize(base.size() - 4);
    const std::string path = base + "_peaks.txt";
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return std::string();
    std::fprintf(f, "# %zu peaks above the expected threshold %.2f (min peak radius %d px)\n", peaks.size(), threshold,
                 min_peak_radius);
    std::fprintf(f, "# x (A), y (A), psi, theta, phi, defocus, pixel size, peak height\n");
    for (const PeakInfo& p : peaks)
        std::fprintf(f, "%f %f %f %f %f %f %f %f\n", p.x_pos, p.y_pos, p.psi, p.theta, p.phi, p.defocus, p.pixel_size,
                     p.peak_height);
    return std::fclose(f) == 0 ? path : std::string();
}

}  // namespace tmhost
