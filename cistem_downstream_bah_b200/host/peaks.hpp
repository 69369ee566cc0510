// peaks.hpp -- peak list of a finished search: the loop of the reference's
// result aggregation (src/programs/match_template/match_template.cpp:1838-1975)
// over the scaled MIP, with Image::FindPeakWithIntegerCoordinates
// (src/core/image.cpp:9961-10110) as the peak search.
#pragma once
#include <string>
#include <vector>

namespace tmhost {

struct PeakInfo {
    float x_pos, y_pos;          // Angstrom (pixel coordinate x pixel size)
    float psi, theta, phi;       // degrees
    float defocus, pixel_size;   // offsets recorded by the search
    float peak_height;           // scaled MIP (z-score) at the peak
    int x, y;                    // pixel coordinates
};

// Repeatedly takes the first maximum of `scaled_mip` in scan order among
// pixels at least template_size/4+1 from every edge, stops when it is below
// `threshold`, records the best orientation there and blanks a disc of
// radius `min_peak_radius` pixels (the reference's half-open square bounds).
// `scaled_mip` is modified.  At most max_peaks peaks (the reference stops at 1000).
std::vector<PeakInfo> find_peaks(int nx, int ny, std::vector<float>& scaled_mip, const float* psi, const float* theta,
                                 const float* phi, const float* defocus, const float* pixel, float threshold,
                                 int min_peak_radius, int template_size, float pixel_size, int max_peaks = 1000);

// The peak records as text -- the values the reference stores in its project
// database -- next to the result image: <result file without .mrc>_peaks.txt,
// two comment lines, then x (A), y (A), psi, theta, phi, defocus, pixel size,
// peak height per line.  Returns the path written, empty on failure.
std::string write_peak_records(const std::string& result_file, const std::vector<PeakInfo>& peaks, float threshold,
                               int min_peak_radius);

}  // namespace tmhost

namespace tmhost {

// The result image of the reference's aggregation (match_template.cpp:1845-1966):
// the template (T^3 real volume, [z][y][x]) divided by the mean of its 100
// largest values on the three central planes (Image::ReturnAverageOfMaxN,
// image.cpp:11930-11974), transformed and scaled by sqrt(T*T*sqrt(T)), with
// the central pixel zeroed and the quadrants swapped; for each peak its
// Fourier slice at the peak's angles (ExtractSlice), scaled by T, transformed
// back, less its edge mean, and added where positive into an nx x ny image
// centred on the peak (InsertOtherImageAtSpecifiedPosition, image.cpp:8468-8520).
std::vector<float> projection_montage(const std::vector<float>& volume, int T, const std::vector<PeakInfo>& peaks,
                                      int nx, int ny);

}  // namespace tmhost
