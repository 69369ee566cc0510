// prep.hpp -- host-side preparation around the GPU search, as the
// reference's MatchTemplateApp::DoCalculation does it
// (src/programs/match_template/match_template.cpp:519-724, 842-898, 1176-1370).
// Real images are compact [y][x] arrays; half spectra hold nx/2+1 complex
// values per row.
#pragma once
#include <complex>
#include <string>
#include <utility>
#include <vector>

namespace tmhost {

struct Image2 {
    int nx = 0, ny = 0;
    std::vector<float> v;   // [y][x]
    float& at(int x, int y) { return v[(size_t)y * nx + x]; }
    float at(int x, int y) const { return v[(size_t)y * nx + x]; }
};

// ReturnAverageOfRealValuesOnEdges, 2-D (image.cpp:5907-5945)
float edge_mean(const Image2& im);
// Image::ClipInto in real space, centre aligned (image.cpp:8554-8590); Resize (:8825-8839)
Image2 clip_into(const Image2& im, int ox, int oy, float pad);
// Rotate2DInPlaceBy90Degrees (image.cpp:11104-11140)
Image2 rotate90(const Image2& im, bool positive);
// match_template.cpp:539-583 for one dimension
int factorize_dimension(int original, int template_size);
bool is_power_of_two(int n);

struct Whitened {
    std::vector<std::complex<float>> spectrum;   // ny*(nx/2+1)
    std::vector<double> curve;                    // whitening filter on [0, sqrt(2)/2]
};
// match_template.cpp:711-724; refine_template.cpp:617-629 whitens the same way
// without the quadrant swap (swap_quadrants = false)
Whitened whiten(const Image2& micrograph, bool swap_quadrants = true);

// Image::SwapRealSpaceQuadrants of a half spectrum (object centred in the box)
void swap_quadrants(int nx, int ny, int nz, std::complex<double>* spec);

// The refine_template template spectrum (refine_template.cpp:586-599): the
// T^3 volume resized to TP^3 with its edge mean (padding factor TP/T), then
// ForwardFFT, ZeroCentralPixel and SwapRealSpaceQuadrants.
std::vector<std::complex<float>> padded_template_spectrum(const std::vector<float>& volume, int T, int TP);

// Template spectrum for the pixel-size factor (ChangePixelSize with
// return_fft, image.cpp:8705-8822, then ZeroCentralPixel and
// SwapRealSpaceQuadrants, match_template.cpp:842-845); volume is T^3 [z][y][x].
std::vector<std::complex<float>> template_spectrum(const std::vector<float>& volume, int T, float factor);

struct CtfParams {
    float kv, cs_mm, amplitude_contrast, defocus1, defocus2, astigmatism_angle_deg, pixel_size, phase_shift_deg;
};
// CalculateCTFImage x ApplyCurveFilter(whitening) on T x (T/2+1) (match_template.cpp:895-898)
std::vector<float> projection_filter(int T, const std::vector<double>& curve, const CtfParams& p, float defocus_offset);

// EulerSearch::InitGrid + C1 theta_max = 180 + CalculateGridSearchPositions(false)
// (euler_search.cpp:129-260, match_template.cpp:687-697); empty on a bad symmetry
std::vector<std::pair<float, float>> search_grid(float angular_step, const std::string& symmetry);
// for (psi = start; psi <= max; psi += step), float accumulation (match_template.cpp:746-750)
std::vector<float> psi_list(float psi_start, float psi_step, float psi_max);
// CalculateAngularStep (functions.cpp:629-632)
float angular_step_for(float resolution, float radius);
// cisTEM_erfcinv (functions.cpp:1270-1302)
double erfcinv_approx(double x);

}  // namespace tmhost
