// template_matching_core.hpp -- C++ drop-in for the reference's
// TemplateMatchingCore (src/gpu/TemplateMatchingCore.h:55-179) over the C ABI
// of libtm_b200 (include/tm_b200.h).
//
// Method names, argument order and the public result members follow the
// reference so that the caller in match_template.cpp:849-986 reads the same:
//   core.Init(this, template_reconstruction, input_image, current_projection, ...);
//   core.RunInnerLoop(projection_filter, size_i, defocus_i, tIDX, position);
//   core.d_max_intensity_projection.CopyDeviceToHost(mip_buffer, true, false);
//   core.histogram.CopyToHostAndAdd(histogram_data);
// Differences, all deliberate:
//   * images are the light tmhost::Image below (compact layouts, no FFTW row
//     padding) instead of the wx-based Image;
//   * histogram_min_scaled / histogram_step_scaled are double, as the
//     reference CPU path (the parity target) keeps them;
//   * d_sum3 / d_sumSq3 hold double sums;
//   * errors throw tmhost::CoreError (status code + message) instead of
//     aborting the process.
#pragma once
#include <array>
#include <complex>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "tm_b200.h"

namespace tmhost {

// Real images: real_values [z][y][x] compact.  Fourier images: complex_values
// [z][y][x] with logical_x_dimension/2+1 values per row.
struct Image {
    int logical_x_dimension = 0, logical_y_dimension = 0, logical_z_dimension = 1;
    bool is_in_real_space = true;
    std::vector<float> real_values;
    std::vector<std::complex<float>> complex_values;

    void Allocate(int nx, int ny, int nz, bool real_space);
    void SetToConstant(float v);
    void CopyFrom(const Image* other) { *this = *other; }
    long ReturnNumberOfPixels() const { return (long)logical_x_dimension * logical_y_dimension * logical_z_dimension; }
};

// EulerSearch subset used by the search (euler_search.h): the grid of
// (phi, theta) search positions.
struct EulerSearch {
    int number_of_search_positions = 0;
    std::vector<std::array<float, 2>> list_of_search_parameters;   // phi, theta
    // InitGrid + (C1: theta_max = 180) + CalculateGridSearchPositions(false),
    // match_template.cpp:687-697; false on a bad symmetry string.
    bool InitGrid(const std::string& symmetry, float angular_step);
};

// AnglesAndShifts is only carried through Init's signature; the core builds
// its own rotation matrices on the device.
struct AnglesAndShifts {};

// Text progress bar on stderr (ProgressBar, src/core/progressbar.h).
class ProgressBar {
public:
    explicit ProgressBar(long total) : total_(total) {}
    ~ProgressBar();
    void Update(long done);
private:
    long total_;
    int last_pct_ = -1;
};

struct CoreError : std::runtime_error {
    int status;
    CoreError(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

class TemplateMatchingCore;

// One result map of the core (the reference's d_max_intensity_projection etc.).
class ResultMap {
public:
    // Copies the map into `dst` (allocated to the core's image size if it is not).
    void CopyDeviceToHost(Image& dst, bool should_block_until_complete = true, bool free_gpu_memory = false) const;
    void CopyDeviceToHost(std::vector<double>& dst) const;   // the double sums
    void Wait() const {}
private:
    friend class TemplateMatchingCore;
    const TemplateMatchingCore* core_ = nullptr;
    int which_ = 0;
};

// Histogram::CopyToHostAndAdd (src/gpu/Histogram.cu)
class HistogramResult {
public:
    void CopyToHostAndAdd(long* histogram_data) const;
private:
    friend class TemplateMatchingCore;
    const TemplateMatchingCore* core_ = nullptr;
};

class TemplateMatchingCore {
public:
    TemplateMatchingCore() = default;
    ~TemplateMatchingCore();
    TemplateMatchingCore(const TemplateMatchingCore&) = delete;
    TemplateMatchingCore& operator=(const TemplateMatchingCore&) = delete;

    // TemplateMatchingCore::Init (TemplateMatchingCore.cu:49-138).
    // template_reconstruction: quadrant-swapped template spectrum (Fourier);
    // input_image: whitened micrograph spectrum (Fourier); current_projection
    // fixes the projection box (must equal the template box).
    void Init(void* parent_pointer, Image& template_reconstruction, Image& input_image, Image& current_projection,
              float pixel_size_search_range, float pixel_size_step, float pixel_size,
              float defocus_search_range, float defocus_step, float defocus1, float defocus2,
              float psi_max, float psi_start, float psi_step,
              AnglesAndShifts& angles, EulerSearch& global_euler_search,
              double histogram_min_scaled, double histogram_step_scaled, int histogram_number_of_bins,
              int max_padding, int first_search_position, int last_search_position,
              ProgressBar* my_progress, long total_correlation_positions, bool is_running_locally,
              int device = 0);

    // TemplateMatchingCore::RunInnerLoop (TemplateMatchingCore.cu:140-368):
    // one (pixel size, defocus) plane over every search position and psi of
    // this core's range.  The per-plane results start from zero (MIP from
    // -FLT_MAX) as in the reference; the caller merges planes.
    void RunInnerLoop(Image& projection_filter, float c_pixel, float c_defocus, int threadIDX,
                      long& current_correlation_position);

    // The template spectrum may be replaced between planes (the reference
    // assigns template_reconstruction directly, match_template.cpp:880).
    void SetTemplate(const Image& template_reconstruction);

    ResultMap d_max_intensity_projection, d_best_psi, d_best_theta, d_best_phi, d_best_defocus, d_best_pixel_size;
    ResultMap d_sum3, d_sumSq3;
    HistogramResult histogram;
    long total_number_of_cccs_calculated = 0;

    int image_x() const { return dims_.image_x; }
    int image_y() const { return dims_.image_y; }
    double last_device_ms() const { return last_ms_; }

private:
    friend class ResultMap;
    friend class HistogramResult;
    void check(int status, const char* what) const;

    tm_ctx* ctx_ = nullptr;
    tm_dims dims_{};
    float psi_max_ = 0, psi_start_ = 0, psi_step_ = 0;
    float defocus_step_ = 0, pixel_size_step_ = 0;
    std::vector<float> orientations_;   // (phi, theta, psi) in the reference's loop order
    ProgressBar* progress_ = nullptr;
    double last_ms_ = 0;
    bool tuned_ = false;   // orientation batch picked at the first RunInnerLoop
    // host copies of the last plane's results
    std::vector<float> mip_, psi_, theta_, phi_, defocus_, pixel_;
    std::vector<double> sum_, sumsq_;
    std::vector<long long> hist_;
};

}  // namespace tmhost
