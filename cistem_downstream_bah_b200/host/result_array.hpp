// result_array.hpp -- the distributed form of match_template: the search
// positions split into jobs (src/gui/MatchTemplatePanel.cpp:674-784), the flat
// float array a worker job sends back (src/programs/match_template/
// match_template.cpp:1373-1530), its merge on the master
// (AggregatedTemplateResult::AddResult, :2015-2103) and the master's statistics
// and histogram table (MasterHandleProgramDefinedResult, :1545-1837).
//
// Result array layout (floats):
//   [0] x size  [1] y size  [2] A = floats per image (FFTW padded layout,
//   (x + 2 - x % 2) * y)  [3] histogram bins  [4] correlation maps computed
//   [5] sqrt(padded pixels); then 8 images of A floats each -- MIP (unscaled),
//   psi, theta, phi, defocus, pixel size, sum, sum of squares -- then the
//   histogram as `bins` 8-byte longs (2 * bins floats).
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "peaks.hpp"
#include "prep.hpp"

namespace tmhost {

constexpr int kResultMetaValues = 6;   // match_template.cpp:6

// [first, last] search positions of each of `number_of_jobs` jobs for one
// image, as the panel assigns them (float counter, rounded ends).
std::vector<std::pair<int, int>> job_search_ranges(int number_of_search_positions, int number_of_jobs);

// Image::ReturnAverageOfRealValues(radius, false) (image.cpp:6263-6330):
// mean of the pixels within `radius` of the box centre (x/2, y/2); the mean
// of all pixels for radius <= 0.
float average_in_disc(const Image2& im, float radius);

// One worker's maps on its (rotated back) padded box, compact [y][x].
struct WorkerMaps {
    int nx = 0, ny = 0;
    std::vector<float> mip, psi, theta, phi, defocus, pixel, sum, sumsq;
};

// Worker side (match_template.cpp:1391-1530): each map is cut to the valid
// area (original size less remove_npix_from_edge) and padded back to the
// original size with its central average, then laid out as above.
std::vector<float> pack_worker_result(const WorkerMaps& m, long original_x, long original_y, int remove_npix_from_edge,
                                      float actual_number_of_ccs, double sqrt_input_pixels, const long* histogram,
                                      int histogram_bins);

// Master side: the running merge of the result arrays of one image.
class AggregatedTemplateResult {
public:
    // Merges one result array: the first one fixes the layout and the zeroed
    // collation buffer; MIP and best parameters where the MIP is strictly
    // larger; sums, sums of squares and histogram added; the count added.
    // Throws std::runtime_error on a malformed or mismatching array.
    void AddResult(const float* result_array, long array_size);

    int number_of_received_results = 0;
    float total_number_of_ccs = 0.0f;

    bool empty() const { return collated_.empty(); }
    int nx() const { return (int)collated_[0]; }
    int ny() const { return (int)collated_[1]; }
    long floats_per_image() const { return (long)collated_[2]; }
    int histogram_bins() const { return (int)collated_[3]; }
    double sqrt_input_pixels() const { return (double)collated_[5]; }
    // image k of the merged array, k = 0 (MIP) .. 7 (sum of squares)
    const float* image(int k) const { return collated_.data() + kResultMetaValues + floats_per_image() * k; }
    float* image(int k) { return collated_.data() + kResultMetaValues + floats_per_image() * k; }
    std::vector<long> histogram() const;
    const std::vector<float>& collated() const { return collated_; }

private:
    std::vector<float> collated_;
};

// What the master writes for one image once every job has reported.
struct MasterOutputs {
    int nx = 0, ny = 0;
    // compact [y][x]: MIP x sqrt(N), psi, theta, phi, defocus, pixel size,
    // scaled MIP (z), average x sqrt(N), standard deviation x sqrt(N)
    Image2 mip, psi, theta, phi, defocus, pixel, scaled_mip, avg, std_dev;
    float expected_threshold = 0.0f;
    // 512 rows: SNR, histogram, survival histogram, expected survival histogram
    std::vector<double> histogram_rows;
};

// The master's output images (:1608-1761: MIP and the statistics from the
// merged sums), expected threshold (:1790-1805) and histogram table
// (:1763-1836; with use_gpu the survival histogram is rescaled to the
// expected total, :1810-1825).
MasterOutputs finalize_master(const AggregatedTemplateResult& r, bool use_gpu);

// The histogram text file as the master writes it (:1777, 1807-1837).
bool write_master_histogram(const std::string& path, const MasterOutputs& o);

// Raw result-array files (native float32, no header).
bool write_result_array(const std::string& path, const std::vector<float>& a);
bool read_result_array(const std::string& path, std::vector<float>& a);

}  // namespace tmhost
