// result_array.cpp -- see result_array.hpp.
#include "result_array.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "prep.hpp"

namespace tmhost {

namespace {

// myroundint(float) (src/core/functions.h:480-483): the 0.5 is a double
int round_half_away(float a) { return a > 0 ? (int)((double)a + 0.5) : (int)((double)a - 0.5); }

constexpr float kHistogramMin = -12.5f;   // match_template.cpp:24-26
constexpr float kHistogramMax = 22.5f;
constexpr int kMasterHistogramBins = 512;

// FFTW padded pitch of a real image of width nx (Image::Allocate, image.cpp:4792-4795)
int padded_pitch(int nx) { return nx + (nx % 2 == 0 ? 2 : 1); }

void put_padded(const Image2& im, float* dst) {
    const int pitch = padded_pitch(im.nx);
    for (int y = 0; y < im.ny; y++) {
        std::memcpy(dst + (size_t)y * pitch, im.v.data() + (size_t)y * im.nx, sizeof(float) * im.nx);
        for (int x = im.nx; x < pitch; x++) dst[(size_t)y * pitch + x] = 0.0f;
    }
}

Image2 get_compact(const float* src, int nx, int ny) {
    Image2 im;
    im.nx = nx;
    im.ny = ny;
    im.v.resize((size_t)nx * ny);
    const int pitch = padded_pitch(nx);
    for (int y = 0; y < ny; y++) std::memcpy(im.v.data() + (size_t)y * nx, src + (size_t)y * pitch, sizeof(float) * nx);
    return im;
}

}  // namespace

std::vector<std::pair<int, int>> job_search_ranges(int number_of_search_positions, int number_of_jobs) {
    // MatchTemplatePanel.cpp:674-675, 715, 775-780
    std::vector<std::pair<int, int>> out;
    if (number_of_search_positions <= 0 || number_of_jobs <= 0) return out;
    float per_job = float(number_of_search_positions) / float(number_of_jobs);
    if (per_job < 1) per_job = 1;
    float counter = 0;
    for (int job = 0; job < number_of_jobs; job++) {
        if (counter >= number_of_search_positions) counter = number_of_search_positions - 1;
        const int first = round_half_away(counter);
        counter += per_job;
        if (counter >= number_of_search_positions || job == number_of_jobs - 1) counter = number_of_search_positions - 1;
        const int last = round_half_away(counter);
        counter++;
        out.emplace_back(first, last);
    }
    return out;
}

float average_in_disc(const Image2& im, float radius) {
    double sum = 0.0;
    long n = 0;
    const int cx = im.nx / 2, cy = im.ny / 2;
    if (radius > 0.0f) {
        const float r2 = powf(radius, 2);
        const float z = powf(0 - 0, 2);
        for (int j = 0; j < im.ny; j++) {
            const float y = powf(float(j - cy), 2);
            for (int i = 0; i < im.nx; i++) {
                const float x = powf(float(i - cx), 2);
                const float d2 = x + y + z;
                if (d2 <= r2) {
                    sum += im.at(i, j);
                    n++;
                }
            }
        }
        return n > 0 ? float(sum / n) : 0.0f;
    }
    for (float v : im.v) sum += v;
    return float(sum / (double)im.v.size());
}

std::vector<float> pack_worker_result(const WorkerMaps& m, long original_x, long original_y, int remove_npix_from_edge,
                                      float actual_number_of_ccs, double sqrt_input_pixels, const long* histogram,
                                      int histogram_bins) {
    const size_t npix = (size_t)m.nx * m.ny;
    for (const std::vector<float>* v : {&m.mip, &m.psi, &m.theta, &m.phi, &m.defocus, &m.pixel, &m.sum, &m.sumsq})
        if (v->size() != npix) throw std::runtime_error("worker map size differs from its box");
    // match_template.cpp:1393-1406
    int trim_x = (int)original_x - remove_npix_from_edge;
    int trim_y = (int)original_y - remove_npix_from_edge;
    const float central_region = 0.35 * (m.nx + m.ny - 2 * remove_npix_from_edge);
    if (original_x > m.nx) trim_x = m.nx - remove_npix_from_edge;
    if (original_y > m.ny) trim_y = m.ny - remove_npix_from_edge;
    if (trim_x <= 0 || trim_y <= 0) throw std::runtime_error("the edge to remove covers the whole image");

    const long pitch = padded_pitch((int)original_x);
    const long per_image = pitch * original_y;
    std::vector<float> result((size_t)(kResultMetaValues + per_image * 8 + (long)histogram_bins * 2));
    result[0] = (float)original_x;
    result[1] = (float)original_y;
    result[2] = (float)per_image;
    result[3] = (float)histogram_bins;
    result[4] = actual_number_of_ccs;
    result[5] = (float)sqrt_input_pixels;
    // the order of the images in the array (:1469-1521)
    const std::vector<float>* maps[8] = {&m.mip, &m.psi, &m.theta, &m.phi, &m.defocus, &m.pixel, &m.sum, &m.sumsq};
    for (int k = 0; k < 8; k++) {
        Image2 im;
        im.nx = m.nx;
        im.ny = m.ny;
        im.v = *maps[k];
        const float central_average = average_in_disc(im, central_region);
        const Image2 trimmed = clip_into(im, trim_x, trim_y, central_average);
        const Image2 resized = clip_into(trimmed, (int)original_x, (int)original_y, central_average);
        put_padded(resized, result.data() + kResultMetaValues + per_image * k);
    }
    std::memcpy(result.data() + kResultMetaValues + per_image * 8, histogram, sizeof(long) * histogram_bins);
    return result;
}

void AggregatedTemplateResult::AddResult(const float* a, long array_size) {
    if (array_size < kResultMetaValues) throw std::runtime_error("result array shorter than its header");
    const long per_image = (long)a[2];
    const int bins = (int)a[3];
    if (a[0] < 1 || a[1] < 1 || per_image != (long)padded_pitch((int)a[0]) * (long)a[1] || bins < 0 ||
        array_size < kResultMetaValues + per_image * 8 + (long)bins * 2)
        throw std::runtime_error("malformed result array");
    if (collated_.empty()) {
        // AddResult (match_template.cpp:2020-2049): a zeroed buffer of the
        // array's size, with the header copied except the count
        collated_.assign((size_t)array_size, 0.0f);
        collated_[0] = a[0];
        collated_[1] = a[1];
        collated_[2] = a[2];
        collated_[3] = a[3];
        collated_[5] = a[5];
        number_of_received_results = 0;
        total_number_of_ccs = 0.0f;
    } else if (a[0] != collated_[0] || a[1] != collated_[1] || a[2] != collated_[2] || a[3] != collated_[3]) {
        throw std::runtime_error("result array layout differs from the first one received");
    }
    total_number_of_ccs += a[4];
    const float* src[8];
    for (int k = 0; k < 8; k++) src[k] = a + kResultMetaValues + per_image * k;
    float* dst[8];
    for (int k = 0; k < 8; k++) dst[k] = image(k);
    for (long p = 0; p < per_image; p++) {
        if (src[0][p] > dst[0][p]) {
            for (int k = 0; k < 6; k++) dst[k][p] = src[k][p];
        }
    }
    for (long p = 0; p < per_image; p++) dst[6][p] += src[6][p];
    for (long p = 0; p < per_image; p++) dst[7][p] += src[7][p];
    // the master adds its own histogram length (histogram_number_of_points)
    const int add_bins = bins < kMasterHistogramBins ? bins : kMasterHistogramBins;
    long* h = reinterpret_cast<long*>(dst[7] + per_image);
    const float* hs = src[7] + per_image;
    for (int i = 0; i < add_bins; i++) {
        long have, add;
        std::memcpy(&have, h + i, sizeof(long));
        std::memcpy(&add, hs + 2 * i, sizeof(long));
        have += add;
        std::memcpy(h + i, &have, sizeof(long));
    }
    number_of_received_results++;
}

std::vector<long> AggregatedTemplateResult::histogram() const {
    std::vector<long> h(histogram_bins());
    std::memcpy(h.data(), image(7) + floats_per_image(), sizeof(long) * h.size());
    return h;
}

MasterOutputs finalize_master(const AggregatedTemplateResult& r, bool use_gpu) {
    if (r.empty()) throw std::runtime_error("no result arrays received");
    MasterOutputs o;
    o.nx = r.nx();
    o.ny = r.ny();
    const long n = r.floats_per_image();
    const double sqrt_input_pixels = r.sqrt_input_pixels();
    std::vector<float> mip(r.image(0), r.image(0) + n);
    // MIP x sqrt(N) (:1608-1619)
    std::vector<float> scaled_out(n);
    for (long p = 0; p < n; p++) scaled_out[p] = mip[p] * sqrt_input_pixels;
    o.mip = get_compact(scaled_out.data(), o.nx, o.ny);
    o.psi = get_compact(r.image(1), o.nx, o.ny);
    o.theta = get_compact(r.image(2), o.nx, o.ny);
    o.phi = get_compact(r.image(3), o.nx, o.ny);
    o.defocus = get_compact(r.image(4), o.nx, o.ny);
    o.pixel = get_compact(r.image(5), o.nx, o.ny);
    // statistics (:1705-1727), in float as the master holds them
    std::vector<float> sums(r.image(6), r.image(6) + n), sq(r.image(7), r.image(7) + n);
    const float total = r.total_number_of_ccs;
    for (long p = 0; p < n; p++) {
        sums[p] /= total;
        sq[p] = sqrtf(sq[p] / total - powf(sums[p], 2));
        if (sq[p] > 0.0f) {
            mip[p] = (mip[p] - sums[p]) / sq[p];
        } else {
            sq[p] = 0.0f;
            mip[p] = 0.0f;
        }
    }
    o.scaled_mip = get_compact(mip.data(), o.nx, o.ny);
    for (long p = 0; p < n; p++) scaled_out[p] = sums[p] * sqrt_input_pixels;
    o.avg = get_compact(scaled_out.data(), o.nx, o.ny);
    for (long p = 0; p < n; p++) scaled_out[p] = sq[p] * sqrt_input_pixels;
    o.std_dev = get_compact(scaled_out.data(), o.nx, o.ny);

    // histogram (:1763-1836)
    const std::vector<long> hist = r.histogram();
    const int bins = kMasterHistogramBins;
    if ((int)hist.size() < bins) throw std::runtime_error("result histogram shorter than 512 bins");
    const float histogram_step = (kHistogramMax - kHistogramMin) / float(bins);
    const float temp_float = kHistogramMin + (histogram_step / 2.0f);
    std::vector<double> survival(bins, 0.0), expected(bins);
    survival[bins - 1] = (double)hist[bins - 1];
    for (int i = bins - 2; i >= 0; i--) survival[i] = survival[i + 1] + (double)hist[i];
    const float counted_area = (float)o.nx * (float)o.ny * total;
    for (int i = 0; i < bins; i++)
        expected[i] = (std::erfc((temp_float + histogram_step * float(i)) / sqrtf(2.0f)) / 2.0f) * counted_area;
    const double erf_input = 2.0 / (1.0 * ((double)(float)o.nx * (double)(float)o.ny * (double)total));
    o.expected_threshold = sqrtf(2.0f) * (float)erfcinv_approx(erf_input) * 1.0f;
    if (use_gpu) {
        double sum_expected = 0.0, sum_counted = 0.0;
        for (int i = 0; i < bins; i++) {
            sum_counted += survival[i];
            sum_expected += expected[i];
        }
        for (int i = 0; i < bins; i++) survival[i] *= (float)(sum_expected / sum_counted);
    }
    o.histogram_rows.resize((size_t)bins * 4);
    for (int i = 0; i < bins; i++) {
        o.histogram_rows[4 * i + 0] = temp_float + histogram_step * float(i);
        o.histogram_rows[4 * i + 1] = (double)hist[i];
        o.histogram_rows[4 * i + 2] = survival[i];
        o.histogram_rows[4 * i + 3] = expected[i];
    }
    return o;
}

bool write_master_histogram(const std::string& path, const MasterOutputs& o) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    std::fprintf(f, "# Expected threshold = %.2f\n", o.expected_threshold);
    std::fprintf(f, "# histogram, expected histogram, survival histogram, expected survival histogram\n");
    for (size_t i = 0; i + 3 < o.histogram_rows.size(); i += 4)
        std::fprintf(f, "%f %f %f %f\n", o.histogram_rows[i], o.histogram_rows[i + 1], o.histogram_rows[i + 2],
                     o.histogram_rows[i + 3]);
    return std::fclose(f) == 0;
}

bool write_result_array(const std::string& path, const std::vector<float>& a) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(a.data(), sizeof(float), a.size(), f) == a.size();
    return std::fclose(f) == 0 && ok;
}

bool read_result_array(const std::string& path, std::vector<float>& a) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (bytes < 0 || bytes % (long)sizeof(float) != 0) {
        std::fclose(f);
        return false;
    }
    a.resize((size_t)bytes / sizeof(float));
    const bool ok = std::fread(a.data(), sizeof(float), a.size(), f) == a.size();
    std::fclose(f);
    return ok;
}

}  // namespace tmhost
