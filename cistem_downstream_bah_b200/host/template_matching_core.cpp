// template_matching_core.cpp -- see template_matching_core.hpp.
#include <cstdlib>
#include <cstdio>
#include "template_matching_core.hpp"

#include <cfloat>
#include <cstring>

#include "prep.hpp"

namespace tmhost {

void Image::Allocate(int nx, int ny, int nz, bool real_space) {
    logical_x_dimension = nx;
    logical_y_dimension = ny;
    logical_z_dimension = nz;
    is_in_real_space = real_space;
    if (real_space) {
        real_values.assign((size_t)nx * ny * nz, 0.f);
        complex_values.clear();
    } else {
        complex_values.assign((size_t)(nx / 2 + 1) * ny * nz, std::complex<float>(0.f, 0.f));
        real_values.clear();
    }
}

void Image::SetToConstant(float v) {
    if (is_in_real_space) std::fill(real_values.begin(), real_values.end(), v);
    else std::fill(complex_values.begin(), complex_values.end(), std::complex<float>(v, 0.f));
}

bool EulerSearch::InitGrid(const std::string& symmetry, float angular_step) {
    const auto grid = search_grid(angular_step, symmetry);
    if (grid.empty()) return false;
    list_of_search_parameters.clear();
    for (const auto& pt : grid) list_of_search_parameters.push_back({pt.first, pt.second});
    number_of_search_positions = (int)grid.size();
    return true;
}

ProgressBar::~ProgressBar() { std::fprintf(stderr, "\n"); }

void ProgressBar::Update(long done) {
    const int pct = total_ > 0 ? (int)(100.0 * (double)done / (double)total_) : 100;
    if (pct != last_pct_) {
        last_pct_ = pct;
        std::fprintf(stderr, "\r%3d%% (%ld / %ld)", pct, done, total_);
        std::fflush(stderr);
    }
}

namespace {
enum Which { kMip, kPsi, kTheta, kPhi, kDefocus, kPixel, kSum, kSumSq };

struct ProgressCtx {
    ProgressBar* bar;
    long base;
};

int progress_cb(long long done, long long /*total*/, void* user) {
    auto* p = static_cast<ProgressCtx*>(user);
    if (p->bar) p->bar->Update(p->base + (long)done);
    return 0;
}
}  // namespace

void ResultMap::CopyDeviceToHost(Image& dst, bool, bool) const {
    if (!core_) throw CoreError(TM_ERR_INVALID, "result map read before Init");
    const int nx = core_->dims_.image_x, ny = core_->dims_.image_y;
    if (!dst.is_in_real_space || dst.logical_x_dimension != nx || dst.logical_y_dimension != ny ||
        dst.logical_z_dimension != 1)
        dst.Allocate(nx, ny, 1, true);
    const std::vector<float>* src = nullptr;
    switch (which_) {
        case kMip: src = &core_->mip_; break;
        case kPsi: src = &core_->psi_; break;
        case kTheta: src = &core_->theta_; break;
        case kPhi: src = &core_->phi_; break;
        case kDefocus: src = &core_->defocus_; break;
        case kPixel: src = &core_->pixel_; break;
        case kSum:
            for (size_t i = 0; i < dst.real_values.size(); i++) dst.real_values[i] = (float)core_->sum_[i];
            return;
        case kSumSq:
            for (size_t i = 0; i < dst.real_values.size(); i++) dst.real_values[i] = (float)core_->sumsq_[i];
            return;
    }
    if (src->size() != dst.real_values.size()) throw CoreError(TM_ERR_INVALID, "no results yet: run RunInnerLoop first");
    std::memcpy(dst.real_values.data(), src->data(), src->size() * sizeof(float));
}

void ResultMap::CopyDeviceToHost(std::vector<double>& dst) const {
    if (!core_ || (which_ != kSum && which_ != kSumSq)) throw CoreError(TM_ERR_INVALID, "not a sum map");
    dst = which_ == kSum ? core_->sum_ : core_->sumsq_;
}

void HistogramResult::CopyToHostAndAdd(long* histogram_data) const {
    if (!core_) throw CoreError(TM_ERR_INVALID, "histogram read before Init");
    for (size_t i = 0; i < core_->hist_.size(); i++) histogram_data[i] += (long)core_->hist_[i];
}

TemplateMatchingCore::~TemplateMatchingCore() {
    if (ctx_) tm_destroy(ctx_);
}

void TemplateMatchingCore::check(int status, const char* what) const {
    if (status == TM_OK) return;
    std::string msg = std::string(what) + " failed (status " + std::to_string(status) + ")";
    if (ctx_) msg += ": " + std::string(tm_last_error(ctx_));
    throw CoreError(status, msg);
}

void TemplateMatchingCore::Init(void*, Image& template_reconstruction, Image& input_image, Image& current_projection,
                                float /*pixel_size_search_range*/, float pixel_size_step, float /*pixel_size*/,
                                float /*defocus_search_range*/, float defocus_step, float /*defocus1*/, float /*defocus2*/,
                                float psi_max, float psi_start, float psi_step, AnglesAndShifts&,
                                EulerSearch& global_euler_search, double histogram_min_scaled,
                                double histogram_step_scaled, int histogram_number_of_bins, int /*max_padding*/,
                                int first_search_position, int last_search_position, ProgressBar* my_progress,
                                long /*total_correlation_positions*/, bool /*is_running_locally*/, int device) {
    if (template_reconstruction.is_in_real_space || input_image.is_in_real_space)
        throw CoreError(TM_ERR_INVALID, "Init expects the template and the micrograph in Fourier space");
    const int T = template_reconstruction.logical_x_dimension;
    if (template_reconstruction.logical_y_dimension != T || template_reconstruction.logical_z_dimension != T)
        throw CoreError(TM_ERR_INVALID, "the template must be a cube");
    if (current_projection.logical_x_dimension != T || current_projection.logical_y_dimension != T)
        throw CoreError(TM_ERR_UNSUPPORTED,
                        "the projection box must equal the template box (template padding is not supported)");
    if (first_search_position < 0 || last_search_position >= global_euler_search.number_of_search_positions ||
        first_search_position > last_search_position)
        throw CoreError(TM_ERR_INVALID, "search position range outside the grid");
    if (ctx_) { tm_destroy(ctx_); ctx_ = nullptr; }
    dims_ = tm_dims{};
    dims_.image_x = input_image.logical_x_dimension;
    dims_.image_y = input_image.logical_y_dimension;
    dims_.template_size = T;
    dims_.histogram_bins = histogram_number_of_bins;
    dims_.histogram_min_scaled = histogram_min_scaled;
    dims_.histogram_step_scaled = histogram_step_scaled;
    dims_.orientation_batch = 0;
    dims_.device = device;
    check(tm_create(&dims_, &ctx_), "tm_create");
    // Opt-in FP16 tensor-core form of the correlation transforms (the reference has
    // no counterpart; its default, the FP32 path, is the one that matches the CPU
    // program).  TM_B200_PRECISION=fp16 selects it where the geometry has the kernels.
    if (const char* prec = std::getenv("TM_B200_PRECISION")) {
        if (std::string(prec) == "fp16") {
            const int rc = tm_set_precision(ctx_, TM_PRECISION_FP16_TENSOR);
            if (rc == TM_ERR_UNSUPPORTED)
                std::fprintf(stderr, "TM_B200_PRECISION=fp16: %s; the FP32 path is used\n", tm_last_error(ctx_));
            else
                check(rc, "tm_set_precision");
        } else if (std::string(prec) != "fp32") {
            throw CoreError(TM_ERR_INVALID, "TM_B200_PRECISION must be fp32 or fp16");
        }
    }
    psi_max_ = psi_max;
    psi_start_ = psi_start;
    psi_step_ = psi_step;
    defocus_step_ = defocus_step;
    pixel_size_step_ = pixel_size_step;
    progress_ = my_progress;
    tuned_ = false;
    // orientation order of RunInnerLoop: search position outer, psi inner,
    // psi accumulated in float (TemplateMatchingCore.cu:200-206)
    orientations_.clear();
    for (int pos = first_search_position; pos <= last_search_position; pos++)
        for (float psi = psi_start; psi <= psi_max; psi += psi_step) {
            orientations_.push_back(global_euler_search.list_of_search_parameters[pos][0]);
            orientations_.push_back(global_euler_search.list_of_search_parameters[pos][1]);
            orientations_.push_back(psi);
        }
    SetTemplate(template_reconstruction);
    check(tm_set_image(ctx_, reinterpret_cast<const float*>(input_image.complex_values.data()), dims_.image_x,
                       dims_.image_y),
          "tm_set_image");
    for (ResultMap* m : {&d_max_intensity_projection, &d_best_psi, &d_best_theta, &d_best_phi, &d_best_defocus,
                         &d_best_pixel_size, &d_sum3, &d_sumSq3})
        m->core_ = this;
    d_max_intensity_projection.which_ = kMip;
    d_best_psi.which_ = kPsi;
    d_best_theta.which_ = kTheta;
    d_best_phi.which_ = kPhi;
    d_best_defocus.which_ = kDefocus;
    d_best_pixel_size.which_ = kPixel;
    d_sum3.which_ = kSum;
    d_sumSq3.which_ = kSumSq;
    histogram.core_ = this;
    total_number_of_cccs_calculated = 0;
}

void TemplateMatchingCore::SetTemplate(const Image& template_reconstruction) {
    if (!ctx_) throw CoreError(TM_ERR_INVALID, "SetTemplate before Init");
    check(tm_set_template(ctx_, reinterpret_cast<const float*>(template_reconstruction.complex_values.data()),
                          template_reconstruction.logical_x_dimension),
          "tm_set_template");
}

void TemplateMatchingCore::RunInnerLoop(Image& projection_filter, float c_pixel, float c_defocus, int,
                                        long& current_correlation_position) {
    if (!ctx_) throw CoreError(TM_ERR_INVALID, "RunInnerLoop before Init");
    const int T = dims_.template_size;
    if (projection_filter.logical_x_dimension != T || projection_filter.logical_y_dimension != T)
        throw CoreError(TM_ERR_INVALID, "projection filter size differs from the template box");
    // the CTF image is real-valued in complex slots; the core takes the real parts
    std::vector<float> filt((size_t)T * (T / 2 + 1));
    if (projection_filter.is_in_real_space) {
        if (projection_filter.real_values.size() != filt.size())
            throw CoreError(TM_ERR_INVALID, "real projection filter must hold T*(T/2+1) values");
        filt = projection_filter.real_values;
    } else {
        for (size_t i = 0; i < filt.size(); i++) filt[i] = projection_filter.complex_values[i].real();
    }
    const int n = (int)(orientations_.size() / 3);
    if (!tuned_) {
        // orientations per device pass, timed on the start of this core's range
        int chosen = 0;
        const int m = n < 256 ? n : 256;
        if (m >= 64) check(tm_autotune_batch(ctx_, filt.data(), orientations_.data(), m, &chosen), "tm_autotune_batch");
        tuned_ = true;
    }
    check(tm_reset_results(ctx_), "tm_reset_results");
    ProgressCtx pc{progress_, current_correlation_position};
    check(tm_run_plane(ctx_, filt.data(), orientations_.data(), n, c_defocus * defocus_step_, c_pixel * pixel_size_step_,
                       progress_cb, &pc),
          "tm_run_plane");
    double ms = 0;
    tm_last_timing(ctx_, &ms, nullptr, nullptr, nullptr);
    last_ms_ = ms;
    const size_t npix = (size_t)dims_.image_x * dims_.image_y;
    mip_.resize(npix); psi_.resize(npix); theta_.resize(npix); phi_.resize(npix);
    defocus_.resize(npix); pixel_.resize(npix); sum_.resize(npix); sumsq_.resize(npix);
    hist_.assign(dims_.histogram_bins, 0);
    check(tm_get_results(ctx_, mip_.data(), psi_.data(), theta_.data(), phi_.data(), defocus_.data(), pixel_.data(),
                         sum_.data(), sumsq_.data(), hist_.data()),
          "tm_get_results");
    total_number_of_cccs_calculated = n;
    current_correlation_position += n;
}

}  // namespace tmhost
