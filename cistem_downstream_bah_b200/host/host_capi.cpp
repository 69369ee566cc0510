// host_capi.cpp -- C entry points of the host preparation library
// (libtm_host.so), so that tests can hold the C++ preparation against the
// oracle and against numpy.  Complex arrays are interleaved float pairs.
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "host_fft.hpp"
#include "mrc.hpp"
#include "peaks.hpp"
#include "refine.hpp"
#include "result_array.hpp"
#include "prep.hpp"

#define TMH_API extern "C" __attribute__((visibility("default")))

using namespace tmhost;

namespace {
Image2 wrap(int nx, int ny, const float* v) {
    Image2 im;
    im.nx = nx;
    im.ny = ny;
    im.v.assign(v, v + (size_t)nx * ny);
    return im;
}
}  // namespace

// whitened half spectrum (ny*(nx/2+1) complex) and the curve; returns the
// number of curve points written (at most curve_cap)
TMH_API int tmh_whiten(int nx, int ny, const float* image, float* spec_out, double* curve_out, int curve_cap) {
    Whitened w = whiten(wrap(nx, ny, image));
    std::memcpy(spec_out, w.spectrum.data(), w.spectrum.size() * sizeof(float) * 2);
    const int n = (int)w.curve.size() < curve_cap ? (int)w.curve.size() : curve_cap;
    std::memcpy(curve_out, w.curve.data(), n * sizeof(double));
    return (int)w.curve.size();
}

TMH_API void tmh_template_spectrum(int T, const float* volume, float factor, float* spec_out) {
    std::vector<float> vol(volume, volume + (size_t)T * T * T);
    auto s = template_spectrum(vol, T, factor);
    std::memcpy(spec_out, s.data(), s.size() * sizeof(float) * 2);
}

TMH_API void tmh_projection_filter(int T, const double* curve, int curve_n, float kv, float cs_mm, float amp, float df1,
                                   float df2, float ang_deg, float pixel, float phase_deg, float defocus_offset,
                                   float* out) {
    std::vector<double> c(curve, curve + curve_n);
    CtfParams p{kv, cs_mm, amp, df1, df2, ang_deg, pixel, phase_deg};
    auto f = projection_filter(T, c, p, defocus_offset);
    std::memcpy(out, f.data(), f.size() * sizeof(float));
}

TMH_API int tmh_search_grid(const char* symmetry, float angular_step, float* out, int max_out) {
    auto g = search_grid(angular_step, symmetry);
    for (int i = 0; i < (int)g.size() && i < max_out; i++) {
        out[2 * i] = g[i].first;
        out[2 * i + 1] = g[i].second;
    }
    return g.empty() ? -1 : (int)g.size();
}

TMH_API int tmh_psi_list(float start, float step, float max, float* out, int max_out) {
    auto p = psi_list(start, step, max);
    for (int i = 0; i < (int)p.size() && i < max_out; i++) out[i] = p[i];
    return (int)p.size();
}

TMH_API int tmh_factorize_dimension(int original, int template_size) { return factorize_dimension(original, template_size); }
TMH_API int tmh_is_power_of_two(int n) { return is_power_of_two(n) ? 1 : 0; }
TMH_API float tmh_angular_step(float resolution, float radius) { return angular_step_for(resolution, radius); }
TMH_API double tmh_erfcinv(double x) { return erfcinv_approx(x); }
TMH_API float tmh_edge_mean(int nx, int ny, const float* image) { return edge_mean(wrap(nx, ny, image)); }

TMH_API void tmh_clip_into(int nx, int ny, const float* in, int ox, int oy, float pad, float* out) {
    Image2 o = clip_into(wrap(nx, ny, in), ox, oy, pad);
    std::memcpy(out, o.v.data(), o.v.size() * sizeof(float));
}

TMH_API void tmh_rotate90(int nx, int ny, const float* in, int positive, float* out) {
    Image2 o = rotate90(wrap(nx, ny, in), positive != 0);
    std::memcpy(out, o.v.data(), o.v.size() * sizeof(float));
}

// MRC: dims (nx, ny, nz) and pixel size of a file, then its data
TMH_API int tmh_mrc_info(const char* path, int* dims, float* pixel_size) {
    MrcData d;
    std::string err;
    if (!read_mrc(path, d, err)) return -1;
    dims[0] = d.nx; dims[1] = d.ny; dims[2] = d.nz;
    *pixel_size = d.pixel_size;
    return 0;
}

TMH_API int tmh_mrc_read(const char* path, float* out) {
    MrcData d;
    std::string err;
    if (!read_mrc(path, d, err)) return -1;
    std::memcpy(out, d.data.data(), d.data.size() * sizeof(float));
    return 0;
}

TMH_API int tmh_mrc_write(const char* path, int nx, int ny, int nz, const float* data, float pixel_size) {
    std::string err;
    return write_mrc(path, nx, ny, nz, data, pixel_size, err) ? 0 : -1;
}

// peak list of a scaled MIP (modified copy); out receives 10 floats per peak:
// x_pos, y_pos, psi, theta, phi, defocus, pixel_size, peak_height, x, y
TMH_API int tmh_find_peaks(int nx, int ny, const float* scaled_mip, const float* psi, const float* theta,
                           const float* phi, const float* defocus, const float* pixel, float threshold,
                           int min_peak_radius, int template_size, float pixel_size, float* out, int max_peaks) {
    std::vector<float> m(scaled_mip, scaled_mip + (size_t)nx * ny);
    auto pk = find_peaks(nx, ny, m, psi, theta, phi, defocus, pixel, threshold, min_peak_radius, template_size,
                         pixel_size, max_peaks);
    for (size_t k = 0; k < pk.size(); k++) {
        float* o = out + 10 * k;
        o[0] = pk[k].x_pos; o[1] = pk[k].y_pos; o[2] = pk[k].psi; o[3] = pk[k].theta; o[4] = pk[k].phi;
        o[5] = pk[k].defocus; o[6] = pk[k].pixel_size; o[7] = pk[k].peak_height; o[8] = (float)pk[k].x; o[9] = (float)pk[k].y;
    }
    return (int)pk.size();
}

// projection montage of peaks given as (x, y, psi, theta, phi) rows; volume T^3 [z][y][x]; out nx*ny
TMH_API void tmh_projection_montage(int T, const float* volume, int n_peaks, const float* peaks, int nx, int ny,
                                    float* out) {
    std::vector<float> vol(volume, volume + (size_t)T * T * T);
    std::vector<PeakInfo> pk(n_peaks);
    for (int k = 0; k < n_peaks; k++) {
        pk[k] = PeakInfo{};
        pk[k].x = (int)peaks[5 * k];
        pk[k].y = (int)peaks[5 * k + 1];
        pk[k].psi = peaks[5 * k + 2];
        pk[k].theta = peaks[5 * k + 3];
        pk[k].phi = peaks[5 * k + 4];
    }
    auto m = projection_montage(vol, T, pk, nx, ny);
    std::memcpy(out, m.data(), m.size() * sizeof(float));
}

// search-position ranges of n_jobs jobs: out receives first, last per job
TMH_API int tmh_job_search_ranges(int n_positions, int n_jobs, int* out) {
    const auto r = job_search_ranges(n_positions, n_jobs);
    for (size_t k = 0; k < r.size(); k++) {
        out[2 * k] = r[k].first;
        out[2 * k + 1] = r[k].second;
    }
    return (int)r.size();
}

// worker result array from 8 compact nx*ny maps (MIP, psi, theta, phi,
// defocus, pixel size, sum, sum of squares); returns its length in floats
// (written when it fits `cap`), -1 on bad arguments
TMH_API long tmh_pack_worker_result(int nx, int ny, const float* maps, long original_x, long original_y, int remove,
                                    float ccs, double sqrt_input_pixels, const long* histogram, int bins, float* out,
                                    long cap) {
    try {
        WorkerMaps m;
        m.nx = nx;
        m.ny = ny;
        const size_t n = (size_t)nx * ny;
        std::vector<float>* dst[8] = {&m.mip, &m.psi, &m.theta, &m.phi, &m.defocus, &m.pixel, &m.sum, &m.sumsq};
        for (int k = 0; k < 8; k++) dst[k]->assign(maps + n * k, maps + n * (k + 1));
        const auto r = pack_worker_result(m, original_x, original_y, remove, ccs, sqrt_input_pixels, histogram, bins);
        if ((long)r.size() <= cap) std::memcpy(out, r.data(), r.size() * sizeof(float));
        return (long)r.size();
    } catch (const std::exception&) {
        return -1;
    }
}

// the master over n result arrays: maps_out receives 9 compact images of the
// first array's size (MIP x sqrt(N), psi, theta, phi, defocus, pixel size,
// scaled MIP, average x sqrt(N), standard deviation x sqrt(N)), rows_out the
// 512 x 4 histogram table, stats_out {expected threshold, correlation maps}
TMH_API int tmh_merge_results(int n, const float* const* arrays, const long* sizes, int use_gpu, float* maps_out,
                              double* rows_out, double* stats_out) {
    try {
        AggregatedTemplateResult agg;
        for (int i = 0; i < n; i++) agg.AddResult(arrays[i], sizes[i]);
        const MasterOutputs o = finalize_master(agg, use_gpu != 0);
        const size_t npix = (size_t)o.nx * o.ny;
        const Image2* ims[9] = {&o.mip, &o.psi, &o.theta, &o.phi, &o.defocus, &o.pixel, &o.scaled_mip, &o.avg,
                                &o.std_dev};
        for (int k = 0; k < 9; k++) std::memcpy(maps_out + npix * k, ims[k]->v.data(), npix * sizeof(float));
        std::memcpy(rows_out, o.histogram_rows.data(), o.histogram_rows.size() * sizeof(double));
        stats_out[0] = o.expected_threshold;
        stats_out[1] = agg.total_number_of_ccs;
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// ---------------------------------------------------------------------------- refine_template
// whitened real micrograph of refine_template (whitening without the quadrant swap, back to real space)
TMH_API int tmh_refine_whiten(int nx, int ny, const float* image, float* out) {
    Whitened w = whiten(wrap(nx, ny, image), false);
    std::vector<std::complex<double>> spec(w.spectrum.begin(), w.spectrum.end());
    std::vector<double> real((size_t)nx * ny);
    irfft2(nx, ny, spec.data(), real.data());
    for (size_t i = 0; i < real.size(); i++) out[i] = (float)real[i];
    return (int)w.curve.size();
}

// peaks as refine_template picks them: out receives x, y (relative to the centre), value per peak
TMH_API int tmh_refine_find_peaks(int nx, int ny, const float* scaled_mip, float threshold, float min_peak_radius,
                                  float* out, int max_out) {
    RefineMaps m;
    m.nx = nx;
    m.ny = ny;
    m.scaled_mip.assign(scaled_mip, scaled_mip + (size_t)nx * ny);
    const auto pk = refine_find_peaks(m, threshold, min_peak_radius);
    const int n = (int)std::min<size_t>(pk.size(), (size_t)max_out);
    for (int k = 0; k < n; k++) {
        out[3 * k] = pk[k].x;
        out[3 * k + 1] = pk[k].y;
        out[3 * k + 2] = pk[k].value;
    }
    return (int)pk.size();
}

TMH_API void tmh_window_particle(int nx, int ny, const float* image, int px, int py, int T, float* out) {
    const auto w = window_particle(wrap(nx, ny, image), px, py, T);
    std::memcpy(out, w.data(), w.size() * sizeof(float));
}

TMH_API void tmh_cosine_mask(int T, float* image, float radius, float edge) {
    std::vector<float> v(image, image + (size_t)T * T);
    cosine_mask(v, T, radius, edge);
    std::memcpy(image, v.data(), v.size() * sizeof(float));
}

// info: identity, pad, new size, has pad value; matrices as in PixelSizeOperator (when not identity)
TMH_API int tmh_pixel_size_operator(int nin, int nout, float factor, float* ar, float* ai, float* brt, float* bit,
                                    int* info) {
    try {
        const PixelSizeOperator o = pixel_size_operator(nin, nout, factor);
        info[0] = o.identity ? 1 : 0;
        info[1] = o.pad;
        info[2] = o.new_size;
        info[3] = o.has_pad_value ? 1 : 0;
        if (!o.identity) {
            std::memcpy(ar, o.ar.data(), o.ar.size() * sizeof(float));
            std::memcpy(ai, o.ai.data(), o.ai.size() * sizeof(float));
            std::memcpy(brt, o.brt.data(), o.brt.size() * sizeof(float));
            std::memcpy(bit, o.bit.data(), o.bit.size() * sizeof(float));
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

TMH_API void tmh_padded_template_spectrum(int T, int TP, const float* volume, float* out) {
    std::vector<float> vol(volume, volume + (size_t)T * T * T);
    const auto spec = padded_template_spectrum(vol, T, TP);
    std::memcpy(out, spec.data(), spec.size() * sizeof(std::complex<float>));
}

// the descent of refine_template over `n_peaks` peaks with a synthetic score:
// value = 10 - ((phi - a)/3)^2 - ((theta - b)/3)^2 - ((psi - c)/3)^2
//         - ((defocus1 - d)/300)^2 - ((factor - e) 50)^2   (double, squares as products, per peak k: target[5k..5k+4])
// x = (int)floor(|phi - a| 10) % 3 - 1, y = (int)floor(|psi - c| 10) % 3 - 1.
// maps: 7 compact nx*ny images (mip, scaled mip, psi, theta, phi, defocus,
// pixel size); params: pixel size, defocus1, defocus2, angular step, in-plane
// step, defocus range, defocus step, pixel-size range, pixel-size step,
// xy threshold, exclude (0/1), threads.  maps_out: 7 images; per_peak: 16
// floats per peak (x, y, psi, theta, phi, defocus, pixel size, height, dx, dy,
// dpsi, dtheta, dphi, ddefocus, dpixel, dheight); log: the candidates scored,
// 6 floats each (phi, theta, psi, defocus1, factor, particle), up to max_log.
TMH_API long tmh_refine_synthetic(int nx, int ny, const float* maps, int n_peaks, const float* peaks_xy,
                                  const double* target, const float* params, float* maps_out, float* per_peak,
                                  float* log, long max_log) {
    RefineMaps m;
    m.nx = nx;
    m.ny = ny;
    const size_t np = (size_t)nx * ny;
    std::vector<float>* dst[7] = {&m.mip, &m.scaled_mip, &m.psi, &m.theta, &m.phi, &m.defocus, &m.pixel_size};
    for (int k = 0; k < 7; k++) dst[k]->assign(maps + np * k, maps + np * (k + 1));
    std::vector<FoundPeak> pk(n_peaks);
    for (int k = 0; k < n_peaks; k++) {
        pk[k].x = peaks_xy[2 * k];
        pk[k].y = peaks_xy[2 * k + 1];
    }
    RefineParams p;
    p.pixel_size = params[0];
    p.defocus1 = params[1];
    p.defocus2 = params[2];
    p.angular_step = params[3];
    p.in_plane_angular_step = params[4];
    p.defocus_search_range = params[5];
    p.defocus_search_step = params[6];
    p.pixel_size_search_range = params[7];
    p.pixel_size_search_step = params[8];
    p.xy_change_threshold = params[9];
    p.exclude_above_xy_threshold = params[10] != 0.0f;
    p.max_threads = (int)params[11];
    std::mutex log_mu;
    long n_log = 0;
    auto score = [&](const RefineCandidate& c) {
        const double* t = target + 5 * c.particle;
        const double a = (c.phi - t[0]) / 3.0, b = (c.theta - t[1]) / 3.0, d = (c.psi - t[2]) / 3.0;
        const double e = (c.defocus1 - t[3]) / 300.0, f = (c.pixel_size_factor - t[4]) * 50.0;
        const double v = 10.0 - a * a - b * b - d * d - e * e - f * f;
        RefineScore s;
        s.value = (float)v;
        s.x = (float)((int)std::floor(std::fabs(c.phi - t[0]) * 10.0) % 3 - 1);
        s.y = (float)((int)std::floor(std::fabs(c.psi - t[2]) * 10.0) % 3 - 1);
        std::lock_guard<std::mutex> lock(log_mu);
        if (n_log < max_log) {
            float* l = log + 6 * n_log;
            l[0] = c.phi; l[1] = c.theta; l[2] = c.psi; l[3] = c.defocus1; l[4] = c.pixel_size_factor;
            l[5] = (float)c.particle;
        }
        n_log++;
        return s;
    };
    const RefineOutputs out = refine_peaks(m, pk, p, 32, score);
    const std::vector<float>* src[7] = {&out.maps.mip, &out.maps.scaled_mip, &out.maps.psi, &out.maps.theta,
                                        &out.maps.phi, &out.maps.defocus, &out.maps.pixel_size};
    for (int k = 0; k < 7; k++) std::memcpy(maps_out + np * k, src[k]->data(), np * sizeof(float));
    for (int k = 0; k < n_peaks; k++) {
        const RefinedPeak& r = out.refined[k];
        const float v[16] = {r.x, r.y, r.psi, r.theta, r.phi, r.defocus, r.pixel_size, r.peak_height,
                             r.dx, r.dy, r.dpsi, r.dtheta, r.dphi, r.ddefocus, r.dpixel_size, r.dpeak_height};
        std::memcpy(per_peak + 16 * k, v, sizeof v);
    }
    return n_log;
}

