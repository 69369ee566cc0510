// refine.cpp -- see refine.hpp.
#include "refine.hpp"

#include <cfloat>
#include <cmath>
#include <complex>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <thread>

namespace tmhost {

namespace {

int round_half_away(float a) { return a > 0 ? (int)((double)a + 0.5) : (int)((double)a - 0.5); }

using cplx = std::complex<double>;

// sum_{k=a}^{b} exp(i theta k), theta = 2 pi num / den with num reduced mod den
cplx geometric(long num, long den, long a, long b) {
    if (b < a) return 0.0;
    num %= den;
    if (num < 0) num += den;
    const long count = b - a + 1;
    if (num == 0) return (double)count;
    const double th = 2.0 * M_PI * (double)num / (double)den;
    const cplx ea = std::polar(1.0, th * (double)a);
    const cplx r = std::polar(1.0, th);
    const cplx rn = std::polar(1.0, th * (double)count);
    return ea * (1.0 - rn) / (1.0 - r);
}

// key of a candidate for the per-peak memo of scores
struct CandKey {
    uint32_t v[6];
    bool operator==(const CandKey& o) const {
        for (int i = 0; i < 6; i++)
            if (v[i] != o.v[i]) return false;
        return true;
    }
};
struct CandHash {
    size_t operator()(const CandKey& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t x : k.v) h = (h ^ x) * 1099511628211ull;
        return (size_t)h;
    }
};
uint32_t bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
CandKey key_of(const RefineCandidate& c) {
    return CandKey{{bits(c.phi), bits(c.theta), bits(c.psi), bits(c.defocus1), bits(c.defocus2), bits(c.pixel_size_factor)}};
}

// A worker's private copies of the parameter maps (the reference's
// best_*_local images, CopyFrom'd once per thread), as overlays of the input
// maps keyed by the address in the FFTW-padded layout.
class LocalMaps {
public:
    LocalMaps(const RefineMaps& in, int pitch) : in_(in), pitch_(pitch) {}
    // 0 psi, 1 theta, 2 phi, 3 defocus, 4 pixel size
    float get(int which, long addr) const {
        auto it = over_[which].find(addr);
        if (it != over_[which].end()) return it->second;
        return base(which, addr);
    }
    void set(int which, long addr, float v) { over_[which][addr] = v; }
    float base(int which, long addr) const {
        const std::vector<float>* m[5] = {&in_.psi, &in_.theta, &in_.phi, &in_.defocus, &in_.pixel_size};
        return read(*m[which], addr);
    }
    float read(const std::vector<float>& m, long addr) const {
        // an address outside the image or in the padding columns reads 0
        if (addr < 0) return 0.0f;
        const long y = addr / pitch_, x = addr % pitch_;
        if (y >= in_.ny || x >= in_.nx) return 0.0f;
        return m[(size_t)y * in_.nx + x];
    }

private:
    const RefineMaps& in_;
    int pitch_;
    std::unordered_map<long, float> over_[5];
};

}  // namespace

std::vector<FoundPeak> refine_find_peaks(const RefineMaps& maps, float wanted_threshold, float min_peak_radius) {
    const int nx = maps.nx, ny = maps.ny;
    std::vector<float> z = maps.scaled_mip;
    std::vector<FoundPeak> out;
    const size_t cap = (size_t)nx * ny / 100;   // found_peaks array (:498)
    const int edge = 50;
    const int cx = nx / 2, cy = ny / 2;
    for (;;) {
        // FindPeakWithIntegerCoordinates(0, FLT_MAX, 50) (image.cpp:9961-10110)
        float best = -FLT_MAX;
        int bx = 0, by = 0;
        for (int j = edge; j <= ny - edge && j < ny; j++)
            for (int i = edge; i <= nx - edge && i < nx; i++) {
                const float v = z[(size_t)j * nx + i];
                if (v > best) {
                    best = v;
                    bx = i;
                    by = j;
                }
            }
        if (best < wanted_threshold || out.size() >= cap) break;
        FoundPeak p;
        p.x = (float)(bx - cx);
        p.y = (float)(by - cy);
        p.value = best;
        out.push_back(p);
        const float px = p.x + (float)cx, py = p.y + (float)cy;
        for (int j = 0; j < ny; j++) {
            const float sy = (float)std::pow((double)(j - py), 2);
            for (int i = 0; i < nx; i++) {
                const float sx = (float)std::pow((double)(i - px), 2);
                if (sx + sy <= min_peak_radius) z[(size_t)j * nx + i] = -FLT_MAX;
            }
        }
    }
    return out;
}

std::vector<float> window_particle(const Image2& im, int peak_x, int peak_y, int T) {
    const long nx = im.nx, ny = im.ny, n = nx * ny;
    // RealSpaceIntegerShift: buffer[shifted + p] = real[p], shifted reduced with remainderf
    long shifted = -(long)peak_x - nx * (long)peak_y;
    shifted = (long)remainderf((float)shifted, (float)n);
    if (shifted < 0) shifted += n;
    std::vector<float> w((size_t)T * T);
    for (int jj = 0; jj < T; jj++) {
        const long j = ny / 2 + (jj - T / 2);
        for (int ii = 0; ii < T; ii++) {
            const long i = nx / 2 + (ii - T / 2);
            float v = 0.0f;
            if (i >= 0 && i < nx && j >= 0 && j < ny) {
                long src = (j * nx + i) - shifted;
                src %= n;
                if (src < 0) src += n;
                v = im.v[(size_t)src];
            }
            w[(size_t)jj * T + ii] = v;
        }
    }
    return w;
}

void cosine_mask(std::vector<float>& img, int T, float wanted_mask_radius, float wanted_mask_edge) {
    const double kPiRef = 3.14159265359;   // PI (src/core/defines.h)
    float mask_radius = wanted_mask_radius - wanted_mask_edge * 0.5;
    if (mask_radius < 0.0) mask_radius = 0.0;
    const float mask_radius_plus_edge = mask_radius + wanted_mask_edge;
    const float r2 = powf(mask_radius, 2), re2 = powf(mask_radius_plus_edge, 2);
    const int c = T / 2;
    auto d2 = [&](int i, int j) { return powf((float)(i - c), 2) + powf((float)(j - c), 2) + powf(0.0f, 2); };
    double pixel_sum = 0.0;
    long n = 0;
    for (int j = 0; j < T; j++)
        for (int i = 0; i < T; i++) {
            const float d = d2(i, j);
            if (d >= r2 && d <= re2) {
                pixel_sum += img[(size_t)j * T + i];
                n++;
            }
        }
    if (n > 0) pixel_sum /= n;
    for (int j = 0; j < T; j++)
        for (int i = 0; i < T; i++) {
            const float d = d2(i, j);
            float& v = img[(size_t)j * T + i];
            if (d >= r2 && d <= re2) {
                const float dist = sqrtf(d);
                const float edge = (1.0 + cosf(kPiRef * (dist - mask_radius) / wanted_mask_edge)) / 2.0;
                v = v * edge + (1.0 - edge) * pixel_sum;
            } else if (d >= re2) {
                v = pixel_sum;
            }
        }
}

PixelSizeOperator pixel_size_operator(int nin, int nout, float factor, float tolerance) {
    PixelSizeOperator op;
    op.nin = nin;
    op.nout = nout;
    if (fabsf(factor - 1.0f) < tolerance) {
        op.identity = true;
        return op;
    }
    // sizes (image.cpp:8741-8775), square images
    const int old = nin, min_dim = nin;
    int pad, nw;
    if (tolerance < 1.0f / (min_dim * factor)) {
        const float inter = 1.0f / (tolerance * min_dim);
        pad = (int)(old * inter);
        if ((old % 2 == 0) != (pad % 2 == 0)) pad++;
        nw = (int)(pad / factor);
        if ((old % 2 == 0) != (nw % 2 == 0)) nw++;
    } else {
        pad = (int)(old * factor);
        if ((old % 2 == 0) != (pad % 2 == 0)) pad++;
        nw = old;
    }
    op.pad = pad;
    op.new_size = nw;
    op.has_pad_value = pad > old;
    if (nw == nout)
        throw std::runtime_error("pixel-size change whose resampled size equals the projection box is not supported");
    if (nw < nout) throw std::runtime_error("pixel-size change to a box smaller than the projection is not supported");
    const bool grow = nw > pad;
    const int P = pad, N = nw;
    const long kx_hi = grow ? P / 2 : N / 2;
    const long k_lo = grow ? -(P / 2) : -(N / 2), k_hi = grow ? P / 2 : N / 2 - 1;
    // input pixel i at P-grid position P/2 + i - nin/2; output t reads N-grid
    // position N/2 + t - nout/2; the phase of frequency k is
    // 2 pi k (q/N - p/P) = 2 pi k (q P - p N) / (N P)
    op.ar.resize((size_t)nout * nin);
    op.ai.resize((size_t)nout * nin);
    op.brt.resize((size_t)nin * nout);
    op.bit.resize((size_t)nin * nout);
    const double inv = 1.0 / ((double)P * (double)P);
    const long NP = (long)N * (long)P;
    for (int t = 0; t < nout; t++) {
        const long q = N / 2 + t - nout / 2;
        for (int i = 0; i < nin; i++) {
            const long pp = P / 2 + i - nin / 2;
            const long num = q * P - pp * N;
            // x axis: half-spectrum weights 1 at k = 0 (and k = N/2 when cropping), 2 elsewhere
            cplx ax = 2.0 * geometric(num, NP, 0, kx_hi) - 1.0;
            if (!grow) ax -= geometric(num, NP, N / 2, N / 2);
            const cplx ay = geometric(num, NP, k_lo, k_hi);
            op.ar[(size_t)t * nin + i] = (float)(ay.real() * inv);
            op.ai[(size_t)t * nin + i] = (float)(ay.imag() * inv);
            op.brt[(size_t)i * nout + t] = (float)ax.real();
            op.bit[(size_t)i * nout + t] = (float)ax.imag();
        }
    }
    return op;
}

// ------------------------------------------------------------------------------------------
void ScoreBatcher::worker_started() {
    std::lock_guard<std::mutex> lock(mu_);
    active_++;
}

void ScoreBatcher::worker_finished() {
    std::unique_lock<std::mutex> lock(mu_);
    active_--;
    if (!running_ && active_ > 0 && (int)pending_.size() == active_) run_locked(lock);
}

// Runs the pending requests as batches until fewer than the active workers
// are waiting; called with the lock held, returns with it held.
void ScoreBatcher::run_locked(std::unique_lock<std::mutex>& lock) {
    while (!running_ && !pending_.empty() && (int)pending_.size() >= active_) {
        running_ = true;
        std::vector<RefineCandidate> batch;
        batch.swap(pending_);
        std::vector<Request*> reqs;
        reqs.swap(requests_);
        lock.unlock();
        std::vector<RefineScore> out(batch.size());
        std::exception_ptr err;
        try {
            run_batch_(batch, out);
        } catch (...) {
            err = std::current_exception();
        }
        lock.lock();
        if (err && !error_) error_ = err;
        for (size_t k = 0; k < reqs.size(); k++) {
            reqs[k]->out = out[k];
            reqs[k]->done = true;
        }
        batches_++;
        scored_ += (long long)batch.size();
        running_ = false;
        cv_.notify_all();
    }
}

RefineScore ScoreBatcher::score(const RefineCandidate& c) {
    std::unique_lock<std::mutex> lock(mu_);
    if (error_) std::rethrow_exception(error_);
    Request req;
    pending_.push_back(c);
    requests_.push_back(&req);
    run_locked(lock);
    cv_.wait(lock, [&] { return req.done; });
    if (error_) std::rethrow_exception(error_);
    return req.out;
}

// ------------------------------------------------------------------------------------------
RefineOutputs refine_peaks(const RefineMaps& in, const std::vector<FoundPeak>& peaks, const RefineParams& prm, int T,
                           const ScoreFn& score, bool verbose, const std::function<void()>& worker_begin,
                           const std::function<void()>& worker_end) {
    const int nx = in.nx, ny = in.ny;
    const int pitch = nx + (nx % 2 == 0 ? 2 : 1);   // FFTW-padded row length of the maps
    const float pixel_size = prm.pixel_size;
    // derived steps (refine_template.cpp:314-320, 620-633)
    float defocus_search_range = prm.defocus_search_range;
    float defocus_refine_step = 2.0f * prm.defocus_search_step;
    float pixel_size_search_range = prm.pixel_size_search_range;
    float pixel_size_refine_step = 2.0f * prm.pixel_size_search_step;
    if (defocus_refine_step <= 0.0) {
        defocus_search_range = 0.0f;
        defocus_refine_step = 100.0f;
    }
    if (pixel_size_refine_step <= 0.0) {
        pixel_size_search_range = 0.0f;
        pixel_size_refine_step = 100.0f;
    }
    const float defocus_step = std::max(defocus_refine_step, 100.0f);
    const float angular_step = prm.angular_step, in_plane_angular_step = prm.in_plane_angular_step;
    const float box_scale = sqrtf((float)(T * T));   // sqrtf(projection_filter x * y)

    RefineOutputs out;
    out.peaks = peaks;
    out.refined.resize(peaks.size());
    out.maps.nx = nx;
    out.maps.ny = ny;
    out.maps.mip.assign((size_t)nx * ny, 0.0f);
    out.maps.scaled_mip.assign((size_t)nx * ny, 0.0f);
    out.maps.psi = in.psi;
    out.maps.theta = in.theta;
    out.maps.phi = in.phi;
    out.maps.defocus = in.defocus;
    out.maps.pixel_size = in.pixel_size;
    std::mutex out_mu;
    std::atomic<int> next{0};
    std::atomic<long long> n_eval{0}, n_distinct{0};
    auto in_read = [&](const std::vector<float>& m, long addr) -> float {
        if (addr < 0) return 0.0f;
        const long y = addr / pitch, x = addr % pitch;
        if (y >= ny || x >= nx) return 0.0f;
        return m[(size_t)y * nx + x];
    };

    auto worker = [&]() {
        LocalMaps local(in, pitch);
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= (int)peaks.size()) break;
            const FoundPeak& fp = peaks[k];
            std::unordered_map<CandKey, RefineScore, CandHash> memo;
            int evals = 0;
            auto eval = [&](const RefineCandidate& c) {
                evals++;
                const CandKey key = key_of(c);
                auto it = memo.find(key);
                if (it != memo.end()) return it->second;
                RefineScore s = score(c);
                memo.emplace(key, s);
                return s;
            };
            const int px = (int)(fp.x + (float)(nx / 2)), py = (int)(fp.y + (float)(ny / 2));
            const long current_address = (long)py * pitch + px;
            float current_phi = local.get(2, current_address);
            float current_theta = local.get(1, current_address);
            float current_psi = local.get(0, current_address);
            float current_defocus = local.get(3, current_address);
            float current_pixel_size = local.get(4, current_address);
            const float scaled_here = in_read(in.scaled_mip, current_address);
            const float mip_here = in_read(in.mip, current_address);
            float best_score = -FLT_MAX;
            RefineScore best_peak;
            long best_address = current_address;
            float offset_distance = 0.0f;
            const float score_adjustment = 1.0f;
            RefineCandidate c;
            c.particle = k;
            c.pixel_size_factor = 1.0f;
            auto set_defocus = [&](float df_offset_total_1, float df_offset_total_2) {
                c.defocus1 = df_offset_total_1;
                c.defocus2 = df_offset_total_2;
            };
            auto set_angles = [&](float phi, float theta, float psi) {
                c.phi = phi;
                c.theta = theta;
                c.psi = psi;
            };
            auto improve = [&](const RefineScore& s) {
                best_peak = s;
                best_score = s.value;
                const long address_offset = (long)pitch * round_half_away(s.y) + round_half_away(s.x);
                best_address = current_address + address_offset;
                offset_distance = sqrtf(powf(s.x, 2) + powf(s.y, 2));
            };
            set_angles(current_phi, current_theta, current_psi);
            set_defocus(prm.defocus1 + current_defocus, prm.defocus2 + current_defocus);
            const RefineScore start = eval(c);
            float starting_score = start.value * box_scale;
            starting_score = score_adjustment * scaled_here * starting_score / mip_here;
            if (verbose && prm.max_threads == 1)
                std::printf("\nRefining peak %i at x, y =  %6i, %6i\n", k + 1, px, py);

            // defocus scan (:806-839)
            if (defocus_search_range != 0.0f) {
                const int nd = round_half_away(float(defocus_search_range) / float(defocus_step));
                for (int defocus_is = -nd; defocus_is <= nd; defocus_is++) {
                    set_defocus(prm.defocus1 + current_defocus + defocus_is * defocus_step,
                                prm.defocus2 + current_defocus + defocus_is * defocus_step);
                    const RefineScore s = eval(c);
                    if (s.value > best_score) {
                        improve(s);
                        local.set(3, best_address, current_defocus + defocus_is * defocus_step);
                    }
                }
                current_defocus = local.get(3, best_address);
            }

            // the angle descent shared by both local searches (:869-926, 1019-1075)
            int phi_i = 0, theta_i = 0, psi_i = 0;
            auto angle_descent = [&](const std::function<void()>& on_improve) {
                for (int kk = 0; kk < 2; kk = -2 * kk + 1) {
                    float best_phi_score;
                    do {
                        best_phi_score = best_score;
                        phi_i += kk;
                        for (int jj = 0; jj < 2; jj = -2 * jj + 1) {
                            float best_theta_score;
                            do {
                                best_theta_score = best_score;
                                theta_i += jj;
                                for (int ii = 0; ii < 2; ii = -2 * ii + 1) {
                                    float best_psi_score;
                                    do {
                                        best_psi_score = best_score;
                                        psi_i += ii;
                                        set_angles(current_phi + phi_i * angular_step,
                                                   current_theta + theta_i * angular_step,
                                                   current_psi + psi_i * in_plane_angular_step);
                                        const RefineScore s = eval(c);
                                        if (s.value > best_score) {
                                            improve(s);
                                            local.set(0, best_address, current_psi + psi_i * in_plane_angular_step);
                                            local.set(1, best_address, current_theta + theta_i * angular_step);
                                            local.set(2, best_address, current_phi + phi_i * angular_step);
                                            on_improve();
                                        }
                                    } while (best_score > best_psi_score);
                                    psi_i -= ii;
                                }
                            } while (best_score > best_theta_score);
                            theta_i -= jj;
                        }
                    } while (best_score > best_phi_score);
                    phi_i -= kk;
                }
            };

            // local search with defocus (:842-931)
            int defocus_i = 0;
            const float mult_i_start = defocus_step / defocus_refine_step;
            for (float mult_i = mult_i_start; mult_i > 0.5f; mult_i /= 2.0f) {
                for (int ll = 0; ll < 2; ll = -2 * ll + 1) {
                    if ((ll != 0) && (defocus_refine_step == 0.0f)) break;
                    float best_defocus_score;
                    do {
                        best_defocus_score = best_score;
                        if (defocus_search_range != 0.0f) defocus_i += round_half_away(mult_i * ll);
                        set_defocus(prm.defocus1 + current_defocus + defocus_i * defocus_refine_step,
                                    prm.defocus2 + current_defocus + defocus_i * defocus_refine_step);
                        angle_descent([&] {
                            local.set(3, best_address, current_defocus + defocus_i * defocus_refine_step);
                            local.set(4, best_address, current_pixel_size);
                        });
                    } while (best_score > best_defocus_score);
                    if (defocus_search_range != 0.0f) defocus_i -= ll;
                }
            }

            // pixel size scan (:934-978)
            current_phi = local.get(2, best_address);
            current_theta = local.get(1, best_address);
            current_psi = local.get(0, best_address);
            current_defocus = local.get(3, best_address);
            current_pixel_size = local.get(4, best_address);
            phi_i = theta_i = psi_i = 0;
            int size_i = 0;
            set_defocus(prm.defocus1 + current_defocus, prm.defocus2 + current_defocus);
            set_angles(current_phi, current_theta, current_psi);
            if (pixel_size_search_range != 0.0f) {
                const int ns = round_half_away(float(pixel_size_search_range) / float(pixel_size_refine_step));
                for (int size_is = -ns; size_is <= ns; size_is++) {
                    c.pixel_size_factor =
                        (pixel_size + current_pixel_size + float(size_is) * pixel_size_refine_step) / pixel_size;
                    const RefineScore s = eval(c);
                    if (s.value > best_score) {
                        improve(s);
                        local.set(4, best_address, current_pixel_size + size_is * pixel_size_refine_step);
                    }
                }
                current_pixel_size = local.get(4, best_address);
            }

            // local search with pixel size (:980-1080)
            phi_i = theta_i = psi_i = 0;
            size_i = 0;
            for (float mult_i = 1.0f; mult_i > 0.5f; mult_i /= 2.0f) {
                for (int ll = 0; ll < 2; ll = -2 * ll + 1) {
                    if ((ll != 0) && (pixel_size_refine_step == 0.0f)) break;
                    float best_pixel_size_score;
                    do {
                        best_pixel_size_score = best_score;
                        if (pixel_size_search_range != 0.0f) size_i += round_half_away(mult_i * ll);
                        c.pixel_size_factor =
                            (pixel_size + current_pixel_size + float(size_i) * pixel_size_refine_step) / pixel_size;
                        angle_descent([&] {
                            local.set(3, best_address, current_defocus);
                            local.set(4, best_address, current_pixel_size + size_i * pixel_size_refine_step);
                        });
                    } while (best_score > best_pixel_size_score);
                    if (pixel_size_search_range != 0.0f) size_i -= ll;
                }
            }

            // results of the peak (:1086-1130)
            const float best_scaled = score_adjustment * scaled_here * best_score / mip_here * box_scale;
            const float best_mip = score_adjustment * best_score * box_scale;
            RefinedPeak r;
            r.x = fp.x + best_peak.x;
            r.y = fp.y + best_peak.y;
            r.psi = local.get(0, best_address);
            r.theta = local.get(1, best_address);
            r.phi = local.get(2, best_address);
            r.defocus = local.get(3, best_address);
            r.pixel_size = local.get(4, best_address);
            r.peak_height = best_scaled;
            r.dx = best_peak.x * pixel_size;
            r.dy = best_peak.y * pixel_size;
            r.dpsi = r.psi - in_read(in.psi, current_address);
            r.dtheta = r.theta - in_read(in.theta, current_address);
            r.dphi = r.phi - in_read(in.phi, current_address);
            r.ddefocus = r.defocus - in_read(in.defocus, current_address);
            r.dpixel_size = r.pixel_size - in_read(in.pixel_size, current_address);
            r.dpeak_height = best_scaled - starting_score;
            r.offset_distance = offset_distance;
            r.best_address = best_address;
            r.evaluations = evals;
            r.distinct_evaluations = (int)memo.size();
            n_eval += evals;
            n_distinct += (long long)memo.size();
            if (verbose)
                std::printf("Peak %4i: dx, dy, dpsi, dtheta, dphi, ddefocus, dpixel size = %12.6f, %12.6f, %12.6f, "
                            "%12.6f, %12.6f, %12.6f, %12.6f | peak in = %10.6f, peak out = %10.6f\n",
                            k + 1, r.dx, r.dy, r.dpsi, r.dtheta, r.dphi, r.ddefocus, r.dpixel_size, starting_score,
                            best_scaled);
            if (offset_distance * pixel_size > prm.xy_change_threshold)
                std::printf("Warning: Peak %4i moved by %g A\n", k + 1, offset_distance * pixel_size);
            {
                std::lock_guard<std::mutex> lock(out_mu);
                out.refined[k] = r;
                const long y = best_address / pitch, x = best_address % pitch;
                const bool on_image = best_address >= 0 && y < ny && x < nx;
                if (on_image && (offset_distance * pixel_size <= prm.xy_change_threshold || !prm.exclude_above_xy_threshold)) {
                    const size_t o = (size_t)y * nx + x;
                    out.maps.scaled_mip[o] = best_scaled;
                    out.maps.mip[o] = best_mip;
                    out.maps.psi[o] = r.psi;
                    out.maps.theta[o] = r.theta;
                    out.maps.phi[o] = r.phi;
                    out.maps.defocus[o] = r.defocus;
                    out.maps.pixel_size[o] = r.pixel_size;
                }
            }
        }
    };

    int workers = prm.max_threads < 1 ? 1 : prm.max_threads;
    if (workers > (int)peaks.size()) workers = (int)peaks.size();
    std::vector<std::thread> pool;
    std::exception_ptr first_error;
    std::mutex err_mu;
    if (worker_begin)
        for (int w = 0; w < workers; w++) worker_begin();
    for (int w = 0; w < workers; w++)
        pool.emplace_back([&] {
            try {
                worker();
            } catch (...) {
                std::lock_guard<std::mutex> lock(err_mu);
                if (!first_error) first_error = std::current_exception();
                next.store((int)peaks.size());
            }
            if (worker_end) worker_end();
        });
    for (auto& t : pool) t.join();
    if (first_error) std::rethrow_exception(first_error);
    out.evaluations = n_eval;
    out.distinct_evaluations = n_distinct;
    return out;
}

}  // namespace tmhost
