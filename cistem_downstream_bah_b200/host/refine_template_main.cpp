// refine_template_main.cpp -- the refine_template program
// (src/programs/refine_template/refine_template.cpp) on the B200 scoring core.
//
//   refine_template                interactive prompts, as DoInteractiveUserInput
//                                  (refine_template.cpp:93-258), read from stdin
//   refine_template ARG0 ... ARG50  the 51 job arguments in the order
//                                  DoCalculation reads them (:296-346)
//
// The search maps of one result (argument 46 picks the slice) are read, the
// micrograph whitened (:612-630), the peaks of the scaled MIP picked
// (:503-553), and each peak refined by the reference's coordinate descent
// (refine.cpp) with TemplateScore evaluated in batches on the GPU
// (tm_refine_score); the refined MIP, scaled MIP and parameter maps are written
// to arguments 29-35 with the pixel size set (:1140-1146).  max_threads
// (argument 47) is the number of peaks refined at once -- the reference's
// OpenMP threads -- and so the width of the GPU batches.  The GUI result
// (arguments 48-50) is not produced.
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "host_fft.hpp"
#include "job_args.hpp"
#include "mrc.hpp"
#include "prep.hpp"
#include "refine.hpp"
#include "tm_b200.h"
#include "user_input.hpp"

using namespace tmhost;

namespace {

struct RefineArgs {
    std::string input_search_images, input_reconstruction;   // 0, 1
    RefineParams p;                                          // 2-21, 36-39, 47
    float low_resolution_limit = 300, high_resolution_limit = 8, angular_range = 2;
    int best_parameters_to_keep = 20;
    bool ctf_refinement = false;
    std::string in_mip, in_scaled_mip, in_psi, in_theta, in_phi, in_defocus, in_pixel_size;   // 22-28
    std::string out_psi, out_theta, out_phi, out_defocus, out_pixel_size, out_mip, out_scaled_mip;   // 29-35
    std::string symmetry = "C1";                             // 40
    int first_search_position = -1, last_search_position = -1, image_number_for_gui = 0;
    int number_of_jobs_per_image_in_gui = 0, result_number = 1;   // 42-46
    std::string directory_for_results, filename_for_gui_result_image;   // 48, 50
    float threshold_for_result_plotting = 0;                 // 49
};

bool parse(int argc, char** argv, RefineArgs& a) {
    if (argc != 52) return false;
    auto S = [&](int i) { return std::string(argv[1 + i]); };
    auto F = [&](int i) { return (float)std::atof(argv[1 + i]); };
    auto I = [&](int i) { return std::atoi(argv[1 + i]); };
    a.input_search_images = S(0);
    a.input_reconstruction = S(1);
    a.p.pixel_size = F(2);
    a.p.voltage_kV = F(3);
    a.p.spherical_aberration_mm = F(4);
    a.p.amplitude_contrast = F(5);
    a.p.defocus1 = F(6);
    a.p.defocus2 = F(7);
    a.p.defocus_angle = F(8);
    a.low_resolution_limit = F(9);
    a.high_resolution_limit = F(10);
    a.angular_range = F(11);
    a.p.angular_step = F(12);
    a.best_parameters_to_keep = I(13);
    a.p.defocus_search_range = F(14);
    a.p.defocus_search_step = F(15);
    a.p.pixel_size_search_range = F(16);
    a.p.pixel_size_search_step = F(17);
    a.p.padding = F(18);
    a.ctf_refinement = parse_bool(S(19));
    a.p.mask_radius = F(20);
    a.p.phase_shift = F(21);
    a.in_mip = S(22);
    a.in_scaled_mip = S(23);
    a.in_psi = S(24);
    a.in_theta = S(25);
    a.in_phi = S(26);
    a.in_defocus = S(27);
    a.in_pixel_size = S(28);
    a.out_psi = S(29);
    a.out_theta = S(30);
    a.out_phi = S(31);
    a.out_defocus = S(32);
    a.out_pixel_size = S(33);
    a.out_mip = S(34);
    a.out_scaled_mip = S(35);
    a.p.wanted_threshold = F(36);
    a.p.min_peak_radius = F(37);
    a.p.xy_change_threshold = F(38);
    a.p.exclude_above_xy_threshold = parse_bool(S(39));
    a.symmetry = S(40);
    a.p.in_plane_angular_step = F(41);
    a.first_search_position = I(42);
    a.last_search_position = I(43);
    a.image_number_for_gui = I(44);
    a.number_of_jobs_per_image_in_gui = I(45);
    a.result_number = I(46);
    a.p.max_threads = I(47);
    a.directory_for_results = S(48);
    a.threshold_for_result_plotting = F(49);
    a.filename_for_gui_result_image = S(50);
    return true;
}

// DoInteractiveUserInput (refine_template.cpp:140-258): the prompts, then the
// job arguments as its ManualSetArguments fills them
RefineArgs interactive() {
    UserInput in;
    RefineArgs a;
    a.input_search_images = in.filename("Input images to be searched", "The input image stack, containing the images that should be searched", "image_stack.mrc", true);
    a.input_reconstruction = in.filename("Input template reconstruction", "The 3D reconstruction from which projections are calculated", "reconstruction.mrc", true);
    a.in_mip = in.filename("Input MIP file", "The file with the maximum intensity projection image", "mip.mrc", false);
    a.in_scaled_mip = in.filename("Input scaled MIP file", "The file with the scaled MIP (peak search done on this image)", "scaled_mip.mrc", false);
    a.in_psi = in.filename("Input psi file", "The file with the best psi image", "psi.mrc", true);
    a.in_theta = in.filename("Input theta file", "The file with the best psi image", "theta.mrc", true);
    a.in_phi = in.filename("Input phi file", "The file with the best psi image", "phi.mrc", true);
    a.in_defocus = in.filename("Input defocus file", "The file with the best defocus image", "defocus.mrc", true);
    a.in_pixel_size = in.filename("Input pixel size file", "The file with the best pixel size image", "pixel_size.mrc", true);
    a.out_mip = in.filename("Output MIP file", "The file for saving the maximum intensity projection image", "out_mip.mrc", false);
    a.out_scaled_mip = in.filename("Output Scaled MIP file", "The file for saving the maximum intensity projection image divided by correlation variance", "out_scaled_mip.mrc", false);
    a.out_psi = in.filename("Output psi file", "The file for saving the best psi image", "out_psi.mrc", false);
    a.out_theta = in.filename("Output theta file", "The file for saving the best psi image", "out_theta.mrc", false);
    a.out_phi = in.filename("Output phi file", "The file for saving the best psi image", "out_phi.mrc", false);
    a.out_defocus = in.filename("Output defocus file", "The file for saving the best defocus image", "out_defocus.mrc", false);
    a.out_pixel_size = in.filename("Output pixel size file", "The file for saving the best pixel size image", "out_pixel_size.mrc", false);
    RefineParams& p = a.p;
    p.wanted_threshold = in.number("Peak threshold", "Peaks over this size will be taken", "7.5", 0.0f);
    p.min_peak_radius = in.number("Min peak radius (px.)", "Essentially the minimum closeness for peaks", "10.0", 0.0f);
    p.pixel_size = in.number("Pixel size of images (A)", "Pixel size of input images in Angstroms", "1.0", 0.0f);
    p.voltage_kV = in.number("Beam energy (keV)", "The energy of the electron beam used to image the sample in kilo electron volts", "300.0", 0.0f);
    p.spherical_aberration_mm = in.number("Spherical aberration (mm)", "Spherical aberration of the objective lens in millimeters", "2.7");
    p.amplitude_contrast = in.number("Amplitude contrast", "Assumed amplitude contrast", "0.07", 0.0f, 1.0f);
    p.defocus1 = in.number("Defocus1 (angstroms)", "Defocus1 for the input image", "10000", 0.0f);
    p.defocus2 = in.number("Defocus2 (angstroms)", "Defocus2 for the input image", "10000", 0.0f);
    p.defocus_angle = in.number("Defocus angle (degrees)", "Defocus Angle for the input image", "0.0");
    p.phase_shift = in.number("Phase shift (degrees)", "Additional phase shift in degrees", "0.0");
    p.angular_step = in.number("Out of plane angular step", "Angular step size for global grid search", "0.2", 0.01f);
    p.in_plane_angular_step = in.number("In plane angular step", "Angular step size for in-plane rotations during the search", "0.1", 0.01f);
    p.defocus_search_range = in.number("Defocus search range (A) (0.0 = no search)", "Search range (-value ... + value) around current defocus", "200.0", 0.0f);
    p.defocus_search_step = in.number("Desired defocus accuracy (A)", "Accuracy to be achieved in defocus search", "10.0", 0.0f);
    p.pixel_size_search_range = in.number("Pixel size search range (A) (0.0 = no search)", "Search range (-value ... + value) around current pixel size", "0.1", 0.0f);
    p.pixel_size_search_step = in.number("Desired pixel size accuracy (A)", "Accuracy to be achieved in pixel size search", "0.01", 0.01f);
    p.padding = in.number("Padding factor", "Factor determining how much the input volume is padded to improve projections", "2.0", 1.0f);
    p.mask_radius = in.number("Mask radius (A) (0.0 = no mask)", "Radius of a circular mask to be applied to the input particles during refinement", "0.0", 0.0f);
    p.xy_change_threshold = in.number("Moved peak warning (A)", "Threshold for displaying warning of peak location changes during refinement", "10.0", 0.0f);
    p.exclude_above_xy_threshold = in.yes_no("Exclude moving peaks", "Should the peaks that move more than the threshold be excluded from the output MIPs?", "No");
    a.result_number = (int)in.number("Result number to refine", "If input files contain results from several searches, which one should be refined?", "1", 1.0f);
    p.max_threads = (int)in.number("Max. threads to use for calculation", "When threading, what is the max threads to run", "1", 1.0f);
    // the values ManualSetArguments passes besides the answers (:189-258)
    a.low_resolution_limit = 300.0f;
    a.high_resolution_limit = 8.0f;
    a.angular_range = 2.0f;
    a.best_parameters_to_keep = 20;
    a.ctf_refinement = false;
    a.symmetry = "C1";
    a.first_search_position = -1;
    a.last_search_position = -1;
    a.image_number_for_gui = 0;
    a.number_of_jobs_per_image_in_gui = 0;
    a.directory_for_results = "/dev/null";
    a.threshold_for_result_plotting = 0.0f;
    a.filename_for_gui_result_image = "";
    return a;
}

std::vector<float> read_slice(const std::string& path, int slice, int* nx, int* ny) {
    MrcData m;
    std::string err;
    if (!read_mrc(path, m, err, slice, slice)) throw std::runtime_error(err);
    if (m.nz < 1) throw std::runtime_error(path + " does not contain the selected result");
    if (nx) *nx = m.nx;
    if (ny) *ny = m.ny;
    return m.data;
}

// TemplateScore on the GPU with the filters and pixel-size operators cached on
// the device by their defocus pair and factor.
class RefineGpu {
public:
    RefineGpu(int device, int T, int TP, const std::vector<std::complex<float>>& tspec, int max_batch, int n_particles,
              std::vector<double> curve, const RefineParams& p)
        : T_(T), TP_(TP), curve_(std::move(curve)), p_(p) {
        max_filters_ = std::max(2 * max_batch, 64);
        max_ops_ = std::min(std::max(max_batch, 8), 64);
        check(tm_refine_create(device, T, TP, reinterpret_cast<const float*>(tspec.data()), max_batch,
                               std::max(n_particles, 1), max_filters_, max_ops_, &ctx_),
              "tm_refine_create");
    }
    ~RefineGpu() {
        if (ctx_) tm_refine_destroy(ctx_);
    }

    void set_particle(int slot, std::vector<float> window) {
        if (p_.mask_radius > 0.0f) cosine_mask(window, T_, p_.mask_radius / p_.pixel_size, 20.0f / p_.pixel_size);
        const int hc = T_ / 2 + 1;
        std::vector<double> w(window.begin(), window.end());
        std::vector<std::complex<double>> spec((size_t)T_ * hc);
        rfft2(T_, T_, w.data(), spec.data());
        const double inv = 1.0 / ((double)T_ * T_);
        for (auto& c : spec) c *= inv;
        swap_quadrants(T_, T_, 1, spec.data());
        std::vector<std::complex<float>> f(spec.size());
        for (size_t i = 0; i < spec.size(); i++) f[i] = std::complex<float>(spec[i]);
        check(tm_refine_set_particle(ctx_, slot, reinterpret_cast<const float*>(f.data())), "tm_refine_set_particle");
    }

    void score(const std::vector<RefineCandidate>& cands, std::vector<RefineScore>& out) {
        out.resize(cands.size());
        size_t start = 0;
        while (start < cands.size()) {
            // a chunk whose filters and operators fit the device caches
            std::vector<float> euler;
            std::vector<int> part, filt, op;
            size_t k = start;
            for (; k < cands.size(); k++) {
                const RefineCandidate& c = cands[k];
                int fs = filter_slot(c.defocus1, c.defocus2, k > start);
                if (fs < 0) break;
                int os = op_slot(c.pixel_size_factor, k > start);
                if (os < -1) break;
                euler.insert(euler.end(), {c.phi, c.theta, c.psi});
                part.push_back(c.particle);
                filt.push_back(fs);
                op.push_back(os);
            }
            std::vector<float> res(3 * part.size());
            check(tm_refine_score(ctx_, (int)part.size(), euler.data(), part.data(), filt.data(), op.data(), res.data()),
                  "tm_refine_score");
            for (size_t j = 0; j < part.size(); j++) out[start + j] = RefineScore{res[3 * j], res[3 * j + 1], res[3 * j + 2]};
            start = k;
        }
    }

    long long filters_built = 0, operators_built = 0;

private:
    void check(int rc, const char* what) {
        if (rc != TM_OK)
            throw std::runtime_error(std::string(what) + " failed: " + (ctx_ ? tm_refine_last_error(ctx_) : "no context"));
    }
    static uint64_t key2(float a, float b) {
        uint32_t x, y;
        std::memcpy(&x, &a, 4);
        std::memcpy(&y, &b, 4);
        return ((uint64_t)x << 32) | y;
    }
    // slot of the filter, building it if needed; -1 when the cache is full and
    // `in_chunk` (the caller then scores what it has first)
    int filter_slot(float df1, float df2, bool in_chunk) {
        const uint64_t key = key2(df1, df2);
        auto it = filters_.find(key);
        if (it != filters_.end()) return it->second;
        if ((int)filters_.size() >= max_filters_) {
            if (in_chunk) return -1;
            filters_.clear();
        }
        const int slot = (int)filters_.size();
        CtfParams ctf{p_.voltage_kV, p_.spherical_aberration_mm, p_.amplitude_contrast, df1, df2, p_.defocus_angle,
                      p_.pixel_size, p_.phase_shift};
        const std::vector<float> f = projection_filter(T_, curve_, ctf, 0.0f);
        check(tm_refine_set_filter(ctx_, slot, f.data()), "tm_refine_set_filter");
        filters_[key] = slot;
        filters_built++;
        return slot;
    }
    // -1 for a factor within the tolerance, -2 when the cache is full in a chunk
    int op_slot(float factor, bool in_chunk) {
        if (fabsf(factor - 1.0f) < 0.001f) return -1;
        uint32_t key;
        std::memcpy(&key, &factor, 4);
        auto it = ops_.find(key);
        if (it != ops_.end()) return it->second;
        if ((int)ops_.size() >= max_ops_) {
            if (in_chunk) return -2;
            ops_.clear();
        }
        const int slot = (int)ops_.size();
        const PixelSizeOperator o = pixel_size_operator(TP_, T_, factor);
        check(tm_refine_set_operator(ctx_, slot, o.ar.data(), o.ai.data(), o.brt.data(), o.bit.data(),
                                     o.has_pad_value ? 1 : 0),
              "tm_refine_set_operator");
        ops_[key] = slot;
        operators_built++;
        return slot;
    }

    int T_, TP_;
    std::vector<double> curve_;
    RefineParams p_;
    tm_refine_ctx* ctx_ = nullptr;
    int max_filters_ = 0, max_ops_ = 0;
    std::map<uint64_t, int> filters_;
    std::map<uint32_t, int> ops_;
};

int run(const RefineArgs& a) {
    const auto t0 = std::chrono::steady_clock::now();
    RefineParams prm = a.p;
    int nx = 0, ny = 0;
    std::vector<float> image = read_slice(a.input_search_images, a.result_number, &nx, &ny);
    RefineMaps maps;
    maps.nx = nx;
    maps.ny = ny;
    struct In {
        const std::string* path;
        std::vector<float>* dst;
    } ins[] = {{&a.in_mip, &maps.mip},         {&a.in_scaled_mip, &maps.scaled_mip}, {&a.in_psi, &maps.psi},
               {&a.in_theta, &maps.theta},     {&a.in_phi, &maps.phi},               {&a.in_defocus, &maps.defocus},
               {&a.in_pixel_size, &maps.pixel_size}};
    for (const In& in : ins) {
        int mx = 0, my = 0;
        *in.dst = read_slice(*in.path, a.result_number, &mx, &my);
        if (mx != nx || my != ny) throw std::runtime_error(*in.path + ": size differs from the micrograph");
    }
    MrcData rec;
    std::string err;
    if (!read_mrc(a.input_reconstruction, rec, err)) throw std::runtime_error(err);
    const int T = rec.nx;
    if (rec.ny != T || rec.nz != T) throw std::runtime_error("the template reconstruction must be a cube");
    const int TP = (int)(T * prm.padding);
    // mask radius at most (T/2 - 1) pixels (:603-604)
    const float max_mask = (float(T) / 2.0f - 1.0f) * prm.pixel_size;
    if (prm.mask_radius > max_mask) prm.mask_radius = max_mask;

    // whitening (:612-630): as match_template's without the quadrant swap, then back to real space
    Image2 mic;
    mic.nx = nx;
    mic.ny = ny;
    mic.v = image;
    Whitened w = whiten(mic, false);
    std::vector<std::complex<double>> spec(w.spectrum.begin(), w.spectrum.end());
    std::vector<double> real((size_t)nx * ny);
    irfft2(nx, ny, spec.data(), real.data());
    Image2 whitened;
    whitened.nx = nx;
    whitened.ny = ny;
    whitened.v.assign(real.begin(), real.end());

    // peaks (:503-553)
    const std::vector<FoundPeak> peaks = refine_find_peaks(maps, prm.wanted_threshold, prm.min_peak_radius);
    std::printf("\n");
    for (size_t k = 0; k < peaks.size(); k++) {
        const long addr = (long)(peaks[k].y + ny / 2) * nx + (long)(peaks[k].x + nx / 2);
        std::printf("Peak %4zu at x, y, psi, theta, phi, defocus, pixel size =  %12.6f, %12.6f, %12.6f, %12.6f, %12.6f, "
                    "%12.6f, %12.6f : %10.6f\n",
                    k + 1, (peaks[k].x + nx / 2) * prm.pixel_size, (peaks[k].y + ny / 2) * prm.pixel_size,
                    maps.psi[addr], maps.theta[addr], maps.phi[addr], maps.defocus[addr], maps.pixel_size[addr],
                    peaks[k].value);
    }
    std::printf("\nRefining %zu positions in the MIP.\n\nPerforming refinement...\n\n", peaks.size());
    std::fflush(stdout);

    RefineOutputs out;
    long long batches = 0, scored = 0;
    if (!peaks.empty()) {
        int workers = prm.max_threads < 1 ? 1 : prm.max_threads;
        if (workers > (int)peaks.size()) workers = (int)peaks.size();
        RefineGpu gpu(0, T, TP, padded_template_spectrum(rec.data, T, TP), workers, (int)peaks.size(), w.curve, prm);
        for (size_t k = 0; k < peaks.size(); k++)
            gpu.set_particle((int)k, window_particle(whitened, (int)peaks[k].x, (int)peaks[k].y, T));
        ScoreBatcher batcher([&](const std::vector<RefineCandidate>& c, std::vector<RefineScore>& s) { gpu.score(c, s); });
        out = refine_peaks(maps, peaks, prm, T, [&](const RefineCandidate& c) { return batcher.score(c); }, true,
                           [&] { batcher.worker_started(); }, [&] { batcher.worker_finished(); });
        batches = batcher.batches();
        scored = batcher.scored();
    } else {
        out.maps = maps;
        std::fill(out.maps.mip.begin(), out.maps.mip.end(), 0.0f);
        std::fill(out.maps.scaled_mip.begin(), out.maps.scaled_mip.end(), 0.0f);
    }

    // outputs (:1140-1146)
    const std::pair<const std::string*, const std::vector<float>*> outs[] = {
        {&a.out_mip, &out.maps.mip},     {&a.out_scaled_mip, &out.maps.scaled_mip}, {&a.out_psi, &out.maps.psi},
        {&a.out_theta, &out.maps.theta}, {&a.out_phi, &out.maps.phi},               {&a.out_defocus, &out.maps.defocus},
        {&a.out_pixel_size, &out.maps.pixel_size}};
    for (const auto& o : outs) {
        Image2 im;
        im.nx = nx;
        im.ny = ny;
        im.v = *o.second;
        write_or_die(*o.first, im, prm.pixel_size);
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("\n%zu peaks refined: %lld TemplateScore calls of the reference's loop, %lld distinct candidates "
                "scored on the GPU in %lld batches; %.3f s\n",
                peaks.size(), out.evaluations, scored, batches, secs);
    std::printf("\nRefine Template: Normal termination\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    RefineArgs a;
    if (argc == 1) {
        a = interactive();
    } else if (!parse(argc, argv, a)) {
        std::fprintf(stderr,
                     "usage: %s                  (interactive)\n"
                     "       %s ARG0 ... ARG50   (the 51 refine_template job arguments)\n",
                     argv[0], argv[0]);
        return 2;
    }
    try {
        return run(a);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "\nError: %s\n", e.what());
        return 1;
    }
}
