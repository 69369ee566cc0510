// match_template_main.cpp -- the match_template program on the B200 search
// core: the reference's MatchTemplateApp (src/programs/match_template/
// match_template.cpp) without wxWidgets, for a local run.
//
// Invocation:
//   match_template                 interactive prompts, as DoInteractiveUserInput
//                                  (match_template.cpp:184-279), read from stdin
//   match_template ARG0 ... ARG41  the 42 job arguments in the order that
//                                  DoCalculation reads them (:346-387)
// The interactive form fills the job arguments exactly as ManualSetArguments
// does (:237-278), so the prompts for the correlation average and variance
// files land in argument slots 36 and 28, which DoCalculation reads as the
// variance and average files: the two outputs are swapped in interactive use,
// as in the reference.  The search always runs on the GPU; use_gpu (40) and
// max_threads (41) are accepted and reported.
//
//   match_template ARG0 ... ARG41 RESULT_ARRAY
//                                  a worker job of a distributed run: the
//                                  search covers search positions ARG32-ARG33
//                                  (not the whole grid) and, instead of the
//                                  output files, writes the flat result array
//                                  the reference's worker sends to its master
//                                  (:1373-1530) to RESULT_ARRAY; the program
//                                  match_template_merge plays the master.
// The reference's socket transport (<address> <port> <job code> <threads>) is
// replaced by these files.
#include <unistd.h>

#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>

#include "job_args.hpp"
#include "user_input.hpp"
#include "mrc.hpp"
#include "result_array.hpp"
#include "peaks.hpp"
#include "prep.hpp"
#include "template_matching_core.hpp"

using namespace tmhost;

namespace {

constexpr float kHistogramMin = -12.5f;      // match_template.cpp:24-26
constexpr float kHistogramMax = 22.5f;
constexpr int kHistogramBins = 512;
constexpr double kPi = 3.14159265359;
constexpr float kPif = 3.14159265359f;

float rad_2_deg(float r) { return (float)((double)r / ((double)kPif / 180.)); }

JobArgs interactive() {
    UserInput in;
    std::string input_search_images = in.filename("Input images to be searched", "The input image stack, containing the images that should be searched", "image_stack.mrc", true);
    std::string input_reconstruction = in.filename("Input template reconstruction", "The 3D reconstruction from which projections are calculated", "reconstruction.mrc", true);
    std::string mip = in.filename("Output MIP file", "The file for saving the maximum intensity projection image", "mip.mrc", false);
    std::string scaled = in.filename("Output Scaled MIP file", "The file for saving the maximum intensity projection image divided by correlation variance", "mip_scaled.mrc", false);
    std::string psi = in.filename("Output psi file", "The file for saving the best psi image", "psi.mrc", false);
    std::string theta = in.filename("Output theta file", "The file for saving the best psi image", "theta.mrc", false);
    std::string phi = in.filename("Output phi file", "The file for saving the best psi image", "phi.mrc", false);
    std::string defocus = in.filename("Output defocus file", "The file for saving the best defocus image", "defocus.mrc", false);
    std::string pixel = in.filename("Output pixel size file", "The file for saving the best pixel size image", "pixel_size.mrc", false);
    std::string avg = in.filename("Correlation average value", "The file for saving the average value of all correlation images", "corr_average.mrc", false);
    std::string var = in.filename("Correlation variance output file", "The file for saving the variance of all correlation images", "corr_variance.mrc", false);
    std::string hist = in.filename("Output histogram of correlation values", "histogram of all correlation values", "histogram.txt", false);
    JobArgs a;
    a.pixel_size = in.number("Pixel size of images (A)", "Pixel size of input images in Angstroms", "1.0", 0.0f);
    a.voltage_kV = in.number("Beam energy (keV)", "The energy of the electron beam used to image the sample in kilo electron volts", "300.0", 0.0f);
    a.spherical_aberration_mm = in.number("Spherical aberration (mm)", "Spherical aberration of the objective lens in millimeters", "2.7");
    a.amplitude_contrast = in.number("Amplitude contrast", "Assumed amplitude contrast", "0.07", 0.0f, 1.0f);
    a.defocus1 = in.number("Defocus1 (angstroms)", "Defocus1 for the input image", "10000", 0.0f);
    a.defocus2 = in.number("Defocus2 (angstroms)", "Defocus2 for the input image", "10000", 0.0f);
    a.defocus_angle = in.number("Defocus Angle (degrees)", "Defocus Angle for the input image", "0.0");
    a.phase_shift = in.number("Phase Shift (degrees)", "Additional phase shift in degrees", "0.0");
    a.high_resolution_limit_search = in.number("High resolution limit (A)", "High resolution limit of the data used for alignment in Angstroms", "8.0", 0.0f);
    a.angular_step = in.number("Out of plane angular step (0.0 = set automatically)", "Angular step size for global grid search", "0.0", 0.0f);
    a.in_plane_angular_step = in.number("In plane angular step (0.0 = set automatically)", "Angular step size for in-plane rotations during the search", "0.0", 0.0f);
    a.defocus_search_range = in.number("Defocus search range (A)", "Search range (-value ... + value) around current defocus", "500.0", 0.0f);
    a.defocus_step = in.number("Defocus step (A) (0.0 = no search)", "Step size used in the defocus search", "50.0", 0.0f);
    a.pixel_size_search_range = in.number("Pixel size search range (A)", "Search range (-value ... + value) around current pixel size", "0.1", 0.0f);
    a.pixel_size_step = in.number("Pixel size step (A) (0.0 = no search)", "Step size used in the pixel size search", "0.01", 0.0f);
    a.padding = in.number("Padding factor", "Factor determining how much the input volume is padded to improve projections", "1.0", 1.0f, 2.0f);
    a.particle_radius_angstroms = in.number("Mask radius for global search (A) (0.0 = max)", "Radius of a circular mask to be applied to the input images during global search", "0.0", 0.0f);
    a.my_symmetry = in.symmetry("Template symmetry", "The symmetry of the template reconstruction", "C1");
    a.use_gpu = in.yes_no("Use GPU", "Offload expensive calcs to GPU", "No");
    a.max_threads = (int)in.number("Max. threads to use for calculation", "when threading, what is the max threads to run", "1", 1.0f);
    // ManualSetArguments (match_template.cpp:237-278): slot 28 receives the
    // variance file and slot 36 the average file
    a.input_search_images = input_search_images;
    a.input_reconstruction = input_reconstruction;
    a.mip_output_file = mip;
    a.best_psi_output_file = psi;
    a.best_theta_output_file = theta;
    a.best_phi_output_file = phi;
    a.best_defocus_output_file = defocus;
    a.best_pixel_size_output_file = pixel;
    a.scaled_mip_output_file = scaled;
    a.correlation_avg_output_file = var;
    a.correlation_std_output_file = avg;
    a.output_histogram_file = hist;
    a.low_resolution_limit = 300.0f;
    a.best_parameters_to_keep = 20;
    a.ctf_refinement = false;
    a.first_search_position = -1;
    a.last_search_position = -1;
    a.directory_for_results = "/dev/null";
    a.result_output_filename = "/dev/null";
    a.min_peak_radius = 10.0f;
    return a;
}

Image2 as_image2(const std::vector<float>& v, int nx, int ny) {
    Image2 im;
    im.nx = nx;
    im.ny = ny;
    im.v = v;
    return im;
}

int run(const JobArgs& a) {
    const auto t_start = std::chrono::steady_clock::now();
    if (!a.use_gpu) std::printf("Note: this build always searches on the GPU (use_gpu = no is ignored).\n");
    if (a.padding != 1.0f)
        throw CoreError(TM_ERR_UNSUPPORTED, "template padding other than 1.0 is not supported by the GPU search "
                                            "(the reference GPU path ignores it as well)");
    std::string err;
    MrcData mic, rec;
    if (!read_mrc(a.input_search_images, mic, err, 1, 1)) throw CoreError(TM_ERR_INVALID, err);
    if (!read_mrc(a.input_reconstruction, rec, err)) throw CoreError(TM_ERR_INVALID, err);
    const int T = rec.nx;
    if (rec.ny != T || rec.nz != T) throw CoreError(TM_ERR_INVALID, "the template reconstruction must be a cube");

    // micrograph size (match_template.cpp:520-596)
    Image2 input;
    input.nx = mic.nx;
    input.ny = mic.ny;
    input.v = mic.data;
    const long original_x = input.nx, original_y = input.ny;
    const int fx = factorize_dimension(input.nx, rec.nx);
    const int fy = factorize_dimension(input.ny, rec.ny);
    std::printf("old x, y; new x, y = %i %i %i %i\n", input.nx, input.ny, fx, fy);
    input = clip_into(input, fx, fy, edge_mean(input));
    bool rotated = false;
    if (!is_power_of_two(fx) && is_power_of_two(fy)) {
        rotated = true;
        input = rotate90(input, true);
    }
    const int X = input.nx, Y = input.ny;
    const size_t npix = (size_t)X * Y;
    const double sqrt_input_pixels = std::sqrt((double)(X * Y));
    const float histogram_step = (kHistogramMax - kHistogramMin) / float(kHistogramBins);
    const double histogram_min_scaled = kHistogramMin / sqrt_input_pixels;
    const double histogram_step_scaled = histogram_step / sqrt_input_pixels;

    // angular sampling (:654-697)
    const float mask_radius_search = a.particle_radius_angstroms < 1.0f ? 200.0f : a.particle_radius_angstroms;
    float angular_step = a.angular_step;
    if (angular_step <= 0) angular_step = angular_step_for(a.high_resolution_limit_search, mask_radius_search);
    float psi_step;
    if (a.in_plane_angular_step <= 0) {
        psi_step = rad_2_deg(a.pixel_size / mask_radius_search);
        psi_step = (float)(360.0 / int(360.0 / psi_step + 0.5));
    } else {
        psi_step = a.in_plane_angular_step;
    }
    const float psi_start = 0.0f, psi_max = 360.0f;
    EulerSearch euler;
    if (!euler.InitGrid(a.my_symmetry, angular_step)) throw CoreError(TM_ERR_INVALID, "unrecognised symmetry " + a.my_symmetry);

    // micrograph whitening (:699-724), on the GPU
    Whitened w;
    {
        const int npts = (int)((X / 2.0 + 1.0) * sqrtf(2.0f) + 1.0);
        w.spectrum.resize((size_t)Y * (X / 2 + 1));
        w.curve.resize(npts);
        int got = 0;
        const int rc = tm_whiten_micrograph(0, input.v.data(), X, Y, reinterpret_cast<float*>(w.spectrum.data()),
                                            w.curve.data(), npts, &got);
        if (rc != TM_OK) throw CoreError(rc, "micrograph whitening on the GPU failed");
    }
    Image input_image;
    input_image.logical_x_dimension = X;
    input_image.logical_y_dimension = Y;
    input_image.is_in_real_space = false;
    input_image.complex_values = std::move(w.spectrum);

    // counts (:733-772)
    // a local run searches the whole grid (:735-739); a worker its range
    const bool worker = !a.worker_result_file.empty();
    int first = 0, last = euler.number_of_search_positions - 1;
    if (worker) {
        if (a.first_search_position < 0 || a.last_search_position >= euler.number_of_search_positions ||
            a.first_search_position > a.last_search_position)
            throw CoreError(TM_ERR_INVALID, "search positions " + std::to_string(a.first_search_position) + "-" +
                                                std::to_string(a.last_search_position) + " outside the grid of " +
                                                std::to_string(euler.number_of_search_positions));
        first = a.first_search_position;
        last = a.last_search_position;
    }
    long total_correlation_positions = 0;
    int number_of_rotations = 0;
    for (float psi = psi_start; psi <= psi_max; psi += psi_step) number_of_rotations++;
    total_correlation_positions = (long)(last - first + 1) * number_of_rotations;
    float defocus_search_range = a.defocus_search_range, defocus_step = a.defocus_step;
    float pixel_size_search_range = a.pixel_size_search_range, pixel_size_step = a.pixel_size_step;
    if (defocus_step <= 0.0f) { defocus_search_range = 0.0f; defocus_step = 100.0f; }
    if (pixel_size_step <= 0.0f) { pixel_size_search_range = 0.0f; pixel_size_step = 0.02f; }
    total_correlation_positions *= (2 * myroundint(float(defocus_search_range) / float(defocus_step)) + 1);

    std::printf("\n\tFor image id %i\n", a.image_number_for_gui);
    std::printf("Searching %i positions on the Euler sphere (first-last: %i-%i)\n", last - first, first, last);
    std::printf("Searching %i rotations per position.\n", number_of_rotations);
    std::printf("There are %li correlation positions total.\n\n", total_correlation_positions);
    std::printf("Performing Search...\n\n");
    std::fflush(stdout);

    std::vector<float> mip(npix, -FLT_MAX), best_psi(npix, 0.f), best_theta(npix, 0.f), best_phi(npix, 0.f);
    std::vector<float> best_defocus(npix, 0.f), best_pixel(npix, 0.f);
    std::vector<double> sum(npix, 0.0), sumsq(npix, 0.0);
    std::vector<long> histogram_data(kHistogramBins, 0);

    CtfParams ctf{a.voltage_kV, a.spherical_aberration_mm, a.amplitude_contrast, a.defocus1, a.defocus2,
                  a.defocus_angle, a.pixel_size, a.phase_shift};
    TemplateMatchingCore core;
    AnglesAndShifts angles;
    Image current_projection;
    current_projection.Allocate(T, T, 1, false);
    ProgressBar progress(total_correlation_positions);
    long current_correlation_position = 0;
    bool first_loop = true;
    double device_ms = 0;
    float actual_number_of_ccs_calculated = 0.0f;
    Image mip_buffer, psi_buffer, theta_buffer, phi_buffer;
    const int n_size = myroundint(float(pixel_size_search_range) / float(pixel_size_step));
    const int n_defocus = myroundint(float(defocus_search_range) / float(defocus_step));
    for (int size_i = -n_size; size_i <= n_size; size_i++) {
        Image template_reconstruction;
        template_reconstruction.logical_x_dimension = T;
        template_reconstruction.logical_y_dimension = T;
        template_reconstruction.logical_z_dimension = T;
        template_reconstruction.is_in_real_space = false;
        // the template spectrum of this pixel size (:842-845), prepared on the GPU
        template_reconstruction.complex_values.resize((size_t)T * T * (T / 2 + 1));
        {
            const float factor = (a.pixel_size + float(size_i) * pixel_size_step) / a.pixel_size;
            const int rc = tm_template_spectrum(0, rec.data.data(), T, factor,
                                                reinterpret_cast<float*>(template_reconstruction.complex_values.data()));
            if (rc != TM_OK) throw CoreError(rc, "template preparation on the GPU failed");
        }
        if (first_loop) {
            core.Init(nullptr, template_reconstruction, input_image, current_projection, pixel_size_search_range,
                      pixel_size_step, a.pixel_size, defocus_search_range, defocus_step, a.defocus1, a.defocus2,
                      psi_max, psi_start, psi_step, angles, euler, histogram_min_scaled, histogram_step_scaled,
                      kHistogramBins, std::max(fx - (int)original_x, fy - (int)original_y), first, last, &progress,
                      total_correlation_positions, true);
            first_loop = false;
        } else {
            core.SetTemplate(template_reconstruction);
        }
        for (int defocus_i = -n_defocus; defocus_i <= n_defocus; defocus_i++) {
            Image projection_filter;
            projection_filter.logical_x_dimension = T;
            projection_filter.logical_y_dimension = T;
            projection_filter.is_in_real_space = true;
            projection_filter.real_values = tmhost::projection_filter(T, w.curve, ctf, float(defocus_i) * defocus_step);
            core.RunInnerLoop(projection_filter, (float)size_i, (float)defocus_i, 0, current_correlation_position);
            device_ms += core.last_device_ms();
            actual_number_of_ccs_calculated += core.total_number_of_cccs_calculated;   // :984
            // host merge of the plane (match_template.cpp:918-984)
            core.d_max_intensity_projection.CopyDeviceToHost(mip_buffer, true, false);
            core.d_best_psi.CopyDeviceToHost(psi_buffer, true, false);
            core.d_best_theta.CopyDeviceToHost(theta_buffer, true, false);
            core.d_best_phi.CopyDeviceToHost(phi_buffer, true, false);
            std::vector<double> plane_sum, plane_sumsq;
            core.d_sum3.CopyDeviceToHost(plane_sum);
            core.d_sumSq3.CopyDeviceToHost(plane_sumsq);
            for (size_t p = 0; p < npix; p++) {
                if (mip_buffer.real_values[p] > mip[p]) {
                    mip[p] = mip_buffer.real_values[p];
                    best_psi[p] = psi_buffer.real_values[p];
                    best_theta[p] = theta_buffer.real_values[p];
                    best_phi[p] = phi_buffer.real_values[p];
                    best_defocus[p] = float(defocus_i) * defocus_step;
                    best_pixel[p] = float(size_i) * pixel_size_step;
                }
                sum[p] += plane_sum[p];
                sumsq[p] += plane_sumsq[p];
            }
            core.histogram.CopyToHostAndAdd(histogram_data.data());
        }
    }
    const double overall_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    std::printf("\n\n\tTimings: Overall: %.3f s (device search %.3f s)\n", overall_s, device_ms * 1e-3);

    // rotate back (:1177-1211): the sums pass through float images
    int ox = X, oy = Y;
    if (rotated) {
        auto rot = [&](std::vector<float>& v) {
            Image2 r = rotate90(as_image2(v, ox, oy), false);
            v = std::move(r.v);
        };
        rot(mip); rot(best_psi); rot(best_theta); rot(best_phi); rot(best_defocus); rot(best_pixel);
        std::vector<float> fs(sum.begin(), sum.end()), fq(sumsq.begin(), sumsq.end());
        rot(fs); rot(fq);
        for (size_t p = 0; p < npix; p++) { sum[p] = (double)fs[p]; sumsq[p] = (double)fq[p]; }
        std::swap(ox, oy);
    }

    if (worker) {
        // the worker's result array (:1373-1530): raw MIP, best parameters and
        // the sums as float images, on the rotated-back box
        WorkerMaps m;
        m.nx = ox;
        m.ny = oy;
        m.mip = mip; m.psi = best_psi; m.theta = best_theta; m.phi = best_phi;
        m.defocus = best_defocus; m.pixel = best_pixel;
        m.sum.assign(sum.begin(), sum.end());
        m.sumsq.assign(sumsq.begin(), sumsq.end());
        const int remove_npix_from_edge = myroundint(a.particle_radius_angstroms / a.pixel_size);   // :494
        const std::vector<float> result =
            pack_worker_result(m, original_x, original_y, remove_npix_from_edge, actual_number_of_ccs_calculated,
                               sqrt_input_pixels, histogram_data.data(), kHistogramBins);
        if (!write_result_array(a.worker_result_file, result))
            throw CoreError(TM_ERR_INVALID, "cannot write " + a.worker_result_file);
        std::printf("Result array of %zu floats (search positions %i-%i, %.0f correlation maps) written to %s\n",
                    result.size(), first, last, (double)actual_number_of_ccs_calculated, a.worker_result_file.c_str());
        return 0;
    }

    // statistics (:1215-1245)
    for (size_t p = 0; p < npix; p++) {
        sum[p] /= float(total_correlation_positions);
        sumsq[p] = sumsq[p] / float(total_correlation_positions) - powf((float)sum[p], 2);
        if (sumsq[p] > 0.0f) sumsq[p] = sqrtf((float)sumsq[p]) * (float)sqrt_input_pixels;
        else sumsq[p] = 0.0f;
        sum[p] *= (float)sqrt_input_pixels;
    }
    for (size_t p = 0; p < npix; p++) mip[p] *= (float)sqrt_input_pixels;

    // expected threshold (:1270-1284).  The reference's non-MKL build discards
    // the value of cisTEM_erfcinv and prints an uninitialised variable; the
    // value is used here.
    const double erf_input = 2.0 / (1.0 * (double)original_x * (double)original_y * (double)total_correlation_positions);
    const double temp_threshold = erfcinv_approx(erf_input);
    const float expected_threshold = sqrtf(2.0f) * (float)temp_threshold * 1.0f;

    // outputs (:1290-1330), resized to the original micrograph size
    auto out = [&](const std::vector<float>& v, bool edge_pad) {
        Image2 im = as_image2(v, ox, oy);
        return clip_into(im, (int)original_x, (int)original_y, edge_pad ? edge_mean(im) : 0.0f);
    };
    write_or_die(a.mip_output_file, out(mip, true), a.pixel_size);
    std::vector<float> scaled(npix), avg(npix), sd(npix);
    for (size_t p = 0; p < npix; p++) {
        float v = (float)((double)mip[p] - sum[p]);
        if (sumsq[p] > 0.0f) v = (float)((double)v / sumsq[p]);
        else v = 0.0f;
        scaled[p] = v;
        avg[p] = (float)sum[p];
        sd[p] = (float)sumsq[p];
    }
    write_or_die(a.scaled_mip_output_file, out(scaled, true), a.pixel_size);
    write_or_die(a.correlation_avg_output_file, out(avg, true), a.pixel_size);
    write_or_die(a.correlation_std_output_file, out(sd, true), a.pixel_size);
    write_or_die(a.best_psi_output_file, out(best_psi, false), a.pixel_size);
    write_or_die(a.best_theta_output_file, out(best_theta, false), a.pixel_size);
    write_or_die(a.best_phi_output_file, out(best_phi, false), a.pixel_size);
    write_or_die(a.best_defocus_output_file, out(best_defocus, false), a.pixel_size);
    write_or_die(a.best_pixel_size_output_file, out(best_pixel, false), a.pixel_size);

    // histogram text file (:1333-1364): NumericTextFile with 4 columns
    FILE* hf = std::fopen(a.output_histogram_file.c_str(), "w");
    if (!hf) throw CoreError(TM_ERR_INVALID, "cannot write " + a.output_histogram_file);
    const float temp_float = kHistogramMin + (histogram_step / 2.0f);
    std::vector<double> expected(kHistogramBins), survival(kHistogramBins, 0.0);
    for (int i = 0; i < kHistogramBins; i++)
        expected[i] = (erfcf((temp_float + histogram_step * float(i)) / sqrtf(2.0f)) / 2.0f) *
                      ((float)(sqrt_input_pixels * sqrt_input_pixels) * float(total_correlation_positions));
    survival[kHistogramBins - 1] = (double)histogram_data[kHistogramBins - 1];
    for (int i = kHistogramBins - 2; i >= 0; i--) survival[i] = survival[i + 1] + (double)histogram_data[i];
    std::fprintf(hf, "# Expected threshold = %.2f\n", expected_threshold);
    std::fprintf(hf, "# SNR, histogram, survival histogram, random survival histogram\n");
    for (int i = 0; i < kHistogramBins; i++)
        std::fprintf(hf, "%f %f %f %f\n", (double)(temp_float + histogram_step * float(i)), (double)histogram_data[i],
                     survival[i], expected[i]);
    if (std::fclose(hf) != 0) throw CoreError(TM_ERR_INVALID, "write failed for " + a.output_histogram_file);
    std::printf("Expected threshold = %.2f\n", expected_threshold);

    // Peaks and result image (the reference's result aggregation,
    // match_template.cpp:1838-1975), when the result file argument (38) names a
    // file: the projection montage is written there as MRC, and the peak
    // records -- which the reference stores in its project database -- as text
    // next to it (<result file without .mrc>_peaks.txt).
    if (!a.result_output_filename.empty() && a.result_output_filename != "/dev/null") {
        Image2 z = out(scaled, true), ps = out(best_psi, false), th = out(best_theta, false), ph = out(best_phi, false);
        Image2 df = out(best_defocus, false), px = out(best_pixel, false);
        const auto peaks = find_peaks(z.nx, z.ny, z.v, ps.v.data(), th.v.data(), ph.v.data(), df.v.data(), px.v.data(),
                                      expected_threshold, (int)a.min_peak_radius, T, a.pixel_size);
        const std::string peak_file = write_peak_records(a.result_output_filename, peaks, expected_threshold,
                                                         (int)a.min_peak_radius);
        if (peak_file.empty()) throw CoreError(TM_ERR_INVALID, "cannot write the peak records next to " +
                                                                   a.result_output_filename);
        Image2 montage;
        montage.nx = z.nx;
        montage.ny = z.ny;
        montage.v = projection_montage(rec.data, T, peaks, z.nx, z.ny);
        write_or_die(a.result_output_filename, montage, a.pixel_size);
        std::printf("%zu peaks written to %s; result image %s\n", peaks.size(), peak_file.c_str(),
                    a.result_output_filename.c_str());
    }
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    JobArgs a;
    if (argc == 1) {
        a = interactive();
    } else if ((argc != 43 && argc != 44) || !parse_job_args(argc, argv, 1, a)) {
        std::fprintf(stderr,
                     "usage: %s                 (interactive)\n"
                     "       %s ARG0 ... ARG41  (the 42 match_template job arguments)\n"
                     "       %s ARG0 ... ARG41 RESULT_ARRAY  (worker job over search positions ARG32-ARG33)\n",
                     argv[0], argv[0], argv[0]);
        return 2;
    }
    if (argc == 44) a.worker_result_file = argv[43];
    try {
        return run(a);
    } catch (const CoreError& e) {
        std::fprintf(stderr, "\nError: %s\n", e.what());
        return 1;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "\nError: %s\n", e.what());
        return 1;
    }
}
