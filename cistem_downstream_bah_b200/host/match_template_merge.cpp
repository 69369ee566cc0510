// match_template_merge.cpp -- the master side of a distributed match_template
// run: MatchTemplateApp::MasterHandleProgramDefinedResult
// (src/programs/match_template/match_template.cpp:1545-1990) over the result
// arrays that worker jobs wrote (match_template ARG0 ... ARG41 RESULT_ARRAY).
//
//   match_template_merge ARG0 ... ARG41 RESULT_ARRAY [RESULT_ARRAY ...]
//
// The job arguments name the output files (21-28, 31, 36, 38) and give the
// template (1), the pixel size of the peak coordinates (2), the minimum peak
// radius (39) and use_gpu (40).  The arrays are merged in the order given
// (AggregatedTemplateResult::AddResult); then the master's outputs are
// written: the 9 images (MRC, pixel size 1.0 as the master leaves it), the
// histogram file and, when argument 38 names a file, the peak records and the
// projection montage (:1839-1975).  No GPU is used.
#include <cstdio>
#include <exception>
#include <string>
#include <vector>

#include "job_args.hpp"
#include "mrc.hpp"
#include "peaks.hpp"
#include "result_array.hpp"

using namespace tmhost;

int main(int argc, char** argv) {
    JobArgs a;
    if (argc < 44 || !parse_job_args(argc, argv, 1, a)) {
        std::fprintf(stderr, "usage: %s ARG0 ... ARG41 RESULT_ARRAY [RESULT_ARRAY ...]\n", argv[0]);
        return 2;
    }
    try {
        AggregatedTemplateResult merged;
        const int expected = argc - 43;
        for (int i = 43; i < argc; i++) {
            std::vector<float> arr;
            if (!read_result_array(argv[i], arr)) throw std::runtime_error(std::string("cannot read ") + argv[i]);
            merged.AddResult(arr.data(), (long)arr.size());
            std::printf("Received %i of %i results\n", merged.number_of_received_results, expected);
        }
        const MasterOutputs o = finalize_master(merged, a.use_gpu);
        // the master writes without a pixel size (QuickAndDirtyWriteSlice -> 1.0)
        const float px = 1.0f;
        write_or_die(a.mip_output_file, o.mip, px);
        write_or_die(a.best_psi_output_file, o.psi, px);
        write_or_die(a.best_theta_output_file, o.theta, px);
        write_or_die(a.best_phi_output_file, o.phi, px);
        write_or_die(a.best_defocus_output_file, o.defocus, px);
        write_or_die(a.best_pixel_size_output_file, o.pixel, px);
        write_or_die(a.scaled_mip_output_file, o.scaled_mip, px);
        write_or_die(a.correlation_avg_output_file, o.avg, px);
        write_or_die(a.correlation_std_output_file, o.std_dev, px);
        if (!write_master_histogram(a.output_histogram_file, o))
            throw std::runtime_error("cannot write " + a.output_histogram_file);
        std::printf("%.0f correlation maps merged; expected threshold = %.2f\n", (double)merged.total_number_of_ccs,
                    o.expected_threshold);
        if (!a.result_output_filename.empty() && a.result_output_filename != "/dev/null") {
            MrcData rec;
            std::string err;
            if (!read_mrc(a.input_reconstruction, rec, err)) throw std::runtime_error(err);
            const int T = rec.nx;
            if (rec.ny != T || rec.nz != T) throw std::runtime_error("the template reconstruction must be a cube");
            std::vector<float> z = o.scaled_mip.v;
            // int min_peak_radius = arguments[39] (:1842): truncated
            const int min_peak_radius = (int)a.min_peak_radius;
            const auto peaks = find_peaks(o.nx, o.ny, z, o.psi.v.data(), o.theta.v.data(), o.phi.v.data(),
                                          o.defocus.v.data(), o.pixel.v.data(), o.expected_threshold, min_peak_radius,
                                          T, a.pixel_size);
            const std::string peak_file = write_peak_records(a.result_output_filename, peaks, o.expected_threshold,
                                                             min_peak_radius);
            if (peak_file.empty()) throw std::runtime_error("cannot write the peak records");
            Image2 montage;
            montage.nx = o.nx;
            montage.ny = o.ny;
            montage.v = projection_montage(rec.data, T, peaks, o.nx, o.ny);
            write_or_die(a.result_output_filename, montage, px);
            std::printf("%zu peaks written to %s; result image %s\n", peaks.size(), peak_file.c_str(),
                        a.result_output_filename.c_str());
        }
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "\nError: %s\n", e.what());
        return 1;
    }
}
