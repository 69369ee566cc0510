// job_args.hpp -- the 42 match_template job arguments, indexed as the
// reference's MatchTemplateApp::DoCalculation reads them
// (src/programs/match_template/match_template.cpp:346-387), shared by the
// match_template program and the result merge program.
#pragma once
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "mrc.hpp"
#include "prep.hpp"

namespace tmhost {

struct JobArgs {
    std::string input_search_images, input_reconstruction;                   // 0, 1
    float pixel_size = 1, voltage_kV = 300, spherical_aberration_mm = 2.7f;   // 2-4
    float amplitude_contrast = 0.07f, defocus1 = 10000, defocus2 = 10000;     // 5-7
    float defocus_angle = 0, low_resolution_limit = 300;                      // 8, 9
    float high_resolution_limit_search = 8, angular_step = 0;                 // 10, 11
    int best_parameters_to_keep = 20;                                         // 12
    float defocus_search_range = 500, defocus_step = 50;                      // 13, 14
    float pixel_size_search_range = 0.1f, pixel_size_step = 0.02f;            // 15, 16
    float padding = 1;                                                        // 17
    bool ctf_refinement = false;                                              // 18
    float particle_radius_angstroms = 0, phase_shift = 0;                     // 19, 20
    std::string mip_output_file, best_psi_output_file, best_theta_output_file; // 21-23
    std::string best_phi_output_file, best_defocus_output_file;               // 24, 25
    std::string best_pixel_size_output_file, scaled_mip_output_file;          // 26, 27
    std::string correlation_avg_output_file, my_symmetry = "C1";              // 28, 29
    float in_plane_angular_step = 0;                                          // 30
    std::string output_histogram_file;                                        // 31
    int first_search_position = -1, last_search_position = -1;                // 32, 33
    int image_number_for_gui = 0, number_of_jobs_per_image_in_gui = 0;        // 34, 35
    std::string correlation_std_output_file, directory_for_results;           // 36, 37
    std::string result_output_filename;                                       // 38
    float min_peak_radius = 10;                                               // 39
    bool use_gpu = true;                                                      // 40
    int max_threads = 1;                                                      // 41
    std::string worker_result_file;   // not a job argument: a worker's result array file
};

inline bool parse_bool(const std::string& s) {
    return !s.empty() && (s[0] == 'y' || s[0] == 'Y' || s[0] == 't' || s[0] == 'T' || s[0] == '1');
}

// Fills `a` from argv[first] ... argv[first + 41]; false when fewer are given.
inline bool parse_job_args(int argc, char** argv, int first, JobArgs& a) {
    if (argc < first + 42) return false;
    auto S = [&](int i) { return std::string(argv[first + i]); };
    auto F = [&](int i) { return (float)std::atof(argv[first + i]); };
    auto I = [&](int i) { return std::atoi(argv[first + i]); };
    a.input_search_images = S(0); a.input_reconstruction = S(1);
    a.pixel_size = F(2); a.voltage_kV = F(3); a.spherical_aberration_mm = F(4); a.amplitude_contrast = F(5);
    a.defocus1 = F(6); a.defocus2 = F(7); a.defocus_angle = F(8); a.low_resolution_limit = F(9);
    a.high_resolution_limit_search = F(10); a.angular_step = F(11); a.best_parameters_to_keep = I(12);
    a.defocus_search_range = F(13); a.defocus_step = F(14); a.pixel_size_search_range = F(15);
    a.pixel_size_step = F(16); a.padding = F(17); a.ctf_refinement = parse_bool(S(18));
    a.particle_radius_angstroms = F(19); a.phase_shift = F(20);
    a.mip_output_file = S(21); a.best_psi_output_file = S(22); a.best_theta_output_file = S(23);
    a.best_phi_output_file = S(24); a.best_defocus_output_file = S(25); a.best_pixel_size_output_file = S(26);
    a.scaled_mip_output_file = S(27); a.correlation_avg_output_file = S(28); a.my_symmetry = S(29);
    a.in_plane_angular_step = F(30); a.output_histogram_file = S(31); a.first_search_position = I(32);
    a.last_search_position = I(33); a.image_number_for_gui = I(34); a.number_of_jobs_per_image_in_gui = I(35);
    a.correlation_std_output_file = S(36); a.directory_for_results = S(37); a.result_output_filename = S(38);
    a.min_peak_radius = F(39); a.use_gpu = parse_bool(S(40)); a.max_threads = I(41);
    return true;
}

inline void write_or_die(const std::string& path, const Image2& im, float pixel_size) {
    std::string err;
    if (!write_mrc(path, im.nx, im.ny, 1, im.v.data(), pixel_size, err)) throw std::runtime_error(err);
}

// myroundint(float) (src/core/functions.h:480-483)
inline int myroundint(float a) { return a > 0 ? (int)((double)a + 0.5) : (int)((double)a - 0.5); }

}  // namespace tmhost
