// refine.hpp -- refine_template: local refinement of match_template peaks
// (src/programs/refine_template/refine_template.cpp).
//
// For every peak of the scaled MIP above a threshold, the reference scores a
// T x T window of the whitened micrograph centred on the peak against
// projections of the template (TemplateScore, :24-80: Fourier slice,
// transform to real space, optional pixel-size change, projection filter,
// normalisation, cross-correlation, integer peak) and moves the angles,
// defocus and pixel size by coordinate descent (:740-1080).  Here each peak's
// descent runs in a host worker; a worker that needs a score hands the
// candidate to a batcher, which sends the candidates of all waiting workers to
// the GPU in one batch (tm_refine_score).  The descent itself -- the order of
// the candidates, the comparisons, which map entries are written -- is the
// reference's.
#pragma once
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <exception>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "prep.hpp"

namespace tmhost {

// One TemplateScore evaluation.
struct RefineCandidate {
    float phi = 0, theta = 0, psi = 0;
    float defocus1 = 0, defocus2 = 0;   // Angstrom, as passed to CTF::SetDefocus times the pixel size
    float pixel_size_factor = 1.0f;
    int particle = 0;                   // window of the peak being refined
};

struct RefineScore {
    float value = 0, x = 0, y = 0;      // Peak of the correlation (x, y relative to the window centre)
};

// Evaluates candidates; called concurrently from the workers.
using ScoreFn = std::function<RefineScore(const RefineCandidate&)>;

// The job arguments refine_template reads (refine_template.cpp:296-346),
// with the derived steps (:314-320, 620-635).
struct RefineParams {
    float pixel_size = 1, voltage_kV = 300, spherical_aberration_mm = 2.7f, amplitude_contrast = 0.07f;
    float defocus1 = 10000, defocus2 = 10000, defocus_angle = 0, phase_shift = 0;
    float angular_step = 0.2f, in_plane_angular_step = 0.1f;
    float defocus_search_range = 200, defocus_search_step = 10;
    float pixel_size_search_range = 0.1f, pixel_size_search_step = 0.01f;
    float padding = 1.0f, mask_radius = 0.0f;
    float wanted_threshold = 7.5f, min_peak_radius = 10.0f;
    float xy_change_threshold = 10.0f;
    bool exclude_above_xy_threshold = false;
    int max_threads = 1;
};

// Maps of a match_template result, compact [y][x] (nx * ny each).
struct RefineMaps {
    int nx = 0, ny = 0;
    std::vector<float> mip, scaled_mip, psi, theta, phi, defocus, pixel_size;
};

// Peaks of the scaled MIP as refine_template picks them (:503-553):
// FindPeakWithIntegerCoordinates(0, FLT_MAX, 50) on a copy, stop below the
// threshold, blank the pixels with squared distance <= min_peak_radius (the
// value is compared with the squared distance as given).  x, y are relative
// to the box centre (nx/2, ny/2).
struct FoundPeak {
    float x = 0, y = 0, value = 0;
};
std::vector<FoundPeak> refine_find_peaks(const RefineMaps& maps, float wanted_threshold, float min_peak_radius);

// The T x T window of the whitened micrograph centred on a peak:
// RealSpaceIntegerShift (image.cpp:9064-9110, a shift of the flat pixel
// array with the reference's float remainder) and a centred ClipInto.
std::vector<float> window_particle(const Image2& whitened, int peak_x, int peak_y, int T);

// Image::CosineMask(radius, edge) on a centred T x T real image
// (image.cpp:3934-4080): values beyond the soft edge are replaced by the mean
// of the edge ring, values in the ring blended with it by a raised cosine.
void cosine_mask(std::vector<float>& image, int T, float wanted_mask_radius, float wanted_mask_edge);

// Image::ChangePixelSize(this, factor, 0.001, return_fft = true)
// (image.cpp:8705-8822) of a real nin x nin projection into an nout x nout
// one, written as a real-linear operator of the projection P:
//   out = Ar P Brt - Ai P Bit + pv C,   pv = mean of P within 0.45 nin of the centre,
// (Ar, Ai: nout x nin rows; Br, Bi: nout x nin columns, stored transposed;
// C: nout x nout), followed by the forward FFT.  The pad / new sizes and the
// disc follow the reference's float arithmetic.  `identity` is set when the
// factor is within the tolerance (the projection is only clipped).
struct PixelSizeOperator {
    int nin = 0, nout = 0;
    bool identity = false;
    int pad = 0, new_size = 0;
    bool has_pad_value = false;
    std::vector<float> ar, ai, brt, bit, c;   // nout*nin, nout*nin, nin*nout, nin*nout, nout*nout
};
PixelSizeOperator pixel_size_operator(int nin, int nout, float factor, float tolerance = 0.001f);

// Output of one refined peak (all_peak_infos / all_peak_changes, :1096-1111).
struct RefinedPeak {
    float x = 0, y = 0;                      // new position, pixels relative to the box centre
    float psi = 0, theta = 0, phi = 0, defocus = 0, pixel_size = 0, peak_height = 0;
    float dx = 0, dy = 0;                    // shift, Angstrom
    float dpsi = 0, dtheta = 0, dphi = 0, ddefocus = 0, dpixel_size = 0, dpeak_height = 0;
    float offset_distance = 0;               // pixels
    long best_address = 0;                   // in the FFTW-padded layout of the maps
    int evaluations = 0;                     // TemplateScore calls the reference makes
    int distinct_evaluations = 0;            // of which distinct candidates (the rest are repeats)
};

struct RefineOutputs {
    RefineMaps maps;                         // best MIP, scaled MIP, psi, theta, phi, defocus, pixel size
    std::vector<FoundPeak> peaks;
    std::vector<RefinedPeak> refined;
    long long evaluations = 0, distinct_evaluations = 0;
};

// The refinement loop of refine_template.cpp:636-1130 over `peaks`, scoring
// through `score`.  Workers = min(max_threads, peaks); each worker keeps its
// own copies of the parameter maps across the peaks it takes (as the
// reference's OpenMP threads do), stored sparsely over the input maps.
// `T` is the template box; `particle_of_peak[k]` is passed to the scorer.
// `worker_begin` runs once per worker before any worker starts and
// `worker_end` when a worker has no peaks left (the batcher's bookkeeping).
RefineOutputs refine_peaks(const RefineMaps& in, const std::vector<FoundPeak>& peaks, const RefineParams& p, int T,
                           const ScoreFn& score, bool verbose = false,
                           const std::function<void()>& worker_begin = nullptr,
                           const std::function<void()>& worker_end = nullptr);

// Gathers concurrent score requests into batches: a worker calls score(); when
// every active worker is waiting, the last one runs `run_batch` on all of
// them.  Workers announce their start and end so that the batch never waits
// on a finished worker.
class ScoreBatcher {
public:
    using BatchFn = std::function<void(const std::vector<RefineCandidate>&, std::vector<RefineScore>&)>;
    explicit ScoreBatcher(BatchFn run_batch) : run_batch_(std::move(run_batch)) {}
    void worker_started();
    void worker_finished();
    RefineScore score(const RefineCandidate& c);
    long long batches() const { return batches_; }
    long long scored() const { return scored_; }

private:
    struct Request {
        RefineScore out;
        bool done = false;
    };
    void run_locked(std::unique_lock<std::mutex>& lock);
    BatchFn run_batch_;
    std::mutex mu_;
    std::condition_variable cv_;
    int active_ = 0;
    bool running_ = false;
    std::exception_ptr error_;
    std::vector<RefineCandidate> pending_;
    std::vector<Request*> requests_;
    long long batches_ = 0, scored_ = 0;
};

}  // namespace tmhost
