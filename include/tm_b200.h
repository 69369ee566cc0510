/*
 * tm_b200.h -- C ABI of the B200 match_template search core.
 *
 * The search core replaces the GPU inner loop of cisTEM's match_template:
 * TemplateMatchingCore (src/gpu/TemplateMatchingCore.h:55-179,
 * src/gpu/TemplateMatchingCore.cu:49-368) and the host merge that consumes its
 * outputs (src/programs/match_template/match_template.cpp:918-986).  Unlike the
 * reference GPU path, slice extraction, filtering, normalisation and both
 * micrograph-size FFTs run on the device, and the numerics follow the
 * reference CPU path (match_template.cpp:996-1166), which is the parity target.
 *
 * All entry points take plain pointers and sizes, return an int status
 * (TM_OK = 0, negative on error) and never abort the process.  Host buffers
 * belong to the caller and are copied during the call.  One context drives one
 * GPU from one host thread.
 */
#ifndef TM_B200_H
#define TM_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define TM_API __attribute__((visibility("default")))
#else
#define TM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define TM_OK 0
#define TM_ERR_INVALID (-1)      /* bad argument or call order */
#define TM_ERR_CUDA (-2)         /* CUDA runtime error (message in tm_last_error) */
#define TM_ERR_UNSUPPORTED (-3)  /* geometry without a compiled kernel variant */
#define TM_ERR_OOM (-4)          /* device allocation failed */
#define TM_ERR_TIMEOUT (-5)      /* a bounded wait ran out */
#define TM_ERR_CANCELLED (-6)    /* the progress callback asked to stop */

typedef struct tm_ctx tm_ctx;

/* Geometry and histogram set-up.  Mirrors the sizes and histogram arguments of
 * TemplateMatchingCore::Init (TemplateMatchingCore.h:147-171):
 * image_x/image_y are the padded (factorised) micrograph dimensions of
 * input_image, template_size the cubic box of template_reconstruction,
 * histogram_min_scaled / histogram_step_scaled / histogram_bins the values of
 * match_template.cpp:633-644. */
typedef struct tm_dims {
    int image_x;
    int image_y;
    int template_size;
    int histogram_bins;            /* 512 in the reference */
    double histogram_min_scaled;   /* histogram_min / sqrt(X*Y) */
    double histogram_step_scaled;  /* histogram_step / sqrt(X*Y) */
    int orientation_batch;         /* orientations per device pass; 0 = automatic (32 until
                                      tm_autotune_batch picks 16, 32, 64 or 128) */
    int device;                    /* CUDA device ordinal */
} tm_dims;

/* Called after each device pass with the number of orientations finished in
 * the current plane; a non-zero return cancels the plane (TM_ERR_CANCELLED). */
typedef int (*tm_progress_fn)(long long orientations_done, long long orientations_total, void *user);

/* Replaces TemplateMatchingCore::Init's device set-up (TemplateMatchingCore.cu:49-138):
 * allocates every device buffer for the geometry.  Geometries with compiled
 * kernel variants run those; any other micrograph with both sides in 64..8192
 * whose lengths (and half width, when even) factor into 2, 3, 5, 7, 11 and 13
 * -- every size the reference's padding picks -- runs the run-time-length
 * kernels, for templates of 32, 48, 64, 128, 256 or 384.  Status
 * TM_ERR_UNSUPPORTED otherwise. */
TM_API int tm_create(const tm_dims *dims, tm_ctx **out);

/* Uploads the template spectrum: the quadrant-swapped Fourier transform of the
 * template volume exactly as match_template.cpp:842-845 leaves it in
 * template_reconstruction (ChangePixelSize(..., return_fft=true),
 * ZeroCentralPixel, SwapRealSpaceQuadrants).  spectrum: T*T*(T/2+1) complex
 * values as interleaved float pairs, layout [z][y][x]. */
TM_API int tm_set_template(tm_ctx *ctx, const float *spectrum, int template_size);

/* Uploads the whitened micrograph spectrum (input_image.complex_values after
 * match_template.cpp:703-724): image_y*(image_x/2+1) complex values as
 * interleaved float pairs, layout [y][x]. */
TM_API int tm_set_image(tm_ctx *ctx, const float *spectrum, int image_x, int image_y);

/* Micrograph whitening on the device (no counterpart in the reference, whose
 * DoCalculation whitens on the CPU, match_template.cpp:699-724): the padded
 * (and, where the reference rotates it, rotated) image_x x image_y micrograph,
 * [y][x] floats, goes through ReplaceOutliersWithMean(5), ForwardFFT,
 * SwapRealSpaceQuadrants, ZeroCentralPixel, Compute1DPowerSpectrumCurve, the
 * square root / reciprocal / 1/max of the curve, ApplyCurveFilter,
 * ZeroCentralPixel and the division by sqrt(ReturnSumOfSquares) -- the
 * spectrum tm_set_image takes -- and becomes the context's micrograph.  curve
 * (may be NULL) receives the whitening filter the projection filters use,
 * int((image_x/2+1) sqrt(2) + 1) points on [0, sqrt(2)/2]; curve_points (may
 * be NULL) that count. */
TM_API int tm_set_micrograph(tm_ctx *ctx, const float *image, int image_x, int image_y, double *curve,
                             int curve_capacity, int *curve_points);

/* The same whitening without a search context, for the sizes the search has
 * kernels for: spectrum receives image_y*(image_x/2+1) complex (float pairs). */
TM_API int tm_whiten_micrograph(int device, const float *image, int image_x, int image_y, float *spectrum,
                                double *curve, int curve_capacity, int *curve_points);

/* Template spectrum on the device (the reference prepares it on the CPU,
 * match_template.cpp:842-845): the T^3 real volume ([z][y][x]) goes through
 * ChangePixelSize(pixel_size_factor, tolerance 0.001, return_fft),
 * ZeroCentralPixel and SwapRealSpaceQuadrants -- the spectrum tm_set_template
 * takes -- and becomes the context's template.  Boxes 32, 48, 64, 128, 256,
 * 384; a factor whose resampled box is not larger than T returns
 * TM_ERR_UNSUPPORTED. */
TM_API int tm_set_template_volume(tm_ctx *ctx, const float *volume, int template_size, float pixel_size_factor);

/* The same without a search context: spectrum receives T*T*(T/2+1) complex
 * (float pairs). */
TM_API int tm_template_spectrum(int device, const float *volume, int template_size, float pixel_size_factor,
                                float *spectrum);

/* Arithmetic of the search's correlation transforms (no counterpart in the
 * reference's CPU path; its GPU path runs cuFFT with FP16 image and
 * correlation buffers, src/gpu/GpuImage.cu:2138-2145,
 * TemplateMatchingCore.cu:388-425).
 *   TM_PRECISION_FP32 (default): every transform in FP32, the parity path.
 *   TM_PRECISION_FP16_TENSOR: the column pass stores its correlation spectra
 *   as FP16 (times a power of two) and the row pass runs its inverse
 *   transform as two DFT-matrix stages on the tensor cores (FP16 operands,
 *   FP32 accumulation); the MIP and the compensated sums stay FP32, their
 *   batch totals FP64.  MIP error about 1e-4 of the MIP scale.
 * TM_ERR_UNSUPPORTED for geometries without the FP16 kernels (image_x of
 * 1024, 2048 or 4096 and image_y a power of two or 3888 have them). */
#define TM_PRECISION_FP32 0
#define TM_PRECISION_FP16_TENSOR 1
TM_API int tm_set_precision(tm_ctx *ctx, int precision);
TM_API int tm_get_precision(const tm_ctx *ctx);

/* Pixel count that the projection variance is formed over (match_template.cpp:1066-1067
 * use the padded micrograph's). 0, the default, is the context's X*Y. A context that
 * searches a window cut from a larger whitened micrograph passes that micrograph's
 * pixel count, so that its correlation values are the larger search's at the
 * window's interior positions (the window search of the learned proposal). */
TM_API int tm_set_normalization_pixels(tm_ctx *ctx, long long n_pixels);

/* Clears the running MIP (to -FLT_MAX), best-orientation, sum, sum-of-squares
 * and histogram state, as RunInnerLoop does at entry (TemplateMatchingCore.cu:143-155);
 * also the results of the image set, if the context has one. */
TM_API int tm_reset_results(tm_ctx *ctx);

/* Image set (no counterpart in the reference): n_images micrograph spectra of
 * the context's size (each laid out as for tm_set_image, one after another),
 * each with its own running MIP / best orientation / sums / histogram.  Starts
 * a new search (as tm_reset_results).  For many small searches that share
 * orientations, e.g. the windows of the learned proposal. */
TM_API int tm_set_image_set(tm_ctx *ctx, int n_images, const float *spectra);

/* tm_run_plane over the images of the set listed in `images`: each orientation
 * batch is sliced, projected and normalised once and correlated with every
 * listed image.  Every call registers its orientations as one plane. */
TM_API int tm_run_plane_images(tm_ctx *ctx, const float *projection_filter, const float *euler_angles,
                               int n_orientations, const int *images, int n_images, float defocus_offset,
                               float pixel_size_offset);

/* MIP and best angles of one image of the set ([y][x], any pointer may be NULL). */
TM_API int tm_get_image_results(tm_ctx *ctx, int image, float *mip, float *best_psi, float *best_theta,
                                float *best_phi);

/* Replaces TemplateMatchingCore::RunInnerLoop (TemplateMatchingCore.cu:140-368)
 * for one (pixel size, defocus) plane: for every orientation in order,
 * extract the Fourier slice, apply the projection filter (CTF x whitening,
 * match_template.cpp:895-898; T*(T/2+1) reals, layout [y][x]), normalise,
 * correlate with the micrograph and fold the correlation map into the running
 * MIP / argmax / sums / histogram.  euler_angles holds n_orientations triples
 * (phi, theta, psi) in degrees, in the reference's loop order (search
 * position outer, psi inner).  defocus_offset / pixel_size_offset are the
 * values recorded for pixels whose maximum comes from this plane
 * (float(defocus_i)*defocus_step, float(size_i)*pixel_size_step).
 * Results accumulate across planes until tm_reset_results. */
TM_API int tm_run_plane(tm_ctx *ctx, const float *projection_filter, const float *euler_angles, int n_orientations,
                 float defocus_offset, float pixel_size_offset, tm_progress_fn progress, void *user);

/* Copies the running results to host memory (any pointer may be NULL).
 * Maps are image_y*image_x, layout [y][x]: MIP (unscaled correlation), best
 * psi/theta/phi (degrees), best defocus and pixel-size offsets, and the per
 * pixel sum and sum of squares of every correlation value in double.
 * histogram receives histogram_bins counts.  These are the outputs that
 * match_template.cpp:918-984 reads from d_max_intensity_projection,
 * d_best_psi/theta/phi, d_sum3, d_sumSq3 and Histogram::CopyToHostAndAdd. */
TM_API int tm_get_results(tm_ctx *ctx, float *mip, float *best_psi, float *best_theta, float *best_phi,
                   float *best_defocus, float *best_pixel_size, double *sum, double *sum_of_squares,
                   long long *histogram);

/* Number of correlation maps computed since the last reset
 * (TemplateMatchingCore::total_number_of_cccs_calculated). */
TM_API long long tm_correlations_computed(const tm_ctx *ctx);

/* Device time of the last tm_run_plane call in milliseconds and its split per
 * kernel family (for roofline accounting); any pointer may be NULL. */
TM_API int tm_last_timing(const tm_ctx *ctx, double *total_ms, double *pass_b_ms, double *pass_c_ms, double *prep_ms);

/* Runs one orientation through every kernel up to the column pass, leaving
 * the running results untouched, and copies the intermediates (any pointer
 * may be NULL): slice = filtered Fourier slice after the inverse FFT along y
 * (T*(T/2+1) complex, [y][x]); projection = real T*T projection before
 * normalisation; normalisation = (edge mean, 1/sigma) as in
 * match_template.cpp:1060-1068; rows = forward FFT along x of the T
 * normalised rows (T*(X/2+1) complex); columns = the correlation spectrum
 * after the inverse FFT along y (Y*(X/2+1) complex).  For kernel-level
 * parity tests and diagnostics; it has no counterpart in the reference. */
TM_API int tm_debug_stage_buffers(tm_ctx *ctx, const float *projection_filter, const float *euler_angle, float *slice,
                                  float *projection, float *normalisation, float *rows, float *columns);

/* One product C = (A - s) B (+ C when accumulate) of the dense-operator GEMMs
 * that the pixel-size change runs on the device (template volume and
 * refine_template), on `device`: tensor = 1 the tensor-core form (split TF32,
 * FP32 accumulation) the library uses, 0 the FP32 CUDA-core form.  Row-major
 * host arrays A (M x K), B (K x N), C (M x N).  For kernel-level tests; it
 * has no counterpart in the reference. */
TM_API int tm_debug_gemm(int device, int M, int N, int K, const float *A, const float *B, float *C, float s,
                         int accumulate, int tensor);

/* Plane search that allocates no device memory, for callers that cannot call
 * cudaMalloc: code inside a host framework that owns every device allocation
 * through its own pool, and plugins that are only handed pre-allocated
 * buffers.  It has no counterpart in the reference.
 *
 * Same search as tm_run_plane, on the caller's device buffers: the template
 * spectrum (as tm_set_template), the whitened micrograph spectrum (as
 * tm_set_image), the projection filter, and the running results -- MIP
 * (start at -FLT_MAX), best orientation index (start at -1; receives
 * first_orientation_index + the orientation's position in euler_angles),
 * sum, sum of squares (start at 0) and histogram (start at 0), each
 * image_y*image_x ([y][x]) or histogram_bins long.  euler_angles is host
 * memory, n_orientations (phi, theta, psi) triples.  The work is ordered on
 * `stream` (a cudaStream_t; NULL = the default stream) and the call returns
 * when it is done.  The caller's current device is restored before return.
 *
 * All intermediates live in one fixed device array of 16 MiB, which every GPU
 * that loads this library holds until the process exits.  The compiled
 * geometries (template 32 on 256x256 or 512x512, template 64 on 512x512) all
 * fit it; any other geometry returns TM_ERR_UNSUPPORTED.  The first call on a
 * device looks up that array's device address and sets kernel attributes, so
 * make it before any stream capture.  Every call reuses the same array: calls
 * that overlap on the GPU (other streams, other host threads) race and corrupt
 * each other's results. */
TM_API int tm_run_plane_noalloc(int device, const tm_dims *dims, const float *d_template_spectrum,
                                const float *d_image_spectrum, const float *d_projection_filter,
                                const float *euler_angles, int n_orientations, int first_orientation_index,
                                float *d_mip, int *d_best, double *d_sum, double *d_sum_of_squares,
                                unsigned long long *d_histogram, void *stream);

/* Automatic orientation batch (no counterpart in the reference, whose GPU
 * path processes one orientation per launch).  For a context created with
 * orientation_batch = 0, times tm_run_plane over the given orientations with
 * 16, 32, 64 and 128 orientations per device pass (the larger ones only when
 * their correlation spectra fit in a quarter of the free device memory at
 * tm_create), keeps the fastest and clears the running results.  Use 256 or
 * more orientations of the real search.
 * chosen (may be NULL) receives the batch.  The template and image must be set. */
TM_API int tm_autotune_batch(tm_ctx *ctx, const float *projection_filter, const float *euler_angles,
                             int n_orientations, int *chosen);

/* Orientations per device pass currently used by the context. */
TM_API int tm_orientation_batch(const tm_ctx *ctx);

/* Frees every device buffer of the context. */
TM_API int tm_destroy(tm_ctx *ctx);

/* Message of the last error on this context (never NULL). */
TM_API const char *tm_last_error(const tm_ctx *ctx);

/* Version string of the library build. */
TM_API const char *tm_version(void);

/* ---------------------------------------------------------------------------
 * refine_template scoring.  Replaces TemplateScore
 * (src/programs/refine_template/refine_template.cpp:24-80), which the
 * reference evaluates one candidate at a time on the CPU inside OpenMP threads;
 * here a batch of candidates is scored in one call.  A candidate's score is
 * the peak (value, x, y relative to the box centre) of the correlation between
 * a particle window and the projection of the template at the candidate's
 * Euler angles: Fourier slice (ExtractSlice), quadrant swap, inverse FFT,
 * optional pixel-size change (ChangePixelSize with return_fft), forward FFT,
 * projection filter, zeroed central pixel, division by the square root of
 * ReturnSumOfSquares, product with the conjugate into the particle spectrum,
 * inverse FFT, FindPeakWithIntegerCoordinates. */
typedef struct tm_refine_ctx tm_refine_ctx;

/* template_box T: the scored box; projection_box TP: T or 2T (the reference's
 * padding factor 1 or 2).  template_spectrum: TP*TP*(TP/2+1) complex (float
 * pairs, [z][y][x]) -- the TP^3 template after ForwardFFT, ZeroCentralPixel
 * and SwapRealSpaceQuadrants (refine_template.cpp:586-599).  Capacities: the
 * candidates per device pass and the slots of particle windows, filters and
 * pixel-size operators.  TM_ERR_UNSUPPORTED for boxes without a compiled
 * variant (T in 32, 48, 64, 128, 256, 384). */
TM_API int tm_refine_create(int device, int template_box, int projection_box, const float *template_spectrum,
                            int max_batch, int max_particles, int max_filters, int max_operators,
                            tm_refine_ctx **out);

/* Particle window slot: T*(T/2+1) complex, the forward FFT (any scale) of the
 * T x T window of the whitened micrograph with quadrants swapped
 * (refine_template.cpp:720-724). */
TM_API int tm_refine_set_particle(tm_refine_ctx *ctx, int slot, const float *spectrum);

/* Projection filter slot: T*(T/2+1) reals (CTF image x whitening curve). */
TM_API int tm_refine_set_filter(tm_refine_ctx *ctx, int slot, const float *filter);

/* Pixel-size operator slot (ChangePixelSize of the TP x TP projection into
 * T x T written as out = Ar (P - pv) Brt - Ai (P - pv) Bit + pv, pv = mean of
 * P within 0.45 TP of its centre when has_pad_value): ar, ai T*TP; brt, bit
 * TP*T, row-major. */
TM_API int tm_refine_set_operator(tm_refine_ctx *ctx, int slot, const float *ar, const float *ai, const float *brt,
                                  const float *bit, int has_pad_value);

/* Scores n candidates: euler 3n (phi, theta, psi in degrees), particle and
 * filter slots, operator slot or -1 (pixel-size factor within the 0.001
 * tolerance: the projection is only clipped to T).  out: 3n floats (value,
 * x, y).  Returns when the scores are on the host. */
TM_API int tm_refine_score(tm_refine_ctx *ctx, int n, const float *euler, const int *particle, const int *filter,
                           const int *op, float *out);

TM_API const char *tm_refine_last_error(const tm_refine_ctx *ctx);
TM_API int tm_refine_destroy(tm_refine_ctx *ctx);

/* ---- Learned proposal network (no reference counterpart) ----------------------------
 * A 5-layer CNN over tile x tile patches of the coarse search's maps
 * (in_channels planes per tile, [tile][channel][y][x]): three 3x3 conv + ReLU +
 * 2x2 max-pool layers (32, 64, 128 channels), a 3x3 conv + ReLU (128) with a
 * global max, and a fully connected layer to 4 outputs per tile: the
 * objectness logit and a direction (x, y, z) whose nearest angular bins get the
 * fine search.  FP32 master weights with Adam state; the forward and
 * backward-data passes use their BF16 copies with FP32 accumulation.
 * Parameter order: for each conv layer its weights [co][ci][3][3] then its
 * bias, then the FC weights [4][128] and bias. */
typedef struct tm_pnet tm_pnet;

/* tile: 16, 32, 64 or 128; max_batch: tiles per call (1..4096). Parameters start at 0. */
TM_API int tm_pnet_create(int device, int in_channels, int tile, int max_batch, tm_pnet **out);
TM_API long long tm_pnet_param_count(const tm_pnet *net);
/* FP32 master values (param_count floats); clears the Adam state */
TM_API int tm_pnet_set_params(tm_pnet *net, const float *params);
TM_API int tm_pnet_get_params(tm_pnet *net, float *params);
/* outputs: 4 floats per tile (objectness logit, direction x, y, z) */
TM_API int tm_pnet_forward(tm_pnet *net, const float *tiles, int n, float *outputs);
/* labels: 4 floats per tile (objectness 0/1, unit target direction x, y, z).
 * Loss L = 1/n sum_i [w_i BCE(o_i, y_i) + dir_weight y_i (1 - cos(d_i, t_i))],
 * w_i = pos_weight for positives.  grads: param_count floats (dL/d of the BF16
 * weights the forward used, and of the biases). */
TM_API int tm_pnet_gradients(tm_pnet *net, const float *tiles, const float *labels, int n, float pos_weight,
                             float dir_weight, double *loss, float *grads);
/* One Adam step (beta 0.9, 0.999, eps 1e-8) at learning rate lr; loss may be null. */
TM_API int tm_pnet_train_step(tm_pnet *net, const float *tiles, const float *labels, int n, float pos_weight,
                              float dir_weight, float lr, double *loss);
TM_API const char *tm_pnet_last_error(const tm_pnet *net);
TM_API int tm_pnet_destroy(tm_pnet *net);

#ifdef __cplusplus
}
#endif

#endif /* TM_B200_H */
