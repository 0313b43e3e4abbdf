/* speckle_b200: B200-native phase retrieval for the speckle.phasing path.
 *
 * C ABI of libspeckle_b200.so.  All pointers named *_dev are device pointers
 * owned by the caller; the library allocates no device memory in any entry
 * point below (scratch lives in a caller-provided workspace).  Complex data is
 * interleaved complex64 (float re, float im), row-major N x N, with q = 0 at
 * the corner for Fourier-space arrays, as in the reference.
 *
 * Every function returns an int status (SP_OK = 0).  sp_status_string()
 * names a status; sp_last_error() returns a description of the most recent
 * failure on the calling thread.  Work is enqueued on the given CUDA stream
 * (NULL = legacy default stream) and runs asynchronously.
 *
 * Reference interfaces replaced (paths within dhparks/als_speckle):
 *   speckle/phasing.py   class phasing: load :291, seed :990, iterate :181,
 *                        _iteration :1088, _fft2 :1067, refine_support :1747,
 *                        align_global_phase :1355, prtf :1406, gpu_prtf :1463
 *   speckle/gpu.py       common._kexec :295 (kernel-by-name dispatch)
 *   speckle/kernels/     phasing_{hio,er,raar,sf,dm1,dm2,fourier,
 *                        copy_to_buffer_f2,prtf_accumulate2}.cl, common_abs_f2_f2.cl
 */
#ifndef SPECKLE_B200_H
#define SPECKLE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* sp_stream_t; /* a cudaStream_t */

enum sp_status {
  SP_OK = 0,
  SP_ERR_INVALID = 1,     /* bad argument (null pointer, bad algorithm code, ...) */
  SP_ERR_SIZE = 2,        /* N not a power of two in [8, 4096], or a size limit exceeded */
  SP_ERR_CUDA = 3,        /* a CUDA runtime call failed; see sp_last_error() */
  SP_ERR_WORKSPACE = 4,   /* workspace missing or smaller than required */
  SP_ERR_UNSUPPORTED = 5, /* request not supported by this build */
  SP_ERR_NOT_FOUND = 6    /* operator name unknown (sp_kexec) */
};

/* real-space update algorithms (phasing.py:1341 `algos`) */
enum sp_algorithm {
  SP_HIO = 0,    /* phasing_hio.cl:16-17  (1-s)(pi - b po) + s po             */
  SP_ER = 1,     /* phasing_er.cl:13-14   s po                                */
  SP_RAAR = 2,   /* phasing_raar.cl:19-20 (1-s)(b pi + (1-2b) po) + s po       */
  SP_SF = 3,     /* phasing_sf.cl:16-17   (1-s)(-po) + s po                    */
  SP_DM = 4,     /* phasing_dm1.cl / phasing_dm2.cl, gamma_m = 1/b, gamma_s = -1/b */
  SP_ER_CPU = 5, /* phasing.py:1257 CPU-branch ER: s pi                        */
  SP_SF_CPU = 6  /* phasing.py:1284 CPU-branch SF: (1-s)(-pi) + s po           */
};

enum sp_init {
  SP_INIT_GIVEN = 0,       /* psi_dev already holds the start (phasing.seed :990-1031) */
  SP_INIT_RANDOM_PHASE = 1 /* psi0 = S * IFFT(M exp(i 2 pi u)), u = hash(seed, trial, pixel) */
};

#define SP_MAX_RUNS 8

/* One independent reconstruction (one "trial" of the reference). */
typedef struct sp_trial {
  int32_t n;                       /* edge N: power of two, 8..4096 */
  int32_t n_iter;                  /* iterations to run (phasing.iterate `iterations`) */
  int32_t n_runs;                  /* entries of the cyclic order (phasing.py:244-257) */
  int32_t run_alg[SP_MAX_RUNS];    /* sp_algorithm per entry */
  int32_t run_count[SP_MAX_RUNS];  /* iterations per entry */
  float beta;                      /* feedback parameter (default 0.8, phasing.py:181) */
  int32_t init;                    /* sp_init */
  uint32_t seed, trial;            /* random-phase start key (SP_INIT_RANDOM_PHASE) */
  int32_t r0, c0, rows, cols;      /* savebuffer crop box (phasing.py:279-287) */
  void* psi_dev;                   /* complex64 N*N, in/out: psi_in */
  const float* modulus_dev;        /* float N*N, corner-centred Fourier modulus */
  const float* support_dev;        /* float N*N, support in [0,1] */
  void* save_dev;                  /* complex64 rows*cols, receives the crop, or NULL */
  double* errors_dev;              /* 2*n_iter doubles (sum(|F|-M)^2, sum||F|-M|) per
                                      iteration, or NULL; zeroed by the run */
  const void* ipsf_dev;            /* complex64 N*N transform of the coherence point spread,
                                      corner-centred (phasing.load ipsf=, phasing.py:413-424;
                                      divisor phasing.py:1122-1137), or NULL for a coherent
                                      projection */
  const float* spectrum_rescale_dev; /* spectrum_n energy / centre-energy rescale factors
                                        (phasing.py:426-450), for the longitudinal divisor
                                        phasing.py:1139-1156 and radial_rescale.cl */
  const float* spectrum_weight_dev;  /* spectrum_n spectral weights */
  int32_t spectrum_n;                /* samples of the spectrum, 0 = none */
} sp_trial;

typedef struct sp_run_opts {
  int64_t l2_group_bytes;  /* run trials in groups whose working set fits this many
                              bytes of L2 (0 = all trials together) */
  int32_t use_graph;       /* capture each group's launch sequence in a CUDA graph
                              (needs a non-default stream; graphs are cached per
                              workspace and launch shape) */
  int32_t ctas_per_sm;     /* cap on resident CTAs per SM of the persistent grid (0 = max) */
  int32_t e_per_logn[13];  /* values per thread (16 or 32) for N = 2^l; 0 = default */
} sp_run_opts;

/* ---- library ---------------------------------------------------------- */
int sp_version(void);
const char* sp_status_string(int status);
const char* sp_last_error(void);
/* Upload the twiddle tables on the current device (also done on first use). */
int sp_device_init(void);

/* ---- fused iteration engine ------------------------------------------- */
/* Replaces phasing.iterate (phasing.py:181-289) for one or many trials.
 * Bytes of workspace that sp_engine_run needs for these trials. */
int sp_engine_workspace_size(const sp_trial* trials, int n_trials, size_t* bytes);
/* Run every trial's iterations (uneven sizes and algorithms allowed), write
 * the final psi_in, the crop into save_dev and the per-iteration errors.
 * The pass kernels are launched with programmatic stream serialization and
 * let the next kernel of the stream start early: work the caller enqueues
 * afterwards with plain launches, copies or events sees the results as usual;
 * a caller kernel launched itself with programmatic stream serialization must
 * wait for its predecessor grid (cudaGridDependencySynchronize) before
 * reading them. */
int sp_engine_run(const sp_trial* trials, int n_trials, void* workspace_dev,
                  size_t workspace_bytes, const sp_run_opts* opts, sp_stream_t stream);
/* Destroy the CUDA graphs cached by sp_engine_run (call before freeing a
 * workspace that was used with use_graph = 1). */
int sp_engine_release_graphs(void);
/* Number of CUDA graphs sp_engine_run holds in its cache (one per workspace
 * and launch shape); a long-running caller whose shapes keep changing can
 * release them (sp_engine_release_graphs) once its stream is idle. */
int64_t sp_engine_graph_count(void);
/* Destroy only the cached graphs of the calling thread's current device
 * (none of them may be running: synchronise that device first). */
int sp_engine_release_device_graphs(void);
/* Kernel launches enqueued by the calling thread's last sp_engine_run
 * (kernels inside a launched graph count individually). */
int64_t sp_engine_last_launches(void);

/* Same as sp_engine_run, but allocating nothing: for callers that cannot call
 * cudaMalloc (a host framework that owns every device allocation, a plugin
 * with no access to an allocator, or code that must not allocate once it is
 * running).  No counterpart in the reference, which allocates its buffers in
 * phasing.load.  Scratch comes from a 48 MiB array in device memory owned by
 * this library; a device reserves it when the library's device code is
 * loaded there -- at the latest on the first sp_engine_run_static call on
 * that device (lazy module loading, CUDA's default), at library load with
 * CUDA_MODULE_LOADING=EAGER -- and holds it until the process exits.
 * Requests needing more (sp_engine_workspace_size) fail with SP_ERR_SIZE.
 * Each call looks up the array's address in the current context (the first
 * lookup on a device may load the module); make the first call on each
 * device before any stream capture.  All calls share the array, so calls that
 * overlap on the GPU (other streams, other threads) race; nothing in it needs
 * to start at zero.  Launches are eager (opts->use_graph is ignored). */
int sp_engine_run_static(const sp_trial* trials, int n_trials, const sp_run_opts* opts,
                         sp_stream_t stream);

/* ---- operator API: one entry per reference OpenCL kernel --------------- */
/* (gpu.py:295 _kexec name lookup; n = number of elements) */
int sp_hio(float beta, const float* support_dev, const void* psi_in_dev, const void* psi_out_dev,
           void* output_dev, int64_t n, sp_stream_t stream);            /* phasing_hio.cl */
int sp_er(const float* support_dev, const void* psi_out_dev, void* output_dev, int64_t n,
          sp_stream_t stream);                                          /* phasing_er.cl */
int sp_raar(float beta, const float* support_dev, const void* psi_in_dev, const void* psi_out_dev,
            void* output_dev, int64_t n, sp_stream_t stream);           /* phasing_raar.cl */
int sp_sf(const float* support_dev, const void* psi_in_dev, const void* psi_out_dev,
          void* output_dev, int64_t n, sp_stream_t stream);             /* phasing_sf.cl */
int sp_dm1(float gamma_m, const float* support_dev, const void* psi_in_dev, void* output_dev,
           int64_t n, sp_stream_t stream);                              /* phasing_dm1.cl */
int sp_dm2(float beta, float gamma_s, const float* support_dev, const void* psi_in_dev,
           const void* psi_out_dev, const void* dm_tmp_dev, void* output_dev, int64_t n,
           sp_stream_t stream);                                         /* phasing_dm2.cl */
int sp_fourier(const void* psi_dev, const void* div_dev, const float* modulus_dev, void* out_dev,
               int64_t n, sp_stream_t stream);                          /* phasing_fourier.cl */
int sp_abs_f2_f2(const void* in_dev, void* out_dev, int64_t n, sp_stream_t stream); /* common_abs_f2_f2.cl */
int sp_copy_to_buffer_f2(void* dst_dev, const void* src_dev, int c0, int r0, int frame, int N,
                         int cols, int rows, sp_stream_t stream);       /* phasing_copy_to_buffer_f2.cl */
int sp_prtf_accumulate(int frames, const void* fft_dev, float* prtf_dev, int N,
                       sp_stream_t stream);                             /* phasing_prtf_accumulate2.cl */
/* 2-D complex FFT of `batch` N x N planes (pyfft Plan.execute, phasing.py:1074).
 * Forward is unnormalised; inverse scales by 1/N^2 (numpy ifft2 convention).
 * in == out is allowed. */
int sp_fft2(const void* in_dev, void* out_dev, int N, int batch, int inverse, sp_stream_t stream);

/* ---- post-processing --------------------------------------------------- */
/* align_global_phase (phasing.py:1355-1404): per frame, FP64 sums
 * A=sum re^2, B=sum re*im, C=sum im^2, D=sum re, F=sum im, then the closed-form
 * minimiser of sum|re sin p + im cos p|^2 with the sign rule, applied in place. */
int sp_align_global_phase(void* frames_dev, int n_frames, int64_t frame_elems,
                          double* angles_dev, double* sums_dev, sp_stream_t stream);
/* prtf (phasing.py:1406-1461): frames (n_frames, rows, cols) embedded at the
 * corner of N x N, |mean_n F_n/|F_n|| fftshifted into prtf_dev (N*N floats).
 * work_dev: complex64 n_frames*N*N scratch. */
int sp_prtf(const void* frames_dev, int n_frames, int rows, int cols, int N, void* work_dev,
            float* prtf_dev, sp_stream_t stream);
/* The two halves of sp_prtf, for PRTFs over frames spread across devices or
 * calls: sp_prtf_phasors adds sum_n F_n/|F_n| (unshifted, complex64 N*N) of its
 * frames into acc_dev; after the partial sums are added together,
 * sp_prtf_finish writes fftshift(|acc|/n_frames) with n_frames the total count. */
int sp_prtf_phasors(const void* frames_dev, int n_frames, int rows, int cols, int N, void* work_dev,
                    void* acc_dev, sp_stream_t stream);
int sp_prtf_finish(const void* acc_dev, int n_frames, int N, float* prtf_dev, sp_stream_t stream);
/* refine_support (phasing.py:1747-1815) on a rows x cols crop: |avg| is blurred
 * by the circular separable kernel kr (rows) x kc (cols) in FP64 (the FFT
 * convolution with the fftshifted, normalised Gaussian is exactly this
 * circular convolution), then
 *   refined = sum_parts (blur*part > max(blur*part)*local_t) * (blur > max(blur)*global_t)
 * where labels (int, rows*cols, 0 = outside, 1..n_labels = connected parts of
 * the support, masking.find_all_objects) define the parts.  kill_weakest drops
 * the part with the smallest sum of |avg| (host synchronises once).
 * work_dev: >= 8*rows*cols + 8*(n_labels+1) bytes.  blurred_dev: rows*cols
 * doubles; refined_dev: rows*cols floats; part_sums_dev: n_labels+1 doubles. */
int sp_shrinkwrap(const void* avg_dev, int rows, int cols, const double* kr_dev,
                  const double* kc_dev, const int* labels_dev, int n_labels, double local_t,
                  double global_t, int kill_weakest, void* work_dev, double* blurred_dev,
                  float* refined_dev, double* part_sums_dev, sp_stream_t stream);
/* Average of aligned frames (basic_phasing_example.py:43): out = mean over n. */
int sp_mean_frames(const void* frames_dev, int n_frames, int64_t frame_elems, void* out_dev,
                   sp_stream_t stream);
/* Integer alignment peak (conditioning.align_frames :316-430 with
 * crosscorr.alignment_coordinates :526-568): argmax over the fftshifted
 * |IFFT(FFT(a) conj(FFT(b)))| of two N x N planes (magnitudes first when
 * use_mag_only).  *best_dev receives (float bits of the peak << 32) |
 * (0xffffffff - shifted index); ties resolve to the first index.
 * work_dev: complex64 2*N*N. */
int sp_xcorr_peak(const void* a_dev, const void* b_dev, int N, int use_mag_only, void* work_dev,
                  unsigned long long* best_dev, sp_stream_t stream);
/* np.roll(np.roll(in, dr, 0), dc, 1) of one rows x cols complex frame; in != out. */
int sp_roll(const void* in_dev, void* out_dev, int rows, int cols, int dr, int dc,
            sp_stream_t stream);
/* center_of_mass_average (phasing.py:1710-1745): FP64 sums (sum|f|,
 * sum r|f|, sum c|f|) per frame into sums_dev (3*n_frames doubles) ... */
int sp_com_sums(const void* frames_dev, int n_frames, int rows, int cols, double* sums_dev,
                sp_stream_t stream);
/* ... then out = sum_n roll(frame_n, -shift_n) with shifts_dev = (dr, dc) per frame. */
int sp_roll_accumulate(const void* frames_dev, int n_frames, int rows, int cols,
                       const int* shifts_dev, void* out_dev, sp_stream_t stream);

/* Subpixel registration and alignment of frames to a reference (the batched
 * workload's "align to trial 0, then average"; the reference itself aligns
 * by whole pixels only: conditioning.align_frames :316-430 with
 * crosscorr.alignment_coordinates :526-568, whose correlation convention and
 * whole-pixel answers this keeps).  Frames (n_frames, rows, cols) and the
 * reference (rows, cols) are embedded at the corner of N x N (N a power of
 * two >= rows, cols); the cross-correlation peak is refined by the
 * upsampled DFT of Guizar-Sicairos, Thurman & Fienup (Opt. Lett. 33, 2008) to
 * 1/upsample pixel (1..170).  shifts_dev receives (dy, dx, theta) per frame
 * (3 doubles): frame_f(y + d) exp(-i theta) lines up with the reference.  If
 * out_dev is not NULL it receives those aligned frames (Fourier-shifted,
 * cropped to rows x cols; may equal frames_dev).  work_dev:
 * sp_register_workspace_size bytes. */
int sp_register_workspace_size(int n_frames, int N, int upsample, size_t* bytes);
int sp_register_subpixel(const void* frames_dev, int n_frames, int rows, int cols,
                         const void* ref_dev, int N, int upsample, void* work_dev,
                         size_t work_bytes, double* shifts_dev, void* out_dev, sp_stream_t stream);

/* Polar unwrap of an N x N float map and its row means: the prtfq / rftfq
 * azimuthal averages (phasing.py:1454-1458, :1512-1516, :1603-1605,
 * :1701-1705), which call wrapping.unwrap(map, (0, N/2, (N/2, N/2)))
 * (wrapping.py:8-67 unwrap_plan, :131-176 unwrap) and np.average(axis=1).
 * Samples radii r_in .. r_out-1 about (cy, cx) at `columns` angles
 * 2 pi k / columns (columns <= 0: int(2 pi r_out)), each by cubic B-spline
 * interpolation in FP64 (scipy.ndimage.map_coordinates order 3: mirror-
 * boundary prefilter) rounded to float; every sample must lie inside the map
 * (SP_ERR_INVALID otherwise).  unwrapped_dev ((r_out - r_in) x columns
 * floats) and mean_dev (r_out - r_in floats) may each be NULL, not both.
 * work_dev: N*N doubles. */
int sp_unwrap(const float* in_dev, int N, int r_in, int r_out, double cy, double cx, int columns,
              double* work_dev, float* unwrapped_dev, float* mean_dev, sp_stream_t stream);

/* ---- trial quality: RFTF, hot pixels, pair-wise covariances ------------- */
/* (|x|^2, 0)  -- kernels/common_abs2_f2_f2.cl */
int sp_abs2_f2_f2(const void* in_dev, void* out_dev, int64_t n, sp_stream_t stream);
/* principal complex square root  -- kernels/common_sqrt_f2.cl */
int sp_sqrt_f2(const void* in_dev, void* out_dev, int64_t n, sp_stream_t stream);
/* (sqrt(|x|), 0): the CPU rftf's blurred modulus (phasing.py:1577) */
int sp_sqrt_abs_f2(const void* in_dev, void* out_dev, int64_t n, sp_stream_t stream);
/* out[f] = in1 * in2[f], in1 real  -- kernels/common_multiply_axis_f_f2.cl */
int sp_multiply_axis_f_f2(int frames, const float* in1_dev, const void* in2_dev, void* out_dev,
                          int64_t plane, sp_stream_t stream);
/* out = a * b, complex  -- kernels/common_multiply_f2_f2.cl */
int sp_multiply_f2_f2(const void* a_dev, const void* b_dev, void* out_dev, int64_t n,
                      sp_stream_t stream);
/* gpu_rftf's accumulation (phasing.py:1611-1708, kernels/phasing_rftf_accumulate.cl):
 * acc = mean over frames of 1/sqrt(1 + (g - Re F)^2/g^2), written fftshifted if shift. */
int sp_rftf_accumulate(int frames, const float* goal_dev, float* accumulation_dev,
                       const void* fourier_dev, int N, int shift, sp_stream_t stream);
/* rftf's error map for one estimate (phasing.py:1583-1601): picks the goal's centring from
 * the FP64 sums |F - g| and |shift(F) - g| (sums_dev: 2 doubles, read back), writes the
 * centred error err_dev and out_dev = sqrt(1/(1+err)) (rescaled to [0,1] if scale). */
int sp_rftf_map(const void* fourier_dev, const float* goal_dev, int N, int scale, double* sums_dev,
                float* err_dev, float* out_dev, sp_stream_t stream);
/* out = sqrt(1/(1+err)), rescaled if scale (phasing.py:1597-1601) */
int sp_rftf_from_error(const float* err_dev, float* out_dev, int64_t n, int scale,
                       sp_stream_t stream);
/* conditioning.remove_hot_pixels, CPU branch (conditioning.py:304-305): per frame and
 * iteration, median = medfilt 3x3 (zero padding) + 0.1; data = median where
 * data/median > threshold.  work_dev: rows*cols floats. */
int sp_remove_hot_pixels(float* data_dev, float* work_dev, int frames, int rows, int cols,
                         int iterations, float threshold, sp_stream_t stream);
/* covar_results (phasing.py:1817-1982): cc[p] = max |IFFT2(conj(D_a) D_b)| for each pair
 * p = (a, b) of pairs_dev (int32 pairs) of transformed frames dfts_dev (N*N complex64 each);
 * work_dev holds work_planes N*N complex64 planes, pairs are done that many at a time. */
int sp_covar_pairs(const void* dfts_dev, int N, const int32_t* pairs_dev, int n_pairs,
                   void* work_dev, int work_planes, float* cc_dev, sp_stream_t stream);

/* ---- coherence estimation (phasing.optimize_coherence, phasing.py:507-930) */
/* out = in1 / in2, complex  -- kernels/common_divide_f2_f2.cl */
int sp_divide_f2_f2(const void* in1_dev, const void* in2_dev, void* out_dev, int64_t n,
                    sp_stream_t stream);
/* out[N-1-i][N-1-j] = in[i][j] for each of `planes` N*N planes (in != out)
 * -- kernels/common_flip_f2.cl */
int sp_flip_f2(const void* in_dev, void* out_dev, int N, int planes, sp_stream_t stream);
/* exp(-i^2/(2 sx^2)) exp(-j^2/(2 sy^2)) in corner-centred coordinates, N*N floats, or
 * complex64 with zero imaginary part if complex_out  -- kernels/common_gaussian_f.cl */
int sp_gaussian(void* out_dev, int N, float sx, float sy, int complex_out, sp_stream_t stream);
/* `iterations` Richardson-Lucy steps for `frames` estimates u at once (_opt_iter_rl,
 * phasing.py:702-738): blur = IFFT(FFT(u) p_hat); blur = d / blur; blur = IFFT(FFT(blur)
 * ph_hat); u *= blur.  p_hat, ph_hat, u, work: frames*N*N complex64; d: N*N complex64. */
int sp_richardson_lucy(void* u_dev, const void* p_hat_dev, const void* ph_hat_dev, const void* d_dev,
                       void* work_dev, int N, int frames, int iterations, sp_stream_t stream);
/* the Gaussian fit's objective (_opt_iter_g, phasing.py:663-700): *sum_dev (FP64) =
 * sum (sqrt|FFT2(gaussian(sx, sy) * ac)| - modulus)^2; work_dev: N*N complex64. */
int sp_coherence_misfit(const void* ac_dev, const float* modulus_dev, float sx, float sy, int N,
                        void* work_dev, double* sum_dev, sp_stream_t stream);

/* ---- plain single-instance path (the reference's GPU dataflow) --------- */
/* One trial, cuFFT C2C plans plus one elementwise kernel per step with a
 * stream synchronisation after each, as phasing.py:1187-1353 drives pyfft and
 * its kernels (gpu.py:349 `.wait()`).  The baseline the fused engine is
 * measured against.  work_dev: complex64 4*N*N scratch.  Unlike every other
 * entry point, the cuFFT plan it creates allocates its own work area. */
int sp_plain_iterate(int N, int n_iter, int n_runs, const int32_t* run_alg, const int32_t* run_count,
                     float beta, void* psi_dev, const float* modulus_dev, const float* support_dev,
                     void* work_dev, sp_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* SPECKLE_B200_H */
