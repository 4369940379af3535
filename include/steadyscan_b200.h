/* steadyscan_b200: B200-native align_group_to_template behind a plain C ABI.
 *
 * The entry points below replace the reference's MATLAB MEX function
 *   void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[])
 * (setup/source/mex/align_group_to_template.cpp:21-85), whose 26 inputs are converted in
 * setup/source/mex/mexgateway.cpp:31-255 and whose outputs are produced in mexgateway.cpp:261-370.
 * The arguments keep the MEX order, names and meaning; matrices keep MATLAB's column-major layout.
 * No torch or CUDA types appear in the signatures. Errors are returned as status codes (the
 * reference aborts the MATLAB call through mexErrMsgIdAndTxt, mex/reporter/reporter.cpp:25-27);
 * ss_last_error() gives the message of the calling thread's last failure.
 */
#ifndef STEADYSCAN_B200_H_
#define STEADYSCAN_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS_ABI_VERSION 6

#if defined(__GNUC__)
#define SS_API __attribute__((visibility("default")))
#else
#define SS_API
#endif

/* Element types of an ss_matrix. */
enum ss_dtype {
  SS_F64 = 0, /* double */
  SS_F32 = 1, /* float */
  SS_U16 = 2, /* uint16 photon counts (frame storage) */
  SS_F16 = 3, /* IEEE half (frame or template storage) */
  SS_U8 = 4,  /* logical / uint8 */
  SS_I32 = 5  /* int32 */
};

/* Where an ss_matrix's data lives. */
enum ss_location {
  SS_HOST = 0,  /* host memory; copied to the device inside the call */
  SS_DEVICE = 1 /* device memory of gpu_device_id; used in place */
};

/* Status codes. */
enum ss_status {
  SS_OK = 0,
  SS_ERR_INVALID_ARGUMENT = -1, /* GPUMC:InvalidArgument / NotEnoughInputs (mex/reporter/reporter.cpp:3-12) */
  SS_ERR_CUDA = -2,             /* GPUMC:CudaError */
  SS_ERR_OUT_OF_MEMORY = -3,    /* device allocation failed (task.cpp:116-131) */
  SS_ERR_NO_DEVICE = -4,
  SS_ERR_BUSY = -5,             /* serving: admission refused (memory budget or queue) */
  SS_ERR_NOT_FOUND = -6         /* serving: unknown session or request */
};

/* A matrix argument, MATLAB layout: element (i, j) at data[i + j * rows]. */
typedef struct ss_matrix {
  const void* data;
  int64_t rows;
  int64_t cols;
  int32_t dtype;    /* enum ss_dtype */
  int32_t location; /* enum ss_location */
} ss_matrix;

/* The 26 inputs of align_group_to_template, in MEX order (mexgateway.cpp:38-174;
 * caller steady_scan.m:239-242). Index comments give the prhs[] slot. */
typedef struct ss_inputs {
  const char* flags;              /*  0: precision letter 'D' or 'S' + gpu_flags (configuration.cpp:83-152) */
  ss_matrix template_image;       /*  1: Ht x Wt */
  ss_matrix xgrad;                /*  2: Ht x Wt, forward difference along x, NaN last column */
  ss_matrix ygrad;                /*  3: Ht x Wt, forward difference along y, NaN last row */
  ss_matrix tfrac;                /*  4: Hb x W, scan-time fraction between knots */
  ss_matrix basex;                /*  5: Hb x W, 0-based template x of each undisplaced pixel */
  ss_matrix basey;                /*  6: Hb x W */
  ss_matrix base_mask;            /*  7: Hb x W logical */
  ss_matrix bm_data;              /*  8: Hb x (W * n_frames) frames in block-matrix order */
  ss_matrix est_dx_knots;         /*  9: (W+1) x n_frames initial x knots */
  ss_matrix est_dy_knots;         /* 10: (W+1) x n_frames initial y knots */
  int32_t group_size;             /* 11: W * gpu_frame_groupsize; a positive multiple of W */
  int32_t n_frames;               /* 12 */
  ss_matrix min_points_per_block; /* 13: >= W entries (int32 or double, truncated) */
  int32_t max_iter;               /* 14 */
  double move_thresh;             /* 15 */
  double halt_correlation;        /* 16 */
  double correlation_increase_threshold; /* 17 */
  double filter_strength;         /* 18 */
  int32_t max_filter_iterations;  /* 19 */
  double filter_deactivation_threshold; /* 20 */
  double lambda;                  /* 21: knot-difference regulariser weight (the reference ignores it; 0 = reference) */
  double linesearch_reduction_multiplier; /* 22 */
  int32_t solver_id;              /* 23: 0 ILU(0) in x|y order, 1 and 2 exact (2 keeps SolverEigen's matrix between solves) */
  int32_t filter_id;              /* 24: 0 none, 1 smearing, 2 range */
  int32_t gpu_device_id;          /* 25 */
  /* Extension: storage type of template samples on the device for precision 'S'
   * (SS_F32 default, or SS_F16). Precision 'D' always keeps FP64. */
  int32_t template_storage;
  /* Extension (a tuning choice, no effect on precision D results): frames per evaluation tile,
   * 1..64; 0 splits the group's frames into even chunks of at most 32. */
  int32_t frames_per_cta;
} ss_inputs;

/* Outputs; every pointer may be NULL (that output is then not produced). Host memory. Index
 * comments give the plhs[] slot (mexgateway.cpp:266-354). */
typedef struct ss_outputs {
  double* dx_knots;           /* 1: (W+1) * n_frames, per-frame knots (last repeats knot W-1) */
  double* dy_knots;           /* 2 */
  double* frame_corr;         /* 3: n_frames */
  int32_t* iter_used;         /* 4: scalar */
  uint8_t* mask;              /* 5: Hb x (W * n_frames) logical, column-major */
  double* residrms;           /* 6: n_frames */
  double* device_init_time;   /* 7: seconds */
  double* iteration_corr;     /* 8: max_iter (flag C) */
  double* frame_corr_history; /* 11: n_frames x max_iter column-major (flag c) */
  double* iteration_errvals;  /* 12: (2 * max_iter) x n_frames column-major (flag e) */
  double* raw_params;         /* 13: 2N chain (flag P) */
  double* all_params;         /* 15: 2N x max_iter column-major */
  double* frame_params;       /* flag p: n_frames x 2(W+1) column-major */
  int32_t stop_reason;        /* StopCriterion (interface/stopcriterion.h:4-10) */
  int32_t trial_cap_hit;      /* a line search hit its trial bound (the reference loops without one) */
  int64_t n_frame_passes;     /* frame evaluations read from memory (assembly, trials, correlation, final) */
  double elapsed_ms;          /* wall time of the call */
  uint8_t* blocks_used;       /* W x n_frames column-major: the block has a valid pixel in the final
                                 mask (output 5), the caller's blocksused (steady_scan.m:264-265) */
  /* Timing and half-step outputs (mexgateway.cpp:266-300; filled with zeros where the flags do not
   * produce them). Flag t also switches the iteration to the reference's TimedMainIteration
   * (task.cpp:99-103), whose bookkeeping differs (timedmainiteration.cpp:45-143): paramsUsed is
   * cleared before every half-step, filterID follows other rules, a retry counts as the next
   * iteration for output 14. */
  double* iteration_times;    /* 9: max_iter seconds per iteration (flags T and t; device clock) */
  double* function_times;     /* 10: 14 seconds per sub-function (flag t; CUDA events over the batch,
                                 whose stages the run's groups share; flag t runs host-launched
                                 cycles): 1 applyParameters with the errval, gradient and system sums
                                 of the same pass, 2 group errvals and parameter mask, 4 compaction,
                                 5 system blocks, 7 solve and filter, 8 expansion, 9 line search,
                                 10 correlation, 11 iteration end; 0, 3, 6, 12 and 13 stay zero */
  double* rg_params;          /* 14: 2N x (2 max_iter) column-major: the chain after every half-step
                                 (flag t; slot shift + 2 (iteration - 1)) */
} ss_outputs;

/* align_group_to_template: one group of frames (replaces mexFunction,
 * mex/align_group_to_template.cpp:21-85, and MexGateway<T>::execute, mexgateway.cpp:372-445). */
SS_API int ss_align_group_to_template(const ss_inputs* in, ss_outputs* out);

/* Many independent groups in one batched run on one GPU (the MATLAB driver's per-set loop,
 * steady_scan.m:216-287, done concurrently). in[i] and out[i] describe group i; all groups must
 * use the same precision letter, frame dtype and device. */
SS_API int ss_align_groups(int32_t n_groups, const ss_inputs* in, ss_outputs* out);

/* A prepared batch: inputs validated and resident on the device, reusable for repeated runs
 * (each run starts every group from its initial knots). ss_align_groups is create + run +
 * collect + destroy. Run statistics come back in ss_batch_stats. */
typedef struct ss_batch ss_batch;

typedef struct ss_batch_stats {
  int32_t n_groups;
  int32_t cycles;             /* half-step cycles of the last run */
  int32_t linesearch_rounds;  /* trial rounds of the last run */
  int32_t kernel_launches;    /* kernels launched by the last run */
  int64_t frame_passes[4];    /* frames evaluated per pass kind: assembly, trial, correlation, final */
  double eval_ms[4];          /* device time of the evaluation kernels per pass kind (timing on) */
  int64_t arena_bytes;        /* device memory held by the batch */
  double run_ms;              /* wall time of the last run */
  /* shared-memory staging of the last run: assembly/final CTAs, of them with a template row window,
   * line-search CTAs, of them with a window, of them on the packed pixel-pair path, and assembly
   * block columns evaluated as pixel pairs */
  int64_t staging[6];
  /* frame block columns of the last run's assembly passes whose knots were those of their previous
   * assembly, so they kept its sums and read no frame data */
  int64_t assembly_columns_kept;
} ss_batch_stats;

SS_API int ss_batch_create(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_batch** batch);
SS_API int ss_batch_run(ss_batch* batch);
SS_API int ss_batch_collect(ss_batch* batch);
/* 1 turns on CUDA-event timing of the evaluation kernels for later runs (adds events to the stream). */
SS_API int ss_batch_set_timing(ss_batch* batch, int32_t on);
/* 1 (the default) runs a batch as one CUDA graph: device-side loops over cycles and line-search trial
 * rounds, launched once per ss_batch_run / ss_batch_step, with no host round trip until every group
 * has stopped (ss_batch_poll then returns 2). 0 launches one cycle per ss_batch_step from the host.
 * Timing (ss_batch_set_timing) always runs host-launched cycles. Results are the same either way. */
SS_API int ss_batch_set_graph(ss_batch* batch, int32_t on);
SS_API int ss_batch_stats_get(const ss_batch* batch, ss_batch_stats* stats);
/* The cudaStream_t the batch launches on, as an opaque pointer (for the caller's own events). */
SS_API void* ss_batch_stream(const ss_batch* batch);
SS_API void ss_batch_destroy(ss_batch* batch);

/* Serving support (no counterpart in the reference, which aligns one group per MEX call).
 *
 * A session keeps one imaging session's template, gradients and scan geometry (the ss_inputs
 * fields 1-7 and 13 of `proto`, with its precision and template_storage) resident on the device,
 * converted once. Groups of a batch made with ss_batch_create_ex, or admitted to a server, may name
 * a session; they then use its buffers and their own fields 1-7 and 13 only give the shapes, which
 * must match. A session must outlive every batch or server group that uses it. */
typedef struct ss_session ss_session;
SS_API int ss_session_create(const ss_inputs* proto, ss_session** session);
SS_API void ss_session_destroy(ss_session* session);

/* Device bytes the batch of these groups needs (no device work, nothing allocated). */
SS_API int ss_batch_measure(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_session* const* sessions,
                            int64_t* arena_bytes);
/* ss_batch_create with per-group sessions (array of n_groups entries, NULL entries or a NULL array
 * for none) and, when arena is not NULL, the caller's device memory of arena_bytes (at least what
 * ss_batch_measure returned) instead of an allocation of its own. */
SS_API int ss_batch_create_ex(int32_t n_groups, const ss_inputs* in, ss_outputs* out, ss_session* const* sessions,
                              void* arena, int64_t arena_bytes, ss_batch** batch);
/* ss_batch_run without blocking: ss_batch_start resets every group to its initial knots
 * (asynchronous); ss_batch_step launches the run: the whole run as one CUDA graph (the default,
 * see ss_batch_set_graph), else one cycle of every group (assembly, solve, line search, iteration
 * control); ss_batch_poll returns 0 while that launch runs, 1 when a host-launched cycle has
 * finished and the next ss_batch_step is due, 2 when every group has stopped (then
 * ss_batch_collect), or an error. */
SS_API int ss_batch_start(ss_batch* batch);
SS_API int ss_batch_step(ss_batch* batch);
SS_API int ss_batch_poll(ss_batch* batch);

/* Continuous batching: a server holds `capacity` group slots on one stream and serves every
 * active group with one launch sequence per cycle. ss_server_admit prepares a group in a free slot
 * (its buffers in the caller's arena of arena_bytes from ss_batch_measure, or an allocation of its
 * own when arena is NULL; its template and geometry from `session` when not NULL; outputs to `out`
 * when it stops) and returns the slot; it joins at the next ss_server_step, which launches one
 * cycle of every active group. ss_server_poll returns 0 while that cycle runs; else it collects the
 * outputs of the groups that stopped, lists their slots in done_slots (up to max_done; call again
 * for more) and returns 1: those slots and their arenas are free. Groups may be admitted while a
 * cycle runs. Every group's results are those it gets alone. */
typedef struct ss_server ss_server;
SS_API int ss_server_create(int32_t capacity, int32_t device, ss_server** server);
SS_API int ss_server_admit(ss_server* server, const ss_inputs* in, ss_outputs* out, ss_session* session, void* arena,
                           int64_t arena_bytes, int32_t* slot);
SS_API int ss_server_step(ss_server* server);
SS_API int ss_server_poll(ss_server* server, int32_t* done_slots, int32_t max_done, int32_t* n_done);
SS_API int32_t ss_server_active(const ss_server* server);
SS_API void ss_server_destroy(ss_server* server);

/* The FP64 knot-chain solve of one half-step on its own: the symmetric positive definite
 * block-tridiagonal normal equations (2x2 blocks, one per used knot) that the reference assembles
 * in task_filldiagonals.cu:47-159 and task_filljtr.cu:3-58 and hands to its sparse solvers
 * (eigensolve.cpp:35-38, cusolversolver.cu:53-56), solved by block cyclic reduction on the
 * device. All pointers are device memory of the current device: diag n x 3 (xx, yy, xy), coupling
 * (n-1) x 4 ([[c0 c2] [c3 c1]] between block i and block i+1), rhs and x n x 2, row-major.
 * stream is a cudaStream_t (NULL: the legacy default stream); the call returns after the solve.
 * The workspace (104 bytes per block) is allocated and freed inside the call. */
SS_API int ss_solve_block_tridiagonal(int32_t n, const double* diag, const double* coupling, const double* rhs,
                                      double* x, void* stream);

/* ss_solve_block_tridiagonal without any device allocation; it has no counterpart in the
 * reference. It is for callers that cannot allocate GPU memory while they run: an acquisition loop
 * that aligns frames while the microscope streams, where cudaMalloc and cudaFree synchronize the
 * device and stall the frames in flight, or a host application whose own allocator has already
 * reserved the GPU's memory. The caller passes the same device buffers as to
 * ss_solve_block_tridiagonal; the workspace is a fixed device array inside this library of
 * 32768 blocks (3.4 MB, held by every GPU that loads the library until the process exits), so
 * n > 32768 is rejected with SS_ERR_INVALID_ARGUMENT. The first call on a device looks up that
 * array's device address and sets the solve kernel's shared-memory attribute (again after the
 * device's context has been reset, e.g. by cudaDeviceReset). Each call waits for `stream`
 * (cudaStreamSynchronize) before it returns. All calls
 * share the one array per device: calls that overlap on the GPU (different streams or threads at
 * the same time) race and corrupt each other's results; serialize them. Each call writes every part
 * of the workspace it reads before reading it. */
SS_API int ss_solve_block_tridiagonal_noalloc(int32_t n, const double* diag, const double* coupling,
                                              const double* rhs, double* x, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Recording-level estimate: the caller loop of the reference's MATLAB driver
 * (estimate_displacements, steady_scan.m:157-288, with the set split of steady_scan.m:97-108),
 * run as one batch on the GPU with its post-estimate validity rules applied on the device.
 *
 * The recording's frames are split into sets of at most frames_per_set frames; every set except
 * the last is extended by the first frame of the next set, and that overlap frame's estimate is
 * discarded (steady_scan.m:216-244, "last frame of set is estimated incorrectly"), so the last
 * frame of the recording is never estimated: its outputs stay NaN. Per kept frame, from the set's
 * final mask: blocks_used (a valid pixel in the block, steady_scan.m:265); no block used ->
 * failed, corr NaN (:269-273); otherwise the knots before the first and after the last used block
 * repeat those blocks' knots (extend_firstandlast, :277-281, :615-623) and
 * failed = !(corr >= corr_thresh) || nknots-1 / (nknots-1) < minblockfrac (:283; the reference
 * divides numel(blocksused), i.e. the block count, not the used count).
 *
 * As in the reference every set is started from the first columns of est_dx_knots / est_dy_knots
 * (the driver passes the whole matrix to each set's MEX call, steady_scan.m:239-240, and
 * ParameterOrganizer::organize2D1 reads the first n_set_frames columns); per_set_estimates = 1
 * starts each set from its own frames' columns instead (extension).
 */
typedef struct ss_recording {
  ss_inputs group;             /* settings, template and geometry; bm_data holds every frame of the
                                  recording (Hb x (W * n_frames)), n_frames their count, est_dx/dy
                                  (W+1) x n_frames (or (W+1) x k with k >= the largest set) */
  int32_t frames_per_set;      /* settings.frames_per_set (default 500) */
  int32_t min_frames_per_set;  /* settings.min_frames_per_set (default 100; see ss_recording_sets) */
  double corr_thresh;          /* settings.corr_thresh (default 0.75) */
  double minblockfrac;         /* settings.minblockfrac (default 0.25) */
  int32_t per_set_estimates;   /* 0: the reference's start (first columns), 1: each set's own */
} ss_recording;

/* Outputs of ss_estimate_displacements (host memory; NULL pointers are not produced). */
typedef struct ss_recording_outputs {
  double* dx_knots;    /* (W+1) x n_frames column-major (steady_scan.m:1 dx_knots) */
  double* dy_knots;
  double* corr;        /* n_frames */
  double* iter_used;   /* n_frames (the set's iteration count; NaN where not estimated) */
  double* residrms;    /* n_frames */
  uint8_t* failed;     /* n_frames */
  uint8_t* blocks_used; /* W x n_frames column-major */
  int32_t n_sets;      /* sets the recording was split into */
} ss_recording_outputs;

SS_API int ss_estimate_displacements(const ss_recording* rec, ss_recording_outputs* out);

/* The set split of steady_scan.m:97-108 as used by estimate_displacements (:216-220): set s covers
 * frames first[s] .. first[s] + count[s] - 1 (0-based, the overlap frame included). The driver
 * also rebalances the sizes of the last two sets when the last holds fewer than
 * min_frames_per_set frames, but the estimate loop reads the unchanged set starts, so that
 * rebalancing moves no frame (reproduced here). No device work. Returns the number of sets in
 * *n_sets and fills at most max_sets entries. */
SS_API int ss_recording_sets(int32_t n_frames, int32_t frames_per_set, int32_t min_frames_per_set, int32_t* first,
                             int32_t* count, int32_t max_sets, int32_t* n_sets);

/* ---------------------------------------------------------------------------------------------
 * Caller-side preparation of frames on the GPU: what the reference's MATLAB driver does to the raw
 * frames of a set before its MEX call (steady_scan.m:229-234): prefilter_foralignment
 * (:625-643), cropimage (:830-834) and image2blockmatrix (:601-613) of every frame.
 *
 * prefilter_foralignment: with pregauss > 0 each frame is blurred by the reference's periodic FFT
 * convolution with a Gaussian of that standard deviation on the frame padded by
 * L = ceil(sqrt(2 pregauss^2 log(10000 / (sqrt(2 pi) pregauss)))) zero rows and columns; with
 * mednorm != 0 each (blurred) frame is then divided by the median of its samples. Both are applied
 * to the whole frame before cropping, as in the reference. The blur needs pregauss < 3989 (the
 * reference's L is not real above that).
 *
 * gather: the caller's block map (host memory), block_h x n_blocks column-major: for entry (r, b)
 * the 0-based column-major index of the cropped frame's pixel there, -1 where the block has fewer
 * pixels (the positions of settings.prevknotind == b + 1 in column-major order, steady_scan.m:609).
 * out: block_h x (n_blocks * n_frames) in device memory, SS_F64, SS_F32 or SS_U16 (SS_U16 only for
 * SS_U16 frames without prefilter, whose samples it copies exactly). Synchronous; allocates work
 * memory for the prefilter. */
typedef struct ss_prep_frames {
  ss_matrix frames;      /* H x (W * n_frames) column-major (frame k in columns k W .. k W + W - 1),
                            host or device, any ss_dtype */
  int32_t n_frames;
  double pregauss;       /* settings.pregauss (0: no blur) */
  int32_t mednorm;       /* settings.mednorm */
  int32_t cropping[4];   /* settings.cropping: [left right bottom top] pixels removed */
  const int32_t* gather; /* block_h x n_blocks column-major, host memory */
  int32_t block_h, n_blocks;
  ss_matrix out;         /* device memory, block_h x (n_blocks * n_frames) */
  int32_t gpu_device_id;
} ss_prep_frames;

SS_API int ss_prepare_frames(const ss_prep_frames* p);

/* ---------------------------------------------------------------------------------------------
 * Reconstruction on the GPU: invert_bilinear_sampling of the reference's MATLAB driver
 * (steady_scan.m:290-404) for the frames of one set, i.e. one call of it (steady_scan.m:128-135).
 * Every frame is reconstructed on the template grid from its knots as the least-squares inverse of
 * its bilinear sampling with the adjacent-difference regulariser (ibs_regfac; vertical differences
 * weighted by 1 / ibs_template_pixel_aspect_ratio), by the reference's 4-colour Gauss-Seidel
 * iteration from its push-grid first guess, stopped when the energy stops decreasing at the
 * reference's check interval, which is carried from frame to frame within the call. Pixels the
 * frame does not constrain are NaN in the output and false in the mask. The reference's optional
 * least-squares gap filling (ibs_inpaint, default off) is not done. Synchronous.
 *
 * Extra channels (steady_scan.m:137-154) are the same call with the channel's frames and the same
 * knots. */
typedef struct ss_reconstruct {
  ss_matrix frames;       /* h x (w * n_frames): the set's cropped (and prefiltered) frames, FP32 or
                             FP64, host or device */
  int32_t n_frames;
  ss_matrix basex;        /* h x w: settings.basex (1-based template x of each pixel), FP64 */
  ss_matrix basey;        /* h x w: settings.basey, FP64 */
  ss_matrix tfrac;        /* h x w: settings.tfrac, FP64 */
  ss_matrix prevknotind;  /* h x w: settings.prevknotind (1-based), SS_I32 or FP64 */
  ss_matrix dx_knots;     /* nknots x n_frames, FP64 (host) */
  ss_matrix dy_knots;
  int32_t template_h, template_w;  /* corrected_data_size = size(template_image) */
  double regfac;          /* settings.ibs_regfac (default 3e-3) */
  double pixel_aspect_ratio;  /* settings.ibs_template_pixel_aspect_ratio (default 1) */
  ss_matrix out;          /* template_h x (template_w * n_frames), FP32 or FP64, host or device */
  uint8_t* mask;          /* template_h x (template_w * n_frames) host, or NULL */
  int32_t* iterations;    /* n_frames host, or NULL: Gauss-Seidel sweeps of each frame (0: skipped) */
  int32_t gpu_device_id;
} ss_reconstruct;

SS_API int ss_reconstruct_frames(const ss_reconstruct* r);

/* Message of the calling thread's last error ("" if none). */
SS_API const char* ss_last_error(void);

/* SS_ABI_VERSION of the loaded library. */
SS_API int32_t ss_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* STEADYSCAN_B200_H_ */
