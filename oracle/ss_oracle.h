/* FP64 CPU oracle for align_group_to_template: TEST INFRASTRUCTURE ONLY.
 *
 * This is a sequential restatement of the reference's motion estimator (setup/source/task/,
 * setup/source/interface/parameterorganizer/, setup/source/task/filter/, setup/source/task/task.cpp,
 * setup/source/task/mainiteration/mainiteration.cpp) used as the checker for the CUDA path. Nothing in
 * the product links it; only tests, smoke() and the benchmark's CPU-baseline arm load it.
 *
 * Matrices are passed in the reference's internal row-major layout (NeutralMatrix RowMajor,
 * setup/source/interface/memory.h:64-83): element (r, c) of an R x C matrix at r*C + c.
 */
#ifndef SS_ORACLE_H_
#define SS_ORACLE_H_

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const char* flags;              /* precision letter + gpu_flags (configuration.cpp:83-152) */
    int templ_h, templ_w;
    const double* templ;            /* templ_h x templ_w */
    const double* xgrad;            /* templ_h x templ_w */
    const double* ygrad;            /* templ_h x templ_w */
    int frame_h, frame_w, n_frames; /* Hb, W, nF */
    const double* frac;             /* frame_h x frame_w */
    const double* basex;            /* frame_h x frame_w, 0-based template x */
    const double* basey;            /* frame_h x frame_w */
    const unsigned char* base_mask; /* frame_h x frame_w */
    const double* image;            /* frame_h x (frame_w * n_frames) */
    const double* est_dx;           /* (frame_w + 1) * n_frames, frame-contiguous */
    const double* est_dy;
    const int* min_points;          /* >= frame_w entries */
    int group_size;
    int max_iter;
    double move_thresh;
    double halt_corr;
    double corr_inc_thresh;
    double filter_strength;
    int max_filter_iter;
    double filter_corr_thresh;
    double lambda;                  /* knot-difference regulariser weight (0 = reference) */
    double ls_mult;
    int solver_id;                  /* 0 ILU(0), 1 and 2 exact (LDL^T) */
    int filter_id;                  /* 0 none, 1 smearing, 2 range */
    int n_threads;                  /* OpenMP threads for the per-column loops (<=0: default) */
} sso_in;

typedef struct {
    double* p_last;          /* 2N raw knot chain returned (task.cpp:207) */
    double* dx_knots;        /* (W+1)*nF per-frame knots, organize1D2 (parameterorganizer.cpp:79-98) */
    double* dy_knots;
    double* frame_corr;      /* nF */
    double* residrms;        /* nF */
    unsigned char* mask;     /* frame_h x (W*nF) row-major, may be NULL */
    double* iter_corr;       /* max_iter, may be NULL (flag C) */
    double* frame_corr_hist; /* max_iter x nF row-major, may be NULL (flag c) */
    double* iter_errvals;    /* 2*max_iter x nF row-major, may be NULL (flag e) */
    double* all_params;      /* 2N x max_iter column-major, may be NULL */
    long long* n_eval;       /* nF: frame evaluations (assembly passes + line-search trials) */
    int iterations;
    int stop_reason;         /* StopCriterion (stopcriterion.h:4-10) */
    int ls_trial_cap_hit;    /* a line search ran into the trial cap */
    double* rg_params;       /* flag t: 2N chain after every half-step, 2*max_iter slots row-major, may be NULL */
} sso_out;

/* Runs one align_group_to_template call. Returns 0 on success, <0 on invalid arguments. */
int sso_align_group(const sso_in* in, sso_out* out);

/* Pieces exposed for unit tests against the reference's own host-compiled functions. */
void sso_organize2d1(const double* px, const double* py, double* p, int n_frames, int frame_w);
void sso_organize1d2(const double* p, double* px, double* py, int n_frames, int frame_w);
void sso_smearing_filter(double* v, int n, double strength);
void sso_range_filter(double* v, int n, double strength);
/* Block LDL^T solve of a symmetric block-tridiagonal system with 2x2 blocks: d is n x 3 diagonal
 * blocks (xx, yy, xy), c is (n-1) x 4 coupling blocks [[c0, c2], [c3, c1]] between block i (rows)
 * and i+1 (cols), b and x are n x 2. */
int sso_block_tridiag_solve(int n, const double* d, const double* c, const double* b, double* x);

#ifdef __cplusplus
}
#endif
#endif
