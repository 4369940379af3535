/* FP64 CPU oracle for align_group_to_template: TEST INFRASTRUCTURE ONLY (see ss_oracle.h).
 *
 * A sequential restatement of the reference's algorithm, one function per reference kernel or host
 * step, each citing the file:line it follows (paths relative to the reference's setup/source/).
 * It keeps the reference's device state (x, y, mask, difference image, gradients, sparse triplets)
 * explicitly, so that each step can be read against the reference line by line.
 *
 * Where the reference reads memory that it never writes, or reads another CTA's data without
 * synchronisation, this restatement fixes one deterministic value and says so:
 *   Q1 paramsUsed[N-1] is never written (task_createparametermask.cuh:11-20 runs for idx < fframeW
 *      only; task_allocate.cu:223 does not initialise it). Fresh device memory reads as zero, so
 *      the last chain knot is treated as unused.
 *   Q2 pnew[N-1] and pnew[2N-1] are never written by the line search (task_linesearch.cu:50-54 runs
 *      for idx < fframeW) and keep the allocation fill value 1e6 (task_allocate.cu:226); the last
 *      frame's trials therefore see that knot at 1e6.
 *   Q3 In the line search, CTA f reads pnew[fW+W], which CTA f+1 writes concurrently
 *      (task_linesearch.cu:98-99 with task_applyparameters.cuh:39-42). Here every frame's trial
 *      reads the committed knot value p[fW+W] as it was when the line search started.
 *   Q4 groupActive is read at index groupId + shift*nGroups, which for an odd number of frames
 *      passes the end of the 2*nGroups-entry array (task_calcerrval.cu:166, task_linesearch.cu:88);
 *      such reads return false (zero-filled allocation padding).
 * The difference regulariser (lambda) is an extension: the reference parses lambda but never uses
 * it (memory.h:50, steady_scan.m:207-208). With lambda = 0 it has no effect.
 */
#include "ss_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define PNEW_FILL 1e6       /* task_allocate.cu:226 */
#define ERRVAL_FILL 1e6     /* task_allocate.cu:244 */
#define LS_TRIAL_CAP 2048   /* bound on line-search trials per frame (the reference has none) */

enum { STOP_CORR_INC = 0, STOP_HALT_CORR = 1, STOP_MOVEMENT = 2, STOP_ITER_LIMIT = 3, STOP_ERROR = 4 };

typedef struct {
    const sso_in* in;
    int Hb, W, nF, fW, N, P, Ht, Wt, group_size, n_groups;
    int flag_M, flag_C, flag_c, flag_e, flag_R;
    int flag_t;                 /* sub-function timing: TimedMainIteration (timedmainiteration.cpp) */
    double* rg_params;          /* flag t: the chain after every half-step (task.cpp:409) */
    /* device state of the reference (memory.h:85-163) */
    double *p, *p_last, *pnew, *delta_p, *new_delta_p, *x, *y, *diff, *wx, *wy, *jtr, *errval;
    double *p_ls;               /* Q3 snapshot */
    unsigned char *mask, *params_used, *blocks_present, *group_active;
    int* offsets;
    int n_used;
    double* corr;
    double* hv; int* hr; int* hc; /* COO triplets, 6P entries (task_filldiagonals.cu:174-181) */
    /* SolverEigen's function-static matrix (eigensolve.cpp:7-8): coupling blocks that persist
     * between solves while the number of used parameters does not change. */
    int eig_size;
    double* eig_c;              /* per list position i: (xx, yy, x_i y_i+1, x_i+1 y_i) */
    unsigned char* eig_valid;
    /* filters */
    int filter_active;          /* the solver's filter is not NoFilter */
    int filter_kind;            /* 1 smearing, 2 range */
    int filter_id, n_filter_iter;
    long long* n_eval;
    int own_n_eval;
    int cap_hit;
} St;

static int has_flag(const char* flags, char c) {
    if (!flags) return 0;
    for (const char* p = flags; *p; p++)
        if (*p == c) return 1;
    return 0;
}

static int group_active(const St* s, int col, int shift) {
    int gid = col / s->group_size + shift * s->n_groups;
    if (gid < 0 || gid >= 2 * s->n_groups) return 0; /* Q4 */
    return s->group_active[gid];
}

/* ParameterOrganizer::organize2D1, two 1-D inputs (parameterorganizer.cpp:31-55). */
void sso_organize2d1(const double* px, const double* py, double* p, int n_frames, int frame_w) {
    int N = frame_w * n_frames + 1;
    for (int f = 0; f < n_frames; f++) {
        int j = f * frame_w + (f != 0);
        for (int i = (f != 0); i < frame_w; i++, j++) {
            p[j] = px[f * (frame_w + 1) + i];
            p[j + N] = py[f * (frame_w + 1) + i];
        }
        if (f < n_frames - 1) {
            p[j] = (px[f * (frame_w + 1) + frame_w] + px[(f + 1) * (frame_w + 1)]) / 2;
            p[j + N] = (py[f * (frame_w + 1) + frame_w] + py[(f + 1) * (frame_w + 1)]) / 2;
        } else {
            p[j] = px[f * (frame_w + 1) + frame_w];
            p[j + N] = py[f * (frame_w + 1) + frame_w];
        }
    }
}

/* ParameterOrganizer::organize1D2, two 1-D outputs (parameterorganizer.cpp:79-98): the last knot
 * of each frame repeats knot W-1. */
void sso_organize1d2(const double* p, double* px, double* py, int n_frames, int frame_w) {
    int N = frame_w * n_frames + 1, ct = 0;
    for (int f = 0; f < n_frames; f++) {
        int fi = f * frame_w, i;
        for (i = fi; i < fi + frame_w; i++) {
            px[ct] = p[i];
            py[ct] = p[i + N];
            ct++;
        }
        px[ct] = p[i - 1];
        py[ct] = p[i - 1 + N];
        ct++;
    }
}

/* SmearingFilter::apply (smearingfilter.cpp:24-33). */
void sso_smearing_filter(double* v, int n, double strength) {
    for (int i = 0; i < n; i++) {
        double prev = (i == 0) ? 0.0 : v[i - 1];
        v[i] = prev * strength + v[i] * (1 - strength);
    }
}

/* RangeFilter::apply (rangefilter.cpp:24-40). */
void sso_range_filter(double* v, int n, double strength) {
    for (int i = 1; i < n - 1; i++) {
        double tc = (v[i - 1] + v[i + 1]) / 2;
        double d = (tc - v[i - 1]) * strength;
        if (v[i - 1] < v[i + 1]) {
            if (v[i] > v[i + 1] + d || v[i] < v[i - 1] - d) v[i] = tc;
        } else {
            if (v[i] < v[i + 1] + d || v[i] > v[i - 1] - d) v[i] = tc;
        }
    }
}

/* 3-tap median of the compact step halves (flag R; d_medianfilter.cu:3-20). The reference kernel
 * filters in place while neighbours are being overwritten and reads one element before the array;
 * this restatement filters out of place and leaves both end elements unchanged. */
static void median3(double* v, int n) {
    if (n < 3) return;
    double* o = (double*)malloc(sizeof(double) * n);
    memcpy(o, v, sizeof(double) * n);
    for (int i = 1; i < n - 1; i++) {
        double a = o[i], b = o[i - 1], c = o[i + 1];
        int k = 1 * ((b >= a && b < c) || (b <= a && b > c)) + 2 * ((c >= a && c < b) || (c >= b && c < a));
        v[i] = k == 0 ? a : (k == 1 ? b : c);
    }
    free(o);
}

/* d_applyParameters for block column idx (task_applyparameters.cuh:33-82), knots kx0/kx1/ky0/ky1.
 * Returns 1 if the column has at least minPointsPerBlock valid pixels. */
static int apply_column(St* s, int idx, double px, double px1, double py, double py1) {
    const sso_in* in = s->in;
    int idxm = idx % s->W;
    double tw = (double)(s->Wt - 1) - DBL_EPSILON; /* templateW - eps<T>() (eps.h:14-22) */
    double th = (double)(s->Ht - 1) - DBL_EPSILON;
    int cnt = 0;
    for (int r = 0; r < s->Hb; r++) {
        int im = r * s->W + idxm, ip = r * s->fW + idx;
        double f = in->frac[im];
        double x = fma(px1, f, fma(px, 1 - f, in->basex[im]));
        double y = fma(py1, f, fma(py, 1 - f, in->basey[im]));
        unsigned char m = in->base_mask[im] && x >= 0 && x < tw && y >= 0 && y < th;
        cnt += m;
        s->mask[ip] = m;
        s->x[ip] = x;
        s->y[ip] = y;
    }
    if (cnt >= in->min_points[idxm]) {
        s->blocks_present[idx] = 1;
        return 1;
    }
    return 0;
}

/* Bilinear template sample at a masked pixel (task_differenceimage.cuh:14-32). */
static inline double sample(const St* s, double x, double y) {
    const double* T = s->in->templ;
    int ix = (int)x, iy = (int)y, i = iy * s->Wt + ix;
    double xf = x - ix, yf = y - iy;
    double a = fma(yf, T[i + s->Wt], (1 - yf) * T[i]);
    double b = fma(yf, T[i + s->Wt + 1], (1 - yf) * T[i + 1]);
    return fma(xf, b, (1 - xf) * a);
}

/* d_createDifferenceImage for column idx (task_differenceimage.cuh:13-33). */
static void diff_column(St* s, int idx) {
    for (int r = 0; r < s->Hb; r++) {
        int ip = r * s->fW + idx;
        s->diff[ip] = s->mask[ip] ? s->in->image[ip] - sample(s, s->x[ip], s->y[ip]) : 0.0;
    }
}

/* d_calcBaseErrval for column idx (task_calcerrval.cu:6-18). */
static void errval_column(const St* s, int idx, double* ssd, int* cnt) {
    double e = 0;
    int c = 0;
    for (int r = 0; r < s->Hb; r++) {
        int ip = r * s->fW + idx;
        e = fma(s->diff[ip], s->diff[ip], e);
        c += s->mask[ip] ? 1 : 0;
    }
    *ssd = e;
    *cnt = c;
}

/* Knot-difference regulariser of frame f (extension): sum over its W chain edges of
 * |k_{t+1} - k_t|^2 in x and y. Own knots t < W come from own_x/own_y (stride 1, y at +N); the
 * frame's right boundary knot is (bx, by). */
static double frame_reg(const St* s, const double* own, double bx, double by) {
    double r = 0;
    for (int t = 0; t < s->W; t++) {
        double x0 = own[t], y0 = own[t + s->N];
        double x1 = t + 1 < s->W ? own[t + 1] : bx;
        double y1 = t + 1 < s->W ? own[t + 1 + s->N] : by;
        r += (x1 - x0) * (x1 - x0) + (y1 - y0) * (y1 - y0);
    }
    return r;
}

/* hd_applyParameters (task_applyparameters.cu:4-16) with blocksPresent cleared before it
 * (mainiteration.cpp:232). */
static void apply_all(St* s) {
    memset(s->blocks_present, 0, s->N);
    int idx;
#pragma omp parallel for schedule(static) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (idx = 0; idx < s->fW; idx++)
        apply_column(s, idx, s->p[idx], s->p[idx + 1], s->p[idx + s->N], s->p[idx + s->N + 1]);
}

/* d_calcAllGroupErrval (task_calcerrval.cu:20-51) incl. d_createParameterMask
 * (task_createparametermask.cuh:11-20). */
static void calc_group_errvals(St* s, int shift) {
    int f;
#pragma omp parallel for schedule(static) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (f = 0; f < s->nF; f++) {
        if (!group_active(s, f * s->W, shift)) continue;
        double e = 0;
        int c = 0;
        for (int t = 0; t < s->W; t++) {
            int idx = f * s->W + t;
            if (idx == 0) s->params_used[idx] = s->blocks_present[idx];
            else if (idx == s->N - 1) s->params_used[idx] = s->blocks_present[idx - 1];
            else s->params_used[idx] = s->blocks_present[idx] | s->blocks_present[idx - 1];
            diff_column(s, idx);
            double ce;
            int cc;
            errval_column(s, idx, &ce, &cc);
            e += ce;
            c += cc;
        }
        double val = e / (double)c;
        if (s->in->lambda != 0) {
            int b0 = f * s->W;
            val = (e + s->in->lambda * frame_reg(s, s->p + b0, s->p[b0 + s->W], s->p[b0 + s->W + s->N])) / (double)c;
        }
        s->errval[shift * s->nF + f] = val;
        s->n_eval[f]++;
    }
}

/* d_updateGradients (task_updategradients.cu:3-29). */
static void update_gradients(St* s) {
    const double* gx = s->in->xgrad;
    const double* gy = s->in->ygrad;
    int idx;
#pragma omp parallel for schedule(static) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (idx = 0; idx < s->fW; idx++) {
        for (int r = 0; r < s->Hb; r++) {
            int ip = r * s->fW + idx;
            if (s->mask[ip]) {
                int ix = (int)s->x[ip], iy = (int)s->y[ip], ti = iy * s->Wt + ix;
                double xf = s->x[ip] - (double)ix, yf = s->y[ip] - (double)iy;
                s->wx[ip] = fma(yf, gx[ti + s->Wt], (1 - yf) * gx[ti]);
                s->wy[ip] = fma(xf, gy[ti + 1], (1 - xf) * gy[ti]);
            } else {
                s->wx[ip] = 0;
                s->wy[ip] = 0;
            }
        }
    }
}

/* hd_generateSubSparseOffsets (task_generatesubsparseoffset.cu:8-27). */
static void sub_sparse_offsets(St* s) {
    int used = 0, off = 0;
    for (int i = 0; i < s->P; i++) {
        if (s->params_used[i % s->N]) used++;
        else off++;
        s->offsets[i] = off;
    }
    s->n_used = used;
}

static void insert_value(St* s, int nz, double v, int row, int col) {
    int mrow = row >= s->N ? row - s->N : row;
    int mcol = col >= s->N ? col - s->N : col;
    if (s->params_used[mrow] && s->params_used[mcol]) {
        s->hv[nz] = v;
        s->hr[nz] = row - s->offsets[row];
        s->hc[nz] = col - s->offsets[col];
    }
}

/* d_fillDiagonals (task_filldiagonals.cu:47-159) with hd_fillDiagonals' INT_MAX reset (:177). */
static void fill_diagonals(St* s) {
    const double* frac = s->in->frac;
    int nnz = s->P * 6;
    for (int i = 0; i < nnz; i++) s->hr[i] = INT_MAX;
    int N = s->N, idx;
#pragma omp parallel for schedule(static) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (idx = 0; idx < N; idx++) {
        if (!s->params_used[idx]) continue;
        double offx = 0, offy = 0, offxy = 0, dgx = 0, dgy = 0, dgxy = 0;
        int last = (idx == s->fW), first = (idx == 0);
        int iy = idx - last, iy1 = idx - 1, idxm = idx % s->W;
        for (int r = 0; r < s->Hb; r++) {
            double f = frac[r * s->W + idxm];
            double fsq = f * f, csq = (1 - f) * (1 - f), fc = f - fsq;
            double gx = s->wx[iy], gy = s->wy[iy];
            double gxx = gx * gx, gyy = gy * gy, gxy = gx * gy;
            offx = fma(gxx, fc, offx);
            offy = fma(gyy, fc, offy);
            offxy = fma(gxy, fc, offxy);
            switch (first + (last << 1)) {
            case 0: {
                double hx = s->wx[iy1], hy = s->wy[iy1];
                dgx += fma(gxx, csq, hx * hx * fsq);
                dgy += fma(gyy, csq, hy * hy * fsq);
                dgxy += fma(gxy, csq, hx * hy * fsq);
                break;
            }
            case 1:
                dgx = fma(gxx, csq, dgx);
                dgy = fma(gyy, csq, dgy);
                dgxy = fma(gxy, csq, dgxy);
                break;
            case 2:
                dgx = fma(gxx, fsq, dgx);
                dgy = fma(gyy, fsq, dgy);
                dgxy = fma(gxy, fsq, dgxy);
                break;
            }
            iy += s->fW;
            iy1 += s->fW;
        }
        if (!last) {
            int z = idx;
            insert_value(s, z, dgx, idx, idx); z += N;
            insert_value(s, z, offx, idx + 1, idx); z += N;
            insert_value(s, z, offx, idx, idx + 1); z += N;
            insert_value(s, z, dgy, idx + N, idx + N); z += N;
            insert_value(s, z, offy, idx + N + 1, idx + N); z += N;
            insert_value(s, z, offy, idx + N, idx + N + 1); z += N;
            insert_value(s, z, dgxy, idx, idx + N); z += N;
            insert_value(s, z, offxy, idx, idx + N + 1); z += N;
            insert_value(s, z, offxy, idx + 1, idx + N); z += N;
            insert_value(s, z, dgxy, idx + N, idx); z += N;
            insert_value(s, z, offxy, idx + N + 1, idx); z += N;
            insert_value(s, z, offxy, idx + N, idx + 1);
        } else {
            int z = idx;
            insert_value(s, z, dgx, idx, idx); z += N;
            insert_value(s, z, dgy, idx + N, idx + N); z += N;
            insert_value(s, z, dgxy, idx + N, idx); z += N;
            insert_value(s, z, dgxy, idx, idx + N);
        }
    }
}

/* d_fillJTr (task_filljtr.cu:3-58). */
static void fill_jtr(St* s) {
    const double* frac = s->in->frac;
    int N = s->N, idx;
#pragma omp parallel for schedule(static) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (idx = 0; idx < N; idx++) {
        if (!s->params_used[idx]) continue;
        double sx = 0, sy = 0, sx2 = 0, sy2 = 0;
        int idxm = idx % s->W;
        if (idx != s->fW) {
            for (int r = 0; r < s->Hb; r++) {
                int ip = r * s->fW + idx;
                double f = frac[r * s->W + idxm];
                double fdi = s->diff[ip] * (1 - f);
                sx = fma(fdi, s->wx[ip], sx);
                sy = fma(fdi, s->wy[ip], sy);
            }
        }
        if (idx != 0) {
            int m = idxm == 0 ? s->W - 1 : idxm - 1;
            for (int r = 0; r < s->Hb; r++) {
                int ip = r * s->fW + idx - 1;
                double f = frac[r * s->W + m];
                double fdi = s->diff[ip] * f;
                sx2 = fma(fdi, s->wx[ip], sx2);
                sy2 = fma(fdi, s->wy[ip], sy2);
            }
        }
        s->jtr[idx - s->offsets[idx]] = sx + sx2;
        s->jtr[idx + N - s->offsets[idx + N]] = sy + sy2;
    }
}

/* Regulariser terms added to the compact system (extension): lambda * L on the used knots and
 * -lambda * L p on the right-hand side, L the chain Laplacian over the full knot vector. */
static void add_regulariser(St* s, double* dg, double* cp, int* knot_of) {
    double lam = s->in->lambda;
    if (lam == 0) return;
    int h = s->n_used / 2, N = s->N;
    for (int i = 0; i < h; i++) {
        int k = knot_of[i];
        int deg = (k > 0) + (k < N - 1);
        dg[3 * i + 0] += lam * deg;
        dg[3 * i + 1] += lam * deg;
        for (int c = 0; c < 2; c++) {
            const double* p = s->p + c * N;
            double lp = deg * p[k] - (k > 0 ? p[k - 1] : 0) - (k < N - 1 ? p[k + 1] : 0);
            s->jtr[i + c * h] -= lam * lp;
        }
        if (i + 1 < h && knot_of[i + 1] == k + 1) {
            cp[4 * i + 0] -= lam;
            cp[4 * i + 1] -= lam;
        }
    }
}

/* Block LDL^T of a symmetric block-tridiagonal system with 2x2 blocks, n blocks.
 * d: n x 3 (xx, yy, xy) diagonal blocks; c: (n-1) x 4 coupling block between i (rows) and i+1
 * (cols): [[c0, c2], [c3, c1]]; b: n x 2; x: n x 2 solution. In knot-major (x_k, y_k) order the
 * block pattern admits no fill, so this factorisation is exact. */
int sso_block_tridiag_solve(int n, const double* d, const double* c, const double* b, double* x) {
    double* dd = (double*)malloc(sizeof(double) * 3 * n);   /* factor D_i (symmetric) */
    double* yv = (double*)malloc(sizeof(double) * 2 * n);
    if (!dd || !yv) { free(dd); free(yv); return -1; }
    /* forward: D_i = A_i - C_{i-1}^T D_{i-1}^{-1} C_{i-1}; y_i = b_i - C_{i-1}^T D_{i-1}^{-1} y_{i-1} */
    for (int i = 0; i < n; i++) {
        double a0 = d[3 * i], a1 = d[3 * i + 1], a2 = d[3 * i + 2];
        double r0 = b[2 * i], r1 = b[2 * i + 1];
        if (i > 0) {
            const double* C = c + 4 * (i - 1);
            double p0 = dd[3 * (i - 1)], p1 = dd[3 * (i - 1) + 1], p2 = dd[3 * (i - 1) + 2];
            double det = p0 * p1 - p2 * p2;
            double q0 = p1 / det, q1 = p0 / det, q2 = -p2 / det; /* inverse of prev D */
            /* C^T = [[c0, c3], [c2, c1]] ; M = C^T Dinv */
            double m00 = C[0] * q0 + C[3] * q2, m01 = C[0] * q2 + C[3] * q1;
            double m10 = C[2] * q0 + C[1] * q2, m11 = C[2] * q2 + C[1] * q1;
            /* D_i -= M C */
            a0 -= m00 * C[0] + m01 * C[3];
            a1 -= m10 * C[2] + m11 * C[1];
            a2 -= m00 * C[2] + m01 * C[1];
            r0 -= m00 * yv[2 * (i - 1)] + m01 * yv[2 * (i - 1) + 1];
            r1 -= m10 * yv[2 * (i - 1)] + m11 * yv[2 * (i - 1) + 1];
        }
        dd[3 * i] = a0; dd[3 * i + 1] = a1; dd[3 * i + 2] = a2;
        yv[2 * i] = r0; yv[2 * i + 1] = r1;
    }
    /* backward: x_i = D_i^{-1} (y_i - C_i x_{i+1}) */
    for (int i = n - 1; i >= 0; i--) {
        double r0 = yv[2 * i], r1 = yv[2 * i + 1];
        if (i < n - 1) {
            const double* C = c + 4 * i;
            r0 -= C[0] * x[2 * (i + 1)] + C[2] * x[2 * (i + 1) + 1];
            r1 -= C[3] * x[2 * (i + 1)] + C[1] * x[2 * (i + 1) + 1];
        }
        double p0 = dd[3 * i], p1 = dd[3 * i + 1], p2 = dd[3 * i + 2];
        double det = p0 * p1 - p2 * p2;
        x[2 * i] = (p1 * r0 - p2 * r1) / det;
        x[2 * i + 1] = (p0 * r1 - p2 * r0) / det;
    }
    free(dd);
    free(yv);
    return 0;
}

/* Gathers the compact triplets into block form indexed by used-list position. */
static void gather_blocks(St* s, double* dg, double* cp, unsigned char* cp_written, int* knot_of) {
    int h = s->n_used / 2, N = s->N;
    int i = 0;
    for (int k = 0; k < N; k++)
        if (s->params_used[k]) knot_of[i++] = k;
    memset(dg, 0, sizeof(double) * 3 * h);
    memset(cp, 0, sizeof(double) * 4 * (h > 0 ? h : 1));
    memset(cp_written, 0, h > 0 ? h : 1);
    int nnz = s->P * 6;
    for (int z = 0; z < nnz; z++) {
        if (s->hr[z] == INT_MAX) continue;
        int r = s->hr[z], c = s->hc[z];
        int rl = r >= h ? r - h : r, cl = c >= h ? c - h : c;
        int ry = r >= h, cy = c >= h;
        double v = s->hv[z];
        if (rl == cl) {
            if (!ry && !cy) dg[3 * rl] = v;
            else if (ry && cy) dg[3 * rl + 1] = v;
            else dg[3 * rl + 2] = v;
        } else if (cl == rl + 1) {   /* upper coupling (rows of rl, cols of rl+1) */
            cp_written[rl] = 1;
            if (!ry && !cy) cp[4 * rl] = v;
            else if (ry && cy) cp[4 * rl + 1] = v;
            else if (!ry && cy) cp[4 * rl + 2] = v; /* (x_i, y_i+1) */
            else cp[4 * rl + 3] = v;                /* (y_i, x_i+1) */
        }
        /* lower-triangle entries mirror the upper ones (symmetric insertion) */
    }
}

/* ISolver::solve: exact LDL^T for ids 1 and 2 (eigensolve.cpp:35-38, cusolversolver.cu:53-56), with
 * the Eigen path's persistent matrix (eigensolve.cpp:7-31); ILU(0) in the compact [x; y] order for
 * id 0 (cusparsesolver.cu:119-158). Writes the compact step into new_delta_p. */
static void ilu0_solve(St* s);

static void solve(St* s) {
    int h = s->n_used / 2;
    if (h == 0) return;
    if (s->in->solver_id == 0) {
        ilu0_solve(s);
        return;
    }
    double* dg = (double*)malloc(sizeof(double) * 3 * h);
    double* cp = (double*)malloc(sizeof(double) * 4 * h);
    unsigned char* cw = (unsigned char*)malloc(h);
    int* knot_of = (int*)malloc(sizeof(int) * h);
    double* b = (double*)malloc(sizeof(double) * 2 * h);
    double* xs = (double*)malloc(sizeof(double) * 2 * h);
    gather_blocks(s, dg, cp, cw, knot_of);
    if (s->in->solver_id == 2) {
        if (s->eig_size != s->n_used) {
            s->eig_size = s->n_used;
            memset(s->eig_valid, 0, s->N);
        }
        for (int i = 0; i + 1 < h; i++) {
            if (cw[i]) {
                memcpy(s->eig_c + 4 * i, cp + 4 * i, 4 * sizeof(double));
                s->eig_valid[i] = 1;
            } else if (s->eig_valid[i]) {
                memcpy(cp + 4 * i, s->eig_c + 4 * i, 4 * sizeof(double));
            }
        }
    }
    add_regulariser(s, dg, cp, knot_of);
    for (int i = 0; i < h; i++) {
        b[2 * i] = s->jtr[i];
        b[2 * i + 1] = s->jtr[i + h];
    }
    sso_block_tridiag_solve(h, dg, cp, b, xs);
    for (int i = 0; i < h; i++) {
        s->new_delta_p[i] = xs[2 * i];
        s->new_delta_p[i + h] = xs[2 * i + 1];
    }
    free(dg); free(cp); free(cw); free(knot_of); free(b); free(xs);
}

/* ILU(0) + two triangular solves in the compact [x; y] ordering, rows sorted and columns sorted
 * within rows (task_filldiagonals.cu:185-214, cusparsesolver.cu:119-158). */
static void ilu0_solve(St* s) {
    int m = s->n_used, nnz_all = s->P * 6;
    int* rowcnt = (int*)calloc(m + 1, sizeof(int));
    for (int z = 0; z < nnz_all; z++)
        if (s->hr[z] != INT_MAX) rowcnt[s->hr[z] + 1]++;
    for (int i = 0; i < m; i++) rowcnt[i + 1] += rowcnt[i];
    int nnz = rowcnt[m];
    int* col = (int*)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
    double* val = (double*)malloc(sizeof(double) * (nnz > 0 ? nnz : 1));
    int* fill = (int*)calloc(m, sizeof(int));
    for (int z = 0; z < nnz_all; z++) {
        if (s->hr[z] == INT_MAX) continue;
        int r = s->hr[z], pos = rowcnt[r] + fill[r]++;
        col[pos] = s->hc[z];
        val[pos] = s->hv[z];
    }
    for (int r = 0; r < m; r++) { /* insertion sort columns (d_sortColumnIndices) */
        for (int a = rowcnt[r] + 1; a < rowcnt[r + 1]; a++) {
            int b = a;
            while (b > rowcnt[r] && col[b - 1] > col[b]) {
                int tc = col[b - 1]; col[b - 1] = col[b]; col[b] = tc;
                double tv = val[b - 1]; val[b - 1] = val[b]; val[b] = tv;
                b--;
            }
        }
    }
    /* the knot-difference regulariser (extension) on the same entries as for the exact solvers
     * (add_regulariser): lambda * deg on the xx and yy diagonals, -lambda on the xx and yy
     * couplings of consecutive used knots, -lambda * L p on the right-hand side */
    if (s->in->lambda != 0 && m > 0) {
        double lam = s->in->lambda;
        int h = m / 2, N = s->N;
        int* knot_of = (int*)malloc(sizeof(int) * h);
        for (int k = 0, i = 0; k < N && i < h; k++)
            if (s->params_used[k]) knot_of[i++] = k;
        for (int i = 0; i < h; i++) {
            int k = knot_of[i];
            int deg = (k > 0) + (k < N - 1);
            int fresh = i + 1 < h && knot_of[i + 1] == k + 1;
            for (int c = 0; c < 2; c++) {
                int r = i + c * h;
                const double* p = s->p + c * N;
                double lp = deg * p[k] - (k > 0 ? p[k - 1] : 0) - (k < N - 1 ? p[k + 1] : 0);
                s->jtr[r] -= lam * lp;
                for (int a = rowcnt[r]; a < rowcnt[r + 1]; a++) {
                    if (col[a] == r) val[a] += lam * deg;
                    if (fresh && col[a] == r + 1) val[a] -= lam;
                }
                if (fresh)
                    for (int a = rowcnt[r + 1]; a < rowcnt[r + 2]; a++)
                        if (col[a] == r) val[a] -= lam;
            }
        }
        free(knot_of);
    }
    int* diag = (int*)malloc(sizeof(int) * m);
    int* pos_of = (int*)malloc(sizeof(int) * m);
    for (int i = 0; i < m; i++) pos_of[i] = -1;
    for (int i = 0; i < m; i++) {
        diag[i] = -1;
        for (int a = rowcnt[i]; a < rowcnt[i + 1]; a++) pos_of[col[a]] = a;
        for (int a = rowcnt[i]; a < rowcnt[i + 1] && col[a] < i; a++) {
            int k = col[a];
            if (diag[k] < 0) continue;
            val[a] /= val[diag[k]];
            for (int bb = diag[k] + 1; bb < rowcnt[k + 1]; bb++) {
                int j = col[bb];
                if (pos_of[j] >= 0) val[pos_of[j]] -= val[a] * val[bb];
            }
        }
        for (int a = rowcnt[i]; a < rowcnt[i + 1]; a++) {
            if (col[a] == i) diag[i] = a;
            pos_of[col[a]] = -1;
        }
    }
    double* z = (double*)malloc(sizeof(double) * m);
    for (int i = 0; i < m; i++) { /* L z = b, unit diagonal */
        double acc = s->jtr[i];
        for (int a = rowcnt[i]; a < rowcnt[i + 1] && col[a] < i; a++) acc -= val[a] * z[col[a]];
        z[i] = acc;
    }
    for (int i = m - 1; i >= 0; i--) { /* U y = z */
        double acc = z[i];
        for (int a = rowcnt[i + 1] - 1; a >= rowcnt[i] && col[a] > i; a--) acc -= val[a] * s->new_delta_p[col[a]];
        s->new_delta_p[i] = diag[i] >= 0 ? acc / val[diag[i]] : acc / 0.0;
    }
    free(rowcnt); free(col); free(val); free(fill); free(diag); free(pos_of); free(z);
}

/* d_expandResults (task_expandresults.cu:9-36). */
static void expand_results(St* s, int shift) {
    int half = s->group_size >> 1;
    for (int idx = 0; idx < s->P; idx++) {
        int j = idx >= s->N ? idx - s->N : idx;
        int fixed = (((idx + 1) - shift * half) % s->group_size) == 0;
        if (fixed) continue; /* keeps deltaP[idx] */
        s->delta_p[idx] = s->params_used[j] ? s->new_delta_p[idx - s->offsets[idx]] : 0.0;
    }
}

/* d_linesearch for one frame (task_linesearch.cu:76-149), with the Q2/Q3 boundary-knot rule.
 * Trials are counted in n_eval. */
static void linesearch_frame(St* s, int shift, int f) {
    int W = s->W, N = s->N, b0 = f * W;
    if (!group_active(s, b0, shift)) return;
    double mult = s->in->ls_mult, thr = s->in->move_thresh;
    double bx = (f < s->nF - 1) ? s->p_ls[b0 + W] : PNEW_FILL;
    double by = (f < s->nF - 1) ? s->p_ls[b0 + W + N] : PNEW_FILL;
    int trials = 0;
    for (;;) {
        if (++trials > LS_TRIAL_CAP) { s->cap_hit = 1; return; }
        for (int t = 0; t < W; t++) { /* d_addDeltaP */
            s->pnew[b0 + t] = s->p[b0 + t] + s->delta_p[b0 + t];
            s->pnew[b0 + t + N] = s->p[b0 + t + N] + s->delta_p[b0 + t + N];
        }
        int present = 0;
        for (int t = 0; t < W; t++) {
            double px1 = t + 1 < W ? s->pnew[b0 + t + 1] : bx;
            double py1 = t + 1 < W ? s->pnew[b0 + t + 1 + N] : by;
            present |= apply_column(s, b0 + t, s->pnew[b0 + t], px1, s->pnew[b0 + t + N], py1);
        }
        s->n_eval[f]++;
        if (!present) {
            int moving = 0;
            for (int t = 0; t < W; t++) { /* d_reduceDeltaP then d_checkMovement */
                s->delta_p[b0 + t] *= mult;
                s->delta_p[b0 + t + N] *= mult;
                if (fabs(s->delta_p[b0 + t]) > thr || fabs(s->delta_p[b0 + t + N]) > thr) moving = 1;
            }
            if (!moving) return;
            continue;
        }
        double e = 0;
        int c = 0;
        for (int t = 0; t < W; t++) {
            diff_column(s, b0 + t);
            double ce;
            int cc;
            errval_column(s, b0 + t, &ce, &cc);
            e += ce;
            c += cc;
        }
        double ev = e / (double)c;
        if (s->in->lambda != 0)
            ev = (e + s->in->lambda * frame_reg(s, s->pnew + b0, s->p_ls[b0 + W], s->p_ls[b0 + W + N])) / (double)c;
        if (ev < s->errval[shift * s->nF + f]) {
            for (int t = 0; t < W; t++) { /* d_setNewP */
                s->p[b0 + t] = s->pnew[b0 + t];
                s->p[b0 + t + N] = s->pnew[b0 + t + N];
            }
            if (b0 == 0) s->errval[shift * s->nF + f] = ev; /* only idx == 0 writes (task_linesearch.cu:135) */
            return;
        }
        int moving = 0;
        for (int t = 0; t < W; t++)
            if (fabs(s->delta_p[b0 + t]) > thr || fabs(s->delta_p[b0 + t + N]) > thr) moving = 1;
        if (!moving) return;
        for (int t = 0; t < W; t++) {
            s->delta_p[b0 + t] *= mult;
            s->delta_p[b0 + t + N] *= mult;
        }
    }
}

/* hd_linesearch (task_linesearch.cu:108-126). */
static int linesearch(St* s, int shift) {
    memcpy(s->p_ls, s->p, sizeof(double) * s->P);
    int f;
#pragma omp parallel for schedule(dynamic) num_threads(s->in->n_threads > 0 ? s->in->n_threads : 1)
    for (f = 0; f < s->nF; f++) linesearch_frame(s, shift, f);
    double e0 = 0, e1 = 0;
    for (int i = 0; i < s->nF; i++) {
        e0 += s->errval[i];
        e1 += s->errval[i + s->nF];
    }
    return (shift && e0 > e1) || (!shift && e0 < e1);
}

/* hd_globalCorrelation (task_correlation.cu:62-99), including its quirks: the image mean is taken
 * over all pixels divided by the valid count, the means are paired crosswise, and the per-column
 * loop only advances while pixels are valid (:24-34). */
static double global_correlation(St* s) {
    int npx = s->Hb * s->fW;
    for (int i = 0; i < npx; i++) /* d_swapWIDiff */
        if (s->mask[i]) s->diff[i] = s->in->image[i] - s->diff[i];
    double sum_a = 0, sum_b = 0;
    long long n = 0;
    for (int i = 0; i < npx; i++) {
        sum_a += s->in->image[i];
        sum_b += s->diff[i];
        n += s->mask[i] ? 1 : 0;
    }
    double div_a = sum_a / (double)n, div_b = sum_b / (double)n;
    double assq = 0, bssq = 0, q = 0;
    for (int idx = 0; idx < s->fW; idx++) {
        int px = idx;
        for (int i = 0; i < s->Hb; i++) {
            if (s->mask[px]) {
                double va = s->diff[px] - div_a;
                double vb = s->in->image[px] - div_b; /* qcImg = image where valid */
                assq += va * va;
                bssq += vb * vb;
                q += va * vb;
                px += s->fW;
            }
        }
    }
    /* the swap back is launched with the per-column kernel's grid (task_correlation.cu:86-98): one
     * block of THREADS_PER_BLOCK per 256 block columns, so only the first 256 ceil(fW / 256)
     * pixels (row-major) are swapped back; the others keep the warped template until a later
     * pass writes their difference image again */
    int swap_back = 256 * ((s->fW + 255) / 256);
    if (swap_back > npx) swap_back = npx;
    for (int i = 0; i < swap_back; i++)
        if (s->mask[i]) s->diff[i] = s->in->image[i] - s->diff[i];
    return q / sqrt(assq * bssq);
}

/* hd_frameCorrelation (task_correlation.cu:101-183). */
static void frame_correlation(St* s) {
    int npx = s->Hb * s->fW;
    for (int i = 0; i < npx; i++)
        if (s->mask[i]) s->diff[i] = s->in->image[i] - s->diff[i];
    for (int f = 0; f < s->nF; f++) {
        double sa = 0, sb = 0;
        long long c = 0;
        for (int t = 0; t < s->W; t++)
            for (int r = 0; r < s->Hb; r++) {
                int ip = r * s->fW + f * s->W + t;
                if (s->mask[ip]) {
                    c++;
                    sb += s->in->image[ip];
                    sa += s->diff[ip];
                }
            }
        double ma = sa / (double)c, mb = sb / (double)c;
        double assq = 0, bssq = 0, q = 0;
        for (int t = 0; t < s->W; t++)
            for (int r = 0; r < s->Hb; r++) {
                int ip = r * s->fW + f * s->W + t;
                double m = s->mask[ip] ? 1.0 : 0.0;
                double va = (s->diff[ip] - ma) * m, vb = (s->in->image[ip] - mb) * m;
                assq += va * va;
                bssq += vb * vb;
                q += va * vb;
            }
        s->corr[f] = q / sqrt(assq * bssq);
    }
    for (int i = 0; i < npx; i++)
        if (s->mask[i]) s->diff[i] = s->in->image[i] - s->diff[i];
}

/* d_maskInactiveGroups (task_maskinactive.cu:3-25), flag M. */
static void mask_inactive(St* s) {
    memset(s->group_active, 0, 2 * s->n_groups);
    int half = s->group_size >> 1;
    for (int idx = 0; idx < s->fW; idx++) {
        int f = idx / s->W;
        if (s->corr[f] < s->in->halt_corr) {
            int g = idx / s->group_size;
            if (g < 2 * s->n_groups) s->group_active[g] = 1;
            if (idx < half || idx >= s->fW - half) continue;
            int g2 = (idx - half) / s->group_size + s->n_groups;
            if (g2 < 2 * s->n_groups) s->group_active[g2] = 1;
        }
    }
}

static void disable_filter(St* s) { s->filter_active = 0; }

/* MainIteration::execute (mainiteration.cpp:62-119), or with flag t TimedMainIteration::execute
 * (timedmainiteration.cpp:45-143), which differs in four ways: it clears paramsUsed before every
 * half-step (:50), so the knots of frames whose group is inactive are unused instead of keeping
 * their last use; at the filter's iteration limit it disables the filter without zeroing filterID
 * (:97-105), and on the retry without filter it zeroes filterID (:136), the reverse of
 * MainIteration (mainiteration.cpp:83-89, 96-106), which changes when alignFrames's
 * filter-deactivation branch (task.cpp:313-325) fires; it copies the chain after every half-step
 * into slot shift + 2 (iteration - 1) of rgParams (:124); and its retry runs as iteration + 1
 * (:141), which moves those slots. The timers and its clearing of the mask (every mask entry is
 * rewritten by applyParameters) leave the results alone. */
static int main_iteration(St* s, int iteration) {
    int improved = 1;
    for (int shift = 0; shift < 2; shift++) {
        if (s->flag_t) memset(s->params_used, 0, s->N);
        apply_all(s);
        calc_group_errvals(s, shift);
        update_gradients(s);
        sub_sparse_offsets(s);
        fill_diagonals(s);
        fill_jtr(s);
        if (s->n_filter_iter != 0 && iteration > s->n_filter_iter) {
            disable_filter(s);
            if (!s->flag_t) s->filter_id = 0;
            s->n_filter_iter = 0;
        }
        solve(s);
        int h = s->n_used / 2;
        if (s->filter_active) {
            if (s->filter_kind == 1) {
                sso_smearing_filter(s->new_delta_p, h, s->in->filter_strength);
                sso_smearing_filter(s->new_delta_p + h, h, s->in->filter_strength);
            } else {
                sso_range_filter(s->new_delta_p, h, s->in->filter_strength);
                sso_range_filter(s->new_delta_p + h, h, s->in->filter_strength);
            }
        }
        if (s->flag_R) {
            median3(s->new_delta_p, h);
            median3(s->new_delta_p + h, h);
        }
        expand_results(s, shift);
        improved &= linesearch(s, shift);
        /* slots past 2 max_iter (a retry in the last iteration) are not written: the reference's
         * host buffer has 2 max_iter slots (task_allocate.cu:122) */
        const int slot = shift + 2 * (iteration - 1);
        if (s->flag_t && s->rg_params && slot < 2 * s->in->max_iter)
            memcpy(s->rg_params + (size_t)slot * s->P, s->p, sizeof(double) * s->P);
    }
    if (!improved) {
        if (s->n_filter_iter != 0) {
            disable_filter(s);
            if (s->flag_t) s->filter_id = 0;
            s->n_filter_iter = 0;
            return main_iteration(s, s->flag_t ? iteration + 1 : iteration);
        }
        return 0;
    }
    return 1;
}

/* Validates the arguments and allocates the reference's device state (task_allocate.cu:159-273). */
static int state_init(St* s, const sso_in* in, long long* n_eval) {
    if (!in || in->frame_w <= 0 || in->frame_h <= 0 || in->n_frames <= 0 || in->group_size <= 0 ||
        in->templ_h < 2 || in->templ_w < 2)
        return -1;
    memset(s, 0, sizeof(St));
    s->in = in;
    s->Hb = in->frame_h; s->W = in->frame_w; s->nF = in->n_frames;
    s->fW = s->W * s->nF; s->N = s->fW + 1; s->P = 2 * s->N;
    s->Ht = in->templ_h; s->Wt = in->templ_w;
    s->group_size = in->group_size;
    s->n_groups = s->fW / s->group_size;
    s->flag_M = has_flag(in->flags, 'M');
    s->flag_C = has_flag(in->flags, 'C');
    s->flag_c = has_flag(in->flags, 'c');
    s->flag_e = has_flag(in->flags, 'e');
    s->flag_R = has_flag(in->flags, 'R');
    s->flag_t = has_flag(in->flags, 't');
    /* Task::initialize filter factory (task.cpp:54-70) */
    s->filter_id = in->filter_id;
    s->n_filter_iter = in->max_filter_iter;
    switch (in->filter_id & (0 - (in->max_filter_iter != 0))) {
    case 0: s->filter_active = 0; s->n_filter_iter = 0; break;
    case 1: s->filter_active = 1; s->filter_kind = 1; break;
    case 2: s->filter_active = 1; s->filter_kind = 2; break;
    default: return -2;
    }
    if (in->solver_id < 0 || in->solver_id > 2) return -3;
    size_t npx = (size_t)s->Hb * s->fW;
    s->p = (double*)calloc(s->P, sizeof(double));
    s->p_last = (double*)calloc(s->P, sizeof(double));
    s->p_ls = (double*)calloc(s->P, sizeof(double));
    s->pnew = (double*)malloc(sizeof(double) * s->P);
    s->delta_p = (double*)calloc(s->P, sizeof(double));
    s->new_delta_p = (double*)calloc(s->P, sizeof(double));
    s->jtr = (double*)calloc(s->P, sizeof(double));
    s->errval = (double*)malloc(sizeof(double) * 2 * s->nF);
    s->x = (double*)calloc(npx, sizeof(double));
    s->y = (double*)calloc(npx, sizeof(double));
    s->diff = (double*)calloc(npx, sizeof(double));
    s->wx = (double*)calloc(npx, sizeof(double));
    s->wy = (double*)calloc(npx, sizeof(double));
    s->mask = (unsigned char*)calloc(npx, 1);
    s->params_used = (unsigned char*)calloc(s->N, 1);     /* Q1 */
    s->blocks_present = (unsigned char*)calloc(s->N, 1);
    s->group_active = (unsigned char*)malloc(2 * s->n_groups + 1);
    s->offsets = (int*)calloc(s->P, sizeof(int));
    s->corr = (double*)calloc(s->nF, sizeof(double));
    s->hv = (double*)calloc((size_t)6 * s->P, sizeof(double));
    s->hr = (int*)malloc(sizeof(int) * 6 * (size_t)s->P);
    s->hc = (int*)calloc((size_t)6 * s->P, sizeof(int));
    s->eig_c = (double*)calloc((size_t)4 * s->N, sizeof(double));
    s->eig_valid = (unsigned char*)calloc(s->N, 1);
    s->eig_size = -1;
    s->own_n_eval = n_eval == NULL;
    s->n_eval = n_eval ? n_eval : (long long*)calloc(s->nF, sizeof(long long));
    memset(s->n_eval, 0, sizeof(long long) * s->nF);
    for (int i = 0; i < s->P; i++) s->pnew[i] = PNEW_FILL;
    for (int i = 0; i < 2 * s->nF; i++) s->errval[i] = ERRVAL_FILL;
    memset(s->group_active, 1, 2 * s->n_groups + 1);
    sso_organize2d1(in->est_dx, in->est_dy, s->p, s->nF, s->W);
    return 0;
}

static void state_free(St* s) {
    free(s->p); free(s->p_last); free(s->p_ls); free(s->pnew); free(s->delta_p); free(s->new_delta_p);
    free(s->jtr); free(s->errval); free(s->x); free(s->y); free(s->diff); free(s->wx); free(s->wy);
    free(s->mask); free(s->params_used); free(s->blocks_present); free(s->group_active); free(s->offsets);
    free(s->corr); free(s->hv); free(s->hr); free(s->hc); free(s->eig_c); free(s->eig_valid);
    if (s->own_n_eval) free(s->n_eval);
}

int sso_align_group(const sso_in* in, sso_out* out) {
    St st;
    St* s = &st;
    if (!out) return -1;
    int rc = state_init(s, in, out->n_eval);
    if (rc) return rc;
    s->rg_params = out->rg_params;

    /* Task::alignFrames (task.cpp:259-412) */
    double correlation = 0, corr = 0;
    int iteration = 0, stop = STOP_ERROR;
    for (;;) {
        iteration++;
        int improved = main_iteration(s, iteration);
        if (out->all_params && iteration <= in->max_iter)
            memcpy(out->all_params + (size_t)s->P * (iteration - 1), s->p, sizeof(double) * s->P);
        corr = global_correlation(s);
        if (s->flag_c) { /* per-frame correlations of this iteration (task.cpp:287-306) */
            frame_correlation(s);
            if (out->frame_corr_hist && iteration <= in->max_iter)
                memcpy(out->frame_corr_hist + (size_t)(iteration - 1) * s->nF, s->corr, sizeof(double) * s->nF);
        }
        if (s->flag_C && out->iter_corr && iteration <= in->max_iter) out->iter_corr[iteration - 1] = corr;
        if (corr - correlation < in->corr_inc_thresh) {
            stop = STOP_CORR_INC;
            break;
        } else if (corr - correlation < in->filter_corr_thresh) {
            if (s->filter_id != 0) {
                disable_filter(s);
                s->n_filter_iter = 0;
                s->filter_id = 0;
                continue;
            }
        }
        if (!improved) { stop = STOP_MOVEMENT; break; }
        else if (in->max_iter == iteration) { stop = STOP_ITER_LIMIT; break; }
        else if (correlation >= in->halt_corr) { stop = STOP_HALT_CORR; break; }
        correlation = corr;
        memcpy(s->p_last, s->p, sizeof(double) * s->P);
        if (s->flag_M) mask_inactive(s); /* reads corr: zero unless flag c refreshed it (task.cpp:349-351) */
        if (s->flag_e && out->iter_errvals && iteration <= in->max_iter)
            for (int i = 0; i < s->nF; i++) {
                out->iter_errvals[(size_t)(2 * (iteration - 1)) * s->nF + i] = s->errval[i];
                out->iter_errvals[(size_t)(2 * (iteration - 1) + 1) * s->nF + i] = s->errval[i + s->nF];
            }
    }
    if (iteration == 1) memcpy(s->p_last, s->p, sizeof(double) * s->P);
    calc_group_errvals(s, 0);
    /* with flag c the frame correlations of the last iteration are the output (task.cpp:392-395) */
    if (!s->flag_c) frame_correlation(s);

    out->iterations = iteration;
    out->stop_reason = stop;
    out->ls_trial_cap_hit = s->cap_hit;
    if (out->p_last) memcpy(out->p_last, s->p_last, sizeof(double) * s->P);
    if (out->dx_knots && out->dy_knots) sso_organize1d2(s->p_last, out->dx_knots, out->dy_knots, s->nF, s->W);
    for (int f = 0; f < s->nF; f++) {
        if (out->frame_corr) out->frame_corr[f] = s->corr[f];
        if (out->residrms) out->residrms[f] = sqrt(s->errval[f]);
    }
    if (out->mask) memcpy(out->mask, s->mask, (size_t)s->Hb * s->fW);

    state_free(s);
    return 0;
}

/* Test hook: runs one assembly pass (mainiteration.cpp:232-244) at the knot chain p (2N) for the
 * given shift and exports the state the reference keeps on the device after it. Any output may be
 * NULL. hv/hr/hc hold the 6P COO triplets (row INT_MAX = unset). */
int sso_debug_assemble(const sso_in* in, const double* p, int shift, double* x, double* y,
                       unsigned char* mask, double* diff, double* wx, double* wy,
                       unsigned char* params_used, unsigned char* blocks_present, int* offsets,
                       double* hv, int* hr, int* hc, double* jtr, double* errval, int* n_used) {
    St st;
    St* s = &st;
    int rc = state_init(s, in, NULL);
    if (rc) return rc;
    memcpy(s->p, p, sizeof(double) * s->P);
    apply_all(s);
    calc_group_errvals(s, shift);
    update_gradients(s);
    sub_sparse_offsets(s);
    fill_diagonals(s);
    fill_jtr(s);
    size_t npx = (size_t)s->Hb * s->fW;
    if (x) memcpy(x, s->x, sizeof(double) * npx);
    if (y) memcpy(y, s->y, sizeof(double) * npx);
    if (mask) memcpy(mask, s->mask, npx);
    if (diff) memcpy(diff, s->diff, sizeof(double) * npx);
    if (wx) memcpy(wx, s->wx, sizeof(double) * npx);
    if (wy) memcpy(wy, s->wy, sizeof(double) * npx);
    if (params_used) memcpy(params_used, s->params_used, s->N);
    if (blocks_present) memcpy(blocks_present, s->blocks_present, s->N);
    if (offsets) memcpy(offsets, s->offsets, sizeof(int) * s->P);
    if (hv) memcpy(hv, s->hv, sizeof(double) * 6 * (size_t)s->P);
    if (hr) memcpy(hr, s->hr, sizeof(int) * 6 * (size_t)s->P);
    if (hc) memcpy(hc, s->hc, sizeof(int) * 6 * (size_t)s->P);
    if (jtr) memcpy(jtr, s->jtr, sizeof(double) * s->P);
    if (errval) memcpy(errval, s->errval, sizeof(double) * 2 * s->nF);
    if (n_used) *n_used = s->n_used;
    state_free(s);
    return 0;
}

/* Test hook: d_expandResults for one shift on caller-provided state (task_expandresults.cu:9-36). */
void sso_debug_expand(int N, int group_size, int shift, const unsigned char* params_used,
                      const int* offsets, const double* new_delta_p, double* delta_p) {
    int P = 2 * N, half = group_size >> 1;
    for (int idx = 0; idx < P; idx++) {
        int j = idx >= N ? idx - N : idx;
        int fixed = (((idx + 1) - shift * half) % group_size) == 0;
        if (fixed) continue;
        delta_p[idx] = params_used[j] ? new_delta_p[idx - offsets[idx]] : 0.0;
    }
}

/* Test hook: global correlation of a given device state (task_correlation.cu:62-99). */
double sso_debug_global_corr(const sso_in* in, const unsigned char* mask, const double* diff) {
    St st;
    St* s = &st;
    if (state_init(s, in, NULL)) return NAN;
    size_t npx = (size_t)s->Hb * s->fW;
    memcpy(s->mask, mask, npx);
    memcpy(s->diff, diff, sizeof(double) * npx);
    double c = global_correlation(s);
    state_free(s);
    return c;
}
