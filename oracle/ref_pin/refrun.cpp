// Runs the reference's own align_group_to_template task layer (Task, MainIteration, the kernels,
// filters and ParameterOrganizer, rewritten by run_transform.py and compiled for the host with
// hostcuda.h) on one group: TEST INFRASTRUCTURE ONLY, the source of the golden trajectories that
// pin the oracle. The steps follow MexGateway<T>::execute (mex/mexgateway.cpp:372-445): settings
// and sizes as MexGateway<T>::preparePersistentMemory derives them (mexgateway.cpp:38-198), then
// Task<T>::initialize, allocateOutput, alignFrames and getParameters.
//
// The solver is the reference's SolverCuSolver (solver id 1, an exact Cholesky solve: its cuSOLVER
// call is answered by hostcuda.cpp). SolverEigen (id 2) needs the un-vendored Eigen and
// SolverCuSparse (id 0) the csrsv2 routines CUDA 12 no longer has; their classes are given bodies
// here that refuse to solve. The line search kernel reads the next frame's first knot from pnew,
// which that frame's block writes at the same time (task_linesearch.cu:50-54, 98-99); with the
// blocks run in order, the harness fixes the race as the oracle does: before every line search
// those knots of pnew hold the committed knots of p.
#include "task/task.h"
#include "task/solver/allsolver.cuh"
#include "mex/configuration.h"

#include <cstdio>
#include <cstdlib>

template <class T>
SolverEigen<T>::SolverEigen(IFilter<T>* filter) : filter(filter) {}
template <class T>
SolverEigen<T>::~SolverEigen() {}
template <class T>
void SolverEigen<T>::solve(DeviceMemory<T>&) {
  std::fprintf(stderr, "refrun: solver id 2 (Eigen) is not available in the host build\n");
  std::abort();
}
template <class T>
IFilter<T>* SolverEigen<T>::setFilter(IFilter<T>* f) {
  IFilter<T>* r = filter;
  filter = f;
  return r;
}
template <class T>
SolverCuSparse<T>::SolverCuSparse(IFilter<T>* filter) : filter(filter) {}
template <class T>
SolverCuSparse<T>::~SolverCuSparse() {}
template <class T>
void SolverCuSparse<T>::solve(DeviceMemory<T>&) {
  std::fprintf(stderr, "refrun: solver id 0 (cuSPARSE csrsv2) is not available in the host build\n");
  std::abort();
}
template <class T>
IFilter<T>* SolverCuSparse<T>::setFilter(IFilter<T>* f) {
  IFilter<T>* r = filter;
  filter = f;
  return r;
}
template class SolverEigen<double>;
template class SolverEigen<float>;
template class SolverCuSparse<double>;
template class SolverCuSparse<float>;

// The committed first knot of every frame but the first (x and y halves) copied into pnew before a
// line search (see the header comment). Called by the host launcher of d_linesearch through
// SS_LINESEARCH_HOOK.
template <class T>
void ss_refrun_sync_boundary(DeviceMemory<T>& mem) {
  for (int f = 1; f < mem.nFrames; f++) {
    const int k = f * mem.frameW;
    mem.pnew[k] = mem.p[k];
    mem.pnew[k + mem.nParamPoints] = mem.p[k + mem.nParamPoints];
  }
}
template void ss_refrun_sync_boundary(DeviceMemory<double>& mem);
template void ss_refrun_sync_boundary(DeviceMemory<float>& mem);

extern "C" {

// Inputs: row-major matrices as the reference holds them after MexConverter (the template and its
// gradients templ_h x templ_w; tfrac, basex, basey, base_mask frame_h x frame_w; image frame_h x
// frame_w * n_frames), initial knots (frame_w + 1) x n_frames column-major, min_points frame_w
// entries.
struct ssrun_in {
  const char* flags;
  int templ_h, templ_w;
  const double *templ, *xgrad, *ygrad;
  int frame_h, frame_w, n_frames;
  const double *frac, *basex, *basey;
  const unsigned char* base_mask;
  const double* image;
  const double *est_dx, *est_dy;
  const int* min_points;
  int group_size, max_iter;
  double move_thresh, halt_corr, corr_inc_thresh, filter_strength;
  int max_filter_iter;
  double filter_corr_thresh, lambda, ls_mult;
  int solver_id, filter_id;
};

// Outputs (each may be NULL): per-frame knots (frame_w + 1) x n_frames, frame correlations,
// residrms, the mask frame_h x (frame_w * n_frames) row-major, the knot chain after every iteration
// (2N x max_iter column-major), the errvals of every half-step (flag e: (2 max_iter) x n_frames
// column-major), the global correlation of every iteration (flag C) and the frame correlations of
// every iteration (flag c).
struct ssrun_out {
  double *dx, *dy, *frame_corr, *residrms;
  unsigned char* mask;
  double *all_params, *iter_errvals, *iter_corr;
  double* frame_corr_hist;  // flag c: n_frames x max_iter column-major
  int iterations, stop_reason;
  int singular_solves;  // solves of a matrix that was not positive definite (x unspecified)
  double* rg_params;    // flag t: the 2N chain after every half-step, 2 max_iter slots (output 14)
};

extern int ss_hostcuda_singular_solves;

int ssrun_align(const ssrun_in* in, ssrun_out* out) {
  typedef double T;
  Configuration config;
  ConfigurationParser::parseFlags(in->flags, &config);
  PreAllocatedMemory<T> rom;
  std::memset(static_cast<ReadOnlyVariables<T>*>(&rom), 0, sizeof(ReadOnlyVariables<T>));
  const int Ht = in->templ_h, Wt = in->templ_w, Hb = in->frame_h, W = in->frame_w, nF = in->n_frames;
  rom.templateImage = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->templ), Ht, Wt);
  rom.xGradients = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->xgrad), Ht, Wt);
  rom.yGradients = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->ygrad), Ht, Wt);
  rom.frac = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->frac), Hb, W);
  rom.baseX = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->basex), Hb, W);
  rom.baseY = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->basey), Hb, W);
  rom.image = NeutralMatrix<T, int, RowMajor<int>>(const_cast<T*>(in->image), Hb, W * nF);
  rom.initParameterX = NeutralMatrix<T>(const_cast<T*>(in->est_dx), W + 1, nF);
  rom.initParameterY = NeutralMatrix<T>(const_cast<T*>(in->est_dy), W + 1, nF);
  rom.minPointsPerBlock = NeutralMatrix<int, int, RowMajor<int>>(const_cast<int*>(in->min_points), 1, W);
  rom.baseMask = NeutralMatrix<bool, int, RowMajor<int>>(
      reinterpret_cast<bool*>(const_cast<unsigned char*>(in->base_mask)), Hb, W);
  // scalar settings in MEX order (mexgateway.cpp:96-174) and the derived sizes (:176-198)
  rom.groupSize = in->group_size;
  rom.nFrames = nF;
  rom.maxIterations = in->max_iter;
  rom.moveThreshold = in->move_thresh;
  rom.haltCorrelation = in->halt_corr;
  rom.correlationIncreaseThreshold = in->corr_inc_thresh;
  rom.filterStrength = in->filter_strength;
  rom.nFilterIterations = in->max_filter_iter;
  rom.filterCorrelationThreshold = in->filter_corr_thresh;
  rom.lambda = in->lambda;
  rom.linesearchReductionMultiplier = in->ls_mult;
  rom.solverID = in->solver_id;
  rom.filterID = in->filter_id;
  rom.gpuDeviceID = 0;
  rom.frameH = Hb;
  rom.frameW = W;
  rom.fframeW = W * nF;
  rom.nParamPoints = W * nF + 1;
  rom.nParams = 2 * rom.nParamPoints;
  rom.templateH = Ht;
  rom.templateW = Wt;
  rom.groupSize2 = 1;
  while (rom.groupSize2 < rom.groupSize) rom.groupSize2 <<= 1;
  rom.frameW2 = 1;
  while (rom.frameW2 < rom.frameW) rom.frameW2 <<= 1;
  rom.nGroups = rom.fframeW / rom.groupSize;

  TaskOutput<T> o;
  Task<T>* task = new Task<T>(&config);
  if (!task->initialize(rom)) return -1;
  task->allocateOutput(o);
  // entries of the history outputs that the run does not write read as NaN (the reference leaves
  // them as its allocation holds them)
  if (config.saveIterationErrvalsEnabled())
    for (int i = 0; i < 2 * in->max_iter * nF; i++) o.iterationErrvals.data()[i] = NAN;
  if (config.saveFrameCorrelationsEnabled())
    for (int i = 0; i < in->max_iter * nF; i++) o.frameCorrelations.data()[i] = NAN;
  ss_hostcuda_singular_solves = 0;
  StopCriterion r = task->alignFrames(o);
  out->singular_solves = ss_hostcuda_singular_solves;
  task->getParameters(o);
  out->iterations = o.iterations;
  out->stop_reason = static_cast<int>(r);
  const int nk = (W + 1) * nF, N = W * nF + 1, mi = in->max_iter;
  for (int i = 0; i < nk; i++) {
    if (out->dx) out->dx[i] = o.blockParametersX.data()[i];
    if (out->dy) out->dy[i] = o.blockParametersY.data()[i];
  }
  for (int f = 0; f < nF; f++) {
    if (out->frame_corr) out->frame_corr[f] = o.finalFrameCorrelations.data()[f];
    if (out->residrms) out->residrms[f] = o.errval.data()[f];
  }
  if (out->mask)
    for (int rr = 0; rr < Hb; rr++)
      for (int c = 0; c < W * nF; c++) out->mask[(size_t)rr * W * nF + c] = o.mask(rr, c) ? 1 : 0;
  if (out->all_params)
    for (int it = 0; it < mi; it++)
      for (int i = 0; i < 2 * N; i++) out->all_params[(size_t)it * 2 * N + i] = o.allParams(i, it);
  if (out->iter_errvals && config.saveIterationErrvalsEnabled())
    for (int f = 0; f < nF; f++)
      for (int k = 0; k < 2 * mi; k++) out->iter_errvals[(size_t)f * 2 * mi + k] = o.iterationErrvals(k, f);
  if (out->frame_corr_hist && config.saveFrameCorrelationsEnabled())
    for (int i = 0; i < nF * mi; i++) out->frame_corr_hist[i] = o.frameCorrelations.data()[i];
  if (out->rg_params && config.subFunctionTimingEnabled())
    for (size_t i = 0; i < (size_t)2 * N * 2 * mi; i++) out->rg_params[i] = o.rgParams.data()[i];
  if (out->iter_corr && config.saveIterationCorrelationsEnabled())
    for (int it = 0; it < mi; it++) out->iter_corr[it] = o.iterationCorrelations.data()[it];
  delete task;
  return 0;
}

}  // extern "C"
