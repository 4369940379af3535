// Host-side driver of the reference's own device functions and host classes, compiled by g++ with
// shim.h from the sources under the reference tree: TEST INFRASTRUCTURE ONLY (oracle pinning).
//
// Each entry walks the launch grid the reference's host launcher would use, one thread at a time
// (the selected kernels have no cross-thread communication), on a DeviceMemory<double> whose
// pointers are host arrays. The few host-side steps the reference does around them (the exclusive
// offset count of task_generatesubsparseoffset.cu:8-27, the per-frame sum that d_calcAllGroupErrval
// does as a shared-memory tree, and the Thrust reductions of hd_globalCorrelation) are restated
// here sequentially.
#include "interface/memory.h"
#include "helper/eps.h"
#include "task/task_applyparameters.cuh"
#include "task/task_differenceimage.cuh"
#include "task/task_createparametermask.cuh"
#include "interface/parameterorganizer/parameterorganizer.h"
#include "task/filter/smearingfilter.h"
#include "task/filter/rangefilter.h"

#include "gen/task_updategradients.gen.inc"
#include "gen/task_filldiagonals.gen.inc"
#include "gen/task_filljtr.gen.inc"
#include "gen/task_expandresults.gen.inc"
#include "gen/task_calcerrval.gen.inc"
#include "gen/task_correlation.gen.inc"

#include <vector>

ss_pin_dim3 blockIdx, blockDim, threadIdx, gridDim;

template <class F>
static void grid(int n_threads, int block, F&& f) {
    blockDim.x = block;
    int nb = (n_threads + block - 1) / block;
    for (int b = 0; b < nb; b++) {
        blockIdx.x = b;
        for (int t = 0; t < block; t++) {
            threadIdx.x = t;
            f();
        }
    }
}


extern "C" {

struct ssref_state {
    int frame_h, frame_w, n_frames, templ_h, templ_w, group_size;
    const double *templ, *xgrad, *ygrad, *frac, *basex, *basey, *image;
    const unsigned char* base_mask;
    const int* min_points;
    double *p, *x, *y, *diff, *wx, *wy, *jtr, *errval, *hv, *delta_p, *new_delta_p;
    unsigned char *mask, *params_used, *blocks_present, *group_active;
    int *offsets, *hr, *hc;
    int n_used;
};

static void fill_mem(DeviceMemory<double>& m, ssref_state* s) {
    std::memset(&m, 0, sizeof(m));
    m.frameH = s->frame_h;
    m.frameW = s->frame_w;
    m.nFrames = s->n_frames;
    m.fframeW = s->frame_w * s->n_frames;
    m.nParamPoints = m.fframeW + 1;
    m.nParams = 2 * m.nParamPoints;
    m.templateH = s->templ_h;
    m.templateW = s->templ_w;
    m.groupSize = s->group_size;
    m.nGroups = m.fframeW / s->group_size;
    m.templateImage = const_cast<double*>(s->templ);
    m.xGradients = const_cast<double*>(s->xgrad);
    m.yGradients = const_cast<double*>(s->ygrad);
    m.frac = const_cast<double*>(s->frac);
    m.baseX = const_cast<double*>(s->basex);
    m.baseY = const_cast<double*>(s->basey);
    m.baseMask = reinterpret_cast<bool*>(const_cast<unsigned char*>(s->base_mask));
    m.minPointsPerBlock = const_cast<int*>(s->min_points);
    m.image = const_cast<double*>(s->image);
    m.p = s->p;
    m.x = s->x;
    m.y = s->y;
    m.mask = reinterpret_cast<bool*>(s->mask);
    m.differenceImage = s->diff;
    m.wxgrad = s->wx;
    m.wygrad = s->wy;
    m.jtr = s->jtr;
    m.errval = s->errval;
    m.paramsUsed = reinterpret_cast<bool*>(s->params_used);
    m.blocksPresent = reinterpret_cast<bool*>(s->blocks_present);
    m.groupActive = reinterpret_cast<bool*>(s->group_active);
    m.subSparseOffsets = s->offsets;
    m.H.values = s->hv;
    m.H.rowInd = s->hr;
    m.H.colInd = s->hc;
    m.deltaP = s->delta_p;
    m.newDeltaP = s->new_delta_p;
}


// One assembly pass at s->p (mainiteration.cpp:232-244); group_active holds 2*nGroups entries.
int ssref_assemble(ssref_state* s, int shift) {
    DeviceMemory<double> m;
    fill_mem(m, s);
    DeviceMemory<double>* mem = &m;
    bool any = false;
    std::memset(s->blocks_present, 0, m.nParamPoints);
    grid(m.nParamPoints, THREADS_PER_BLOCK, [&] {
        int idx = blockIdx.x * blockDim.x + threadIdx.x;
        if (idx >= mem->nParamPoints) return;
        d_applyParameters(mem, idx, mem->p, &any);
    });
    // d_calcAllGroupErrval: grid nFrames x frameW (task_calcerrval.cu:20-51)
    for (int f = 0; f < m.nFrames; f++) {
        int g = (f * m.frameW) / m.groupSize + shift * m.nGroups;
        if (g >= 2 * m.nGroups || !m.groupActive[g]) continue;
        double sum = 0;
        int cnt = 0;
        blockIdx.x = f;
        blockDim.x = m.frameW;
        for (int t = 0; t < m.frameW; t++) {
            threadIdx.x = 0;
            int idx = f * m.frameW + t;
            d_createParameterMask<double>(mem, idx);
            d_createDifferenceImage<double>(mem, idx);
            double part;
            int pc;
            d_calcBaseErrval<double>(mem, idx, &part, &pc);
            sum += part;
            cnt += pc;
        }
        m.errval[shift * m.nFrames + f] = sum / static_cast<double>(cnt);
    }
    grid(m.fframeW, THREADS_PER_BLOCK, [&] { d_updateGradients<double>(mem); });
    // hd_generateSubSparseOffsets (task_generatesubsparseoffset.cu:8-27)
    int used = 0, off = 0;
    for (int i = 0; i < m.nParams; i++) {
        if (m.paramsUsed[i % m.nParamPoints]) used++;
        else off++;
        m.subSparseOffsets[i] = off;
    }
    m.nParamsUsed = used;
    s->n_used = used;
    for (int i = 0; i < m.nParams * 6; i++) m.H.rowInd[i] = INT_MAX;
    grid(m.nParamPoints, THREADS_PER_BLOCK, [&] { d_fillDiagonals<double>(mem); });
    grid(m.nParamPoints, THREADS_PER_BLOCK, [&] { d_fillJTr<double>(mem); });
    return 0;
}

int ssref_expand(ssref_state* s, int shift) {
    DeviceMemory<double> m;
    fill_mem(m, s);
    DeviceMemory<double>* mem = &m;
    grid(m.nParams, THREADS_PER_BLOCK, [&] { d_expandResults<double>(mem, shift); });
    return 0;
}

// hd_globalCorrelation (task_correlation.cu:62-99) with the Thrust reductions done sequentially.
double ssref_global_corr(ssref_state* s) {
    DeviceMemory<double> m;
    fill_mem(m, s);
    DeviceMemory<double>* mem = &m;
    int npx = m.frameH * m.fframeW;
    std::vector<double> qc_img(npx), assq(m.fframeW), bssq(m.fframeW), q(m.fframeW);
    m.qcAssq = assq.data();
    m.qcBssq = bssq.data();
    m.qcq = q.data();
    grid(npx, THREADS_PER_BLOCK, [&] {
        d_clearImage<double>(reinterpret_cast<bool*>(s->mask), m.image, qc_img.data(), npx);
    });
    grid(npx, THREADS_PER_BLOCK, [&] { d_swapWIDiff<double>(mem, npx); });
    double a = 0, b = 0;
    long long n = 0;
    for (int i = 0; i < npx; i++) {
        a += m.image[i];
        b += m.differenceImage[i];
        n += m.mask[i] ? 1 : 0;
    }
    a /= n;
    b /= n;
    grid(m.fframeW, THREADS_PER_BLOCK, [&] { d_globalCorrelation<double>(mem, a, b, qc_img.data()); });
    double sa = 0, sb = 0, sq = 0;
    for (int i = 0; i < m.fframeW; i++) {
        sa += assq[i];
        sb += bssq[i];
        sq += q[i];
    }
    grid(npx, THREADS_PER_BLOCK, [&] { d_swapWIDiff<double>(mem, npx); });
    return sq / std::sqrt(sa * sb);
}

void ssref_organize2d1(const double* px, const double* py, double* p, int n_frames, int frame_w) {
    int n = (frame_w + 1) * n_frames, N = frame_w * n_frames + 1;
    NeutralMatrix<double> x(const_cast<double*>(px), n, 1), y(const_cast<double*>(py), n, 1);
    NeutralMatrix<double, int, RowMajor<int>> out;
    ParameterOrganizer<double>::organize2D1(x, y, out, n_frames, frame_w, N);
    std::memcpy(p, out.data(), sizeof(double) * 2 * N);
}

void ssref_organize1d2(const double* p, double* px, double* py, int n_frames, int frame_w) {
    int n = (frame_w + 1) * n_frames, N = frame_w * n_frames + 1;
    NeutralMatrix<double> in(const_cast<double*>(p), 2 * N, 1), x(px, n, 1), y(py, n, 1);
    ParameterOrganizer<double>::organize1D2(in, x, y, n_frames, frame_w, N);
}

void ssref_smearing_filter(double* v, int n, double strength) {
    SmearingFilter<double> f(strength);
    f.apply(v, n);
}

void ssref_range_filter(double* v, int n, double strength) {
    RangeFilter<double> f(strength);
    f.apply(v, n);
}

}  // extern "C"
