// Launch arguments of the FFT-product kernels (grid.cu, grid_fast.cu).
#pragma once

#include "fft.cuh"
#include "grid.h"
#include "internal.h"

namespace rtm {

// One right-hand side of a plate batch: its plate's face grid, spectra and face sizes (the transform grid,
// tables and vector stride are the batch's).
template <typename T> struct PlateDesc {
    int rows[2], cols[2];
    int64_t off[2];
    const typename Cx<T>::T2* spec;
    T inv_a2, inv_b2, inv_ab;
};

template <typename T> struct GridArgs {
    using T2 = typename Cx<T>::T2;
    int P, Q, nsx, nsy;
    int rows[2], cols[2];
    int64_t off[2];
    int64_t n;
    int ncomp;
    int ti;          // x columns per y-tile
    int py0, npy;    // y subbands handled by this launch (lean: one at a time)
    int accumulate;  // y-inverse adds into y (second parity of the lean product)
    FftPlan planP, planQ;
    const T2* twP;
    const T2* twQ;
    const T2* modP;
    const T2* modQ;
    T2* work;
    int64_t work_rhs;  // elements of W per right-hand side
    int mode;
    const T2* spec;
    const T2* ux0;
    const T2* ux1;
    const T2* vy0;
    const T2* vy1;
    T inv_a2, inv_b2, inv_ab, scale;
    const int* skip;  // per right-hand side, nonzero: leave it alone
    int skip_stride;
    int cb, ls;  // x-mix: y frequencies per CTA and the padded line stride
    int* fault;  // the device's fault word: set to RTM_ERR_TIMEOUT by a bounded wait that ran out
    const PlateDesc<T>* plates;  // plate batch: per right-hand side (device); null: every one on this plate
};

// The plate of right-hand side rhs: its own entry of a plate batch, else the launch's.
template <typename T> __device__ __forceinline__ PlateDesc<T> plate_of(const GridArgs<T>& a, int rhs) {
    if (a.plates) return a.plates[rhs];
    PlateDesc<T> d;
    for (int c = 0; c < 2; ++c) {
        d.rows[c] = a.rows[c];
        d.cols[c] = a.cols[c];
        d.off[c] = a.off[c];
    }
    d.spec = a.spec;
    d.inv_a2 = a.inv_a2;
    d.inv_b2 = a.inv_b2;
    d.inv_ab = a.inv_ab;
    return d;
}

template <typename A> __device__ __forceinline__ bool skipped(const A& a, int rhs) {
    return a.skip != nullptr && a.skip[(int64_t)rhs * a.skip_stride] != 0;
}


// Power-of-two split products with register-resident line transforms (grid_fast.cu). Eligible when
// both transform sizes are powers of two in [32, 1024] (FP64: [32, 512]) for a product that keeps both
// y subbands. Returns RTM_OK after launching the three kernels with the given schedule (grid.h).
template <typename T>
int launch_fast_split(const GridArgs<T>& a, int nrhs, const void* x, void* y, const FastSchedule& f, cudaStream_t s);

}  // namespace rtm
