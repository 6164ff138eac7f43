// Block-Toeplitz / block-circulant products by FFTs on a P x Q grid (device code in grid.cu).
//
// A GridApplicator applies y = A x for the rooftop layout of a countX x countY face grid:
//   GEN3   - the Green's matrix from the spectra of its three generators (E, MXX, MYY) per subband;
//            the 2x2 blocks are formed on the fly with the shift factors u = 1 - s_x, v = 1 - s_y
//            (generateBlockSpectra.m:35-47). Split products have 2 x 2 subbands on the fast-FFT grid
//            (generateSubbandSpectra.m), the 'fft' product 1 subband on the embedding grid 2n - 2.
//   BLOCK4 - explicit 2x2 block spectra (the inverted circulant preconditioner, FFTApplicator.m).
//   STRIP  - a grid one face wide: explicit 1x1 block spectra per subband on a line.
// A product of a 2-D grid runs as three kernels over a working grid W[rhs][parity_y][component][Q][P]:
//   y-forward: modulate (odd y subband), FFT along y, for tiles of x columns;
//   x-mix:     per y frequency: modulate, FFT along x, 2x2 block mix, inverse FFT, demodulate, sum
//              over the x subbands (in place in W);
//   y-inverse: inverse FFT along y, demodulate, sum over the y subbands, crop to the rooftop grids.
#pragma once

#include <vector>

#include "internal.h"
#include "ops.h"

namespace rtm {

enum GridMode { kGen3 = 0, kBlock4 = 1, kStrip = 2 };

// How the three kernels of a power-of-two split product run (grid_fast.cu): the CTAs an SM holds in
// the y passes (the launch bound; 1 to 3, 3 for FP64 only) and the form of the x-mix. A product takes the
// schedule the autotuner measured best for its precision and transform grid (tune.cpp), or the rules of
// default_fast_schedule when none was measured.
enum MixKind { kMixDirect1 = 0, kMixDirect2 = 1, kMixDirect3 = 2, kMixPipelined = 3 };
struct FastSchedule {
    int y_blocks = 2;
    int x_kind = kMixDirect1;
};
// True when both transform sizes take the power-of-two kernels: powers of two in [32, 1024] (FP64:
// [32, 512]).
bool fast_split_eligible(int P, int Q, bool fp64);
FastSchedule default_fast_schedule(int P, int Q, bool fp64);

struct GridApplicator : LinearOp {
    int mode = kGen3;
    int content = RTM_BOTH;
    int count_x = 0, count_y = 0;
    double size_x = 0, size_y = 0;
    int rows[2] = {0, 0}, cols[2] = {0, 0};
    int64_t off[2] = {0, 0};
    int P = 1, Q = 1;       // transform grid (STRIP: P = line length, Q = 1)
    int nsx = 1, nsy = 1;   // subbands along x and y
    bool lean = false;      // one y subband at a time (half the working grid)
    int max_rhs = 1;
    const FftTables* tP = nullptr;
    const FftTables* tQ = nullptr;
    const void* ux[2] = {nullptr, nullptr};  // shift factors per x parity (precision of the product)
    const void* vy[2] = {nullptr, nullptr};
    DeviceBuffer spec;      // GEN3: [sub][3][Q][P]; BLOCK4: [4][Q][P]; STRIP: [sub][P]
    DeviceBuffer work;      // W
    int spec_blocks = 0;    // blocks stored
    int* fault = nullptr;   // the device's fault word (looked up in reserve(), outside any capture)
    FastSchedule sched;     // schedule of the power-of-two kernels (set when the product is built)

    // y = A x on the device for nrhs vectors of length n (precision of the product).
    int apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) override;
    int reserve(int nrhs) override;
    size_t work_bytes_per_rhs() const;
    double stored_bytes() const override { return (double)spec.bytes; }
    double working_bytes() const override { return (double)work.bytes; }
};

// Plate batches (several plates, one right-hand side each, in one launch of each kernel): whether a
// product can join one (a split product on the power-of-two path), the device table of the plates'
// descriptors, and the product of a batch whose products share their transform grid and precision (vectors
// of `stride` elements, one per plate; work holds a working grid per plate).
bool batchable(const GridApplicator& g);
int plate_descs(const std::vector<const GridApplicator*>& plates, DeviceBuffer& out, cudaStream_t s);
int apply_plate_batch(const std::vector<const GridApplicator*>& plates, const void* descs, int64_t stride, void* work,
                      int* fault, const void* x, void* y, cudaStream_t s, SkipFlags skip);

// y = A x with the working grid in a fixed device array of fixed_scratch_bytes() instead of the
// product's own buffer; allocates nothing (RTM_ERR_SIZE when nrhs working grids do not fit).
int apply_fixed_scratch(const GridApplicator& g, const void* x, void* y, int nrhs, cudaStream_t s);
size_t fixed_scratch_bytes();

// Generator set on the device (FP64 complex, column-major).
struct DeviceGenerators {
    int count_x = 0, count_y = 0;
    int content = RTM_BOTH;
    bool is_real = false;   // modified by @real / @imag: the spectra drop their imaginary rounding
    DeviceBuffer xx, yy, e;
};

// Builds the split ('splitFFT' / 'leanSplitFFT') or embedding ('fft') product of the generators. A split
// product takes the transform grid and schedule the autotuner chose for its face grid and precision
// (tuned_choice), else the reference's sizes (generateFastFFTSize.m) and default_fast_schedule;
// force_P / force_Q (> 0) impose a transform grid (the autotuner's candidates).
int build_product(const DeviceGenerators& g, double size_x, double size_y, int product, int precision, int max_rhs,
                  GridApplicator& out, cudaStream_t s, int force_P = 0, int force_Q = 0,
                  const FastSchedule* force_sched = nullptr);

// The autotuner's measured choice for a face grid and precision on the current device (tune.cpp): false
// when none was measured.
bool tuned_choice(int count_x, int count_y, int precision, int* P, int* Q, FastSchedule* sched);
// Records a transform grid for a face grid and precision as if the autotuner had chosen it (schedule by
// default_fast_schedule).
void register_choice(int count_x, int count_y, int precision, int P, int Q);

// Builds the inverted circulant preconditioner on the face grid (generateCirculant.m:16-25).
int build_circulant(const DeviceGenerators& g, double size_x, double size_y, int kernel, int builder,
                    const int* bandwidth, int precision, GridApplicator& out, cudaStream_t s);

// Copies generators within the device applying a modifier (0 none, 1 real, 2 imag).
int modify_generators(const DeviceGenerators& in, int modifier, DeviceGenerators& out, cudaStream_t s);

// Assembles the generators on the device (assembly.cu).
int assemble_generators(int count_x, int count_y, double size_x, double size_y, double k, int near_order,
                        int far_order, DeviceGenerators& out, cudaStream_t s);

}  // namespace rtm
