/*
 * rtm.h - C ABI of librtm.so, the B200 (sm_100a) solve path of rooftop-mom.
 *
 * A thin MEX gateway (mex/rtm_mex.c) binds these entry points under the unchanged MATLAB
 * +rooftopMoM call signatures; the tests bind them through Python ctypes.
 *
 * Conventions
 *   - Complex arrays are interleaved (re, im) doubles (MATLAB R2018a+ interleaved complex, the same
 *     layout as cuDoubleComplex). FP32 device vectors are interleaved floats.
 *   - Grids are column-major with the x index fastest, exactly as the MATLAB arrays: generator
 *     magneticXX is (countX-1) x countY, magneticYY countX x (countY-1), electric countX x countY.
 *   - Rooftop vectors hold the x-directed rooftops first, then the y-directed ones, each grid
 *     column-major (src/+rooftopMoM/+basisFunctions/UniformRooftops.m:1-8).
 *   - `where` says whether a pointer is host (RTM_HOST) or device (RTM_DEVICE) memory. Host
 *     arguments are copied in and out inside the call.
 *   - `stream` is a cudaStream_t passed as void*; NULL means the library's own stream of the handle.
 *   - `nrhs`, the vectors of one batched call, is 1 to 65535 (RTM_ERR_ARG below, RTM_ERR_SIZE above):
 *     the batched kernels span the vectors in one grid dimension.
 *   - Every call returns an rtm_status; rtm_last_error() gives the message of the last failure on
 *     the calling thread. Nothing here aborts the process or falls back to the CPU.
 */
#ifndef RTM_H
#define RTM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define RTM_API __attribute__((visibility("default")))
#else
#define RTM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define RTM_VERSION_MAJOR 3
#define RTM_VERSION_MINOR 5
#define RTM_VERSION_PATCH 0

typedef enum rtm_status {
    RTM_OK = 0,
    RTM_ERR_ARG = 1,        /* invalid argument (null pointer, bad enum, non-finite) */
    RTM_ERR_SIZE = 2,       /* vector length does not match the operator */
    RTM_ERR_OOM_BUDGET = 3, /* the HBM budget (rtm_budget_configure) or the device refuses the bytes */
    RTM_ERR_CUDA = 4,       /* a CUDA call failed */
    RTM_ERR_TIMEOUT = 5,    /* a bounded wait ran out */
    RTM_ERR_SINGULAR = 6,   /* the circulant approximation is singular at some frequency */
    RTM_ERR_UNSUPPORTED = 7 /* size or option outside what this build supports */
} rtm_status;

typedef enum rtm_content { RTM_NONE = 0, RTM_XONLY = 1, RTM_YONLY = 2, RTM_BOTH = 3 } rtm_content;
typedef enum rtm_product { RTM_PRODUCT_FFT = 0, RTM_PRODUCT_SPLIT = 1, RTM_PRODUCT_LEAN = 2 } rtm_product;
typedef enum rtm_precision { RTM_FP64 = 0, RTM_FP32 = 1 } rtm_precision;
typedef enum rtm_where { RTM_HOST = 0, RTM_DEVICE = 1 } rtm_where;
typedef enum rtm_modifier { RTM_MODIFY_NONE = 0, RTM_MODIFY_REAL = 1, RTM_MODIFY_IMAG = 2 } rtm_modifier;
typedef enum rtm_kernel {
    RTM_KERNEL_STRANG = 0, RTM_KERNEL_TCHAN = 1, RTM_KERNEL_RCHAN = 2, RTM_KERNEL_HUCKLE = 3,
    RTM_KERNEL_SUPEROPTIMAL = 4
} rtm_kernel;
typedef enum rtm_builder { RTM_BUILDER_PARTWISE = 0, RTM_BUILDER_BLOCKWISE = 1, RTM_BUILDER_HYBRID = 2 } rtm_builder;
typedef enum rtm_method { RTM_METHOD_CG = 0, RTM_METHOD_GMRES = 1, RTM_METHOD_FGMRES_IR = 2 } rtm_method;

typedef struct rtm_generators rtm_generators;
typedef struct rtm_operator rtm_operator;
typedef struct rtm_preconditioner rtm_preconditioner;

/* Library ------------------------------------------------------------------------------------ */

/* Package version of the reference this build follows (src/+rooftopMoM/version.m:7, '3.5.0'). */
RTM_API int rtm_version(int* major, int* minor, int* patch);

/* Copies the message of the last failed call of this thread into buf (always NUL-terminated). */
RTM_API int rtm_last_error(char* buf, size_t len);

/* Selects the CUDA device of the calling thread for the handles it creates next. */
RTM_API int rtm_set_device(int device);

/* Number of launches of this library's own kernels since load (a counter for benchmarks). */
RTM_API int rtm_launch_count(int64_t* count);

/* Budget ------------------------------------------------------------------------------------- */
/* The HBM admission ledger; replaces src/+rooftopMoM/+resources/Budget.m:43-106 for device memory.
 * ceiling_bytes <= 0 means no ceiling (device free memory still applies). */
RTM_API int rtm_budget_configure(double ceiling_bytes);
RTM_API int rtm_budget_query(double* ceiling_bytes, double* held_bytes);
/* Fails with RTM_ERR_OOM_BUDGET if bytes do not fit below the ceiling and the device's free memory
 * (Budget.require, Budget.m:82-106). */
RTM_API int rtm_budget_require(double bytes);

/* Byte models of every stage before it is built (src/+rooftopMoM/+resources/estimate*.m).
 * out[0] generators, out[1] product spectra, out[2] product working, out[3] preconditioner
 * spectra, out[4] preconditioner working, out[5] solver vectors. */
RTM_API int rtm_estimate_bytes(int count_x, int count_y, int product, int method, int preconditioned, int restart,
                       int max_iterations, double out[6]);

/* Generators (Problem.generators / MomentAssembler.generate) ---------------------------------- */

/* Assembles the generators on the device (replaces
 * src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/generate.m:10-59): near pairs with the
 * order near_order, far pairs on the shared lattice with far_order, touching pairs by singularity
 * extraction with closed-form moments in FP64. */
RTM_API int rtm_generators_assemble(int count_x, int count_y, double size_x, double size_y, double wavenumber,
                            int near_order, int far_order, void* stream, rtm_generators** out);

/* Wraps given generators (e.g. the reference's stored ones; Generators.m:16-21). Pointers may be
 * NULL for a missing direction. */
RTM_API int rtm_generators_create(int count_x, int count_y, const double* magnetic_xx, const double* magnetic_yy,
                          const double* electric, int where, rtm_generators** out);

/* Applies @real / @imag to every generator into a new handle (Generators.modify, Generators.m:25-37). */
RTM_API int rtm_generators_modify(const rtm_generators* g, int modifier, rtm_generators** out);

/* Copies the generators out; any pointer may be NULL. */
RTM_API int rtm_generators_read(const rtm_generators* g, double* magnetic_xx, double* magnetic_yy, double* electric,
                        int where);
RTM_API int rtm_generators_info(const rtm_generators* g, int* count_x, int* count_y, int* content);
RTM_API int rtm_generators_destroy(rtm_generators* g);

/* Operator (Operator.m:7-54, Applicator.apply) ----------------------------------------------- */

/* Builds the spectra on the device and the product of the kind 'fft' (circulant embedding,
 * generateEmbeddingSpectra.m), 'splitFFT' (subbands, generateSubbandSpectra.m) or 'leanSplitFFT'
 * (same spectra, half the working grid). max_rhs bounds the number of right-hand sides of one
 * rtm_operator_apply. */
RTM_API int rtm_operator_create(const rtm_generators* g, double size_x, double size_y, int product, int precision,
                        int max_rhs, rtm_operator** out);

/* y = A x for nrhs vectors of length n, stored one after another (replaces Applicator.apply,
 * src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/apply.m:10-20 and
 * FFTApplicator.m:14-32). For an FP64 operator x, y are complex doubles; for an FP32 operator they
 * are complex floats when where == RTM_DEVICE and complex doubles (converted) when RTM_HOST. */
RTM_API int rtm_operator_apply(rtm_operator* op, const void* x, void* y, int64_t n, int nrhs, int where, void* stream);

/* y = A x like rtm_operator_apply with where == RTM_DEVICE, but allocating no device memory: the
 * product's working grid lives in one fixed array compiled into the library
 * (rtm_fixed_scratch_bytes, 32 MiB) instead of the operator's own buffer. No counterpart in the
 * reference: it exists for callers whose device memory belongs to another allocator or ledger and
 * that must not allocate per call. FFT products only; RTM_ERR_SIZE when the working grids of nrhs
 * vectors exceed the array. The array takes 32 MiB of device memory on each device where it is first
 * looked up (the first call there; under CUDA_MODULE_LOADING=EAGER, every context of the process) and
 * keeps it until the process exits, outside the budget ledger. Every call looks the array's address up
 * again; the first call on a device loads it, so make that call before any stream capture. All calls
 * on a device share the array: calls that can overlap in time race, so the caller serialises them. A
 * null stream runs on the operator's stream and waits for the result. */
RTM_API int rtm_operator_apply_fixed_scratch(const rtm_operator* op, const void* x, void* y, int64_t n, int nrhs,
                                             void* stream);
/* Size of the fixed scratch array in bytes. */
RTM_API int rtm_fixed_scratch_bytes(double* bytes);

/* Autotuner of the split product. No counterpart in the reference (whose benchmarks/measureFFTPlanner.m
 * times FFTW's planner for the same purpose). For a plate of count_x x count_y faces (both at least 2) and
 * a precision, measures every candidate transform grid, the reference's 7-smooth sizes
 * (generateFastFFTSize.m:11-15) and the next powers of two, and on power-of-two grids every kernel
 * schedule (CTAs per SM of the y passes, form of the x-mix), each timed on the device over applies to
 * nrhs vectors; with RTM_TUNE_FLUSH_L2 each apply follows a write of 256 MB, so that the spectra start
 * out of L2 as inside a solve. The fastest is kept for this device: split products created afterwards for
 * that face grid and precision use it (a larger transform grid gives the same product up to rounding).
 * RTM_TUNE_REFERENCE_SIZES keeps the reference's sizes and sweeps the schedules only; RTM_TUNE_VERBOSE
 * writes every configuration's time to stderr. */
#define RTM_TUNE_FLUSH_L2 1
#define RTM_TUNE_REFERENCE_SIZES 2
#define RTM_TUNE_VERBOSE 4
typedef struct rtm_tune_result {
    int fft_x, fft_y;          /* chosen transform grid */
    int y_blocks, mix_kind;    /* chosen schedule: CTAs per SM of the y passes (1..3) and the x-mix form
                                  (0..2 direct with 1..3 CTAs per SM, 3 pipelined); 0 and -1 off the
                                  power-of-two path */
    double seconds;            /* device time of one product (nrhs vectors) with the choice */
    double reference_seconds;  /* the same with the reference's sizes and the default schedule */
    int candidates;            /* configurations measured */
} rtm_tune_result;
RTM_API int rtm_tune_product(int count_x, int count_y, int precision, int nrhs, int flags, rtm_tune_result* out);
/* Forgets every choice of the autotuner (products created afterwards take the reference's sizes). */
/* Records fft_x x fft_y (at least the face counts) as the transform grid of the split products built
 * afterwards for this face grid and precision on the calling thread's device, with the default kernel
 * schedule, as if the autotuner had chosen it (e.g. powers of two for plates that go into one batch). */
RTM_API int rtm_tune_set(int count_x, int count_y, int precision, int fft_x, int fft_y);
RTM_API int rtm_tune_clear(void);

/* A dense n x n complex operator (column-major), for solving any small system with the same solvers
 * (the matrix operator of IterativeMethod.solve, convertToHandle.m:10-16). */
RTM_API int rtm_operator_create_dense(const double* matrix, int64_t n, int where, rtm_operator** out);

/* Spectra bytes held and the grid of the transforms. */
RTM_API int rtm_operator_info(const rtm_operator* op, int64_t* n, int* fft_x, int* fft_y, double* spectra_bytes,
                      double* working_bytes);
/* Copies the stored spectra out (complex doubles): count blocks of fft_x*fft_y each, in the order
 * subband-major, then E, MXX, MYY (split / fft products). Returns the block count in *count. */
RTM_API int rtm_operator_read_spectra(const rtm_operator* op, double* out, int* count);
RTM_API int rtm_operator_destroy(rtm_operator* op);

/* Preconditioner (Preconditioner.m:7-70) ------------------------------------------------------ */

/* Circulant preconditioner on the face grid: kernel (strang, tChan, rChan, huckle, superoptimal) x
 * builder (partwise, blockwise, hybrid) (generateCirculant.m:16-25). bandwidth may be NULL (whole
 * grid). Fails with RTM_ERR_SINGULAR when the approximation is singular (Preconditioner.m:60-67). */
RTM_API int rtm_preconditioner_create(const rtm_generators* g, double size_x, double size_y, int kernel, int builder,
                              const int* bandwidth, int precision, rtm_preconditioner** out);

/* Block-Jacobi preconditioner with blocks of block_x x block_y faces (the rooftops whose first face
 * lies in a block). Each block of the Green's matrix is formed from the generators and inverted on
 * the device. Not in the reference. */
RTM_API int rtm_preconditioner_create_block_jacobi(const rtm_generators* g, double size_x, double size_y, int block_x,
                                           int block_y, int precision, rtm_preconditioner** out);

RTM_API int rtm_preconditioner_apply(rtm_preconditioner* pc, const void* x, void* y, int64_t n, int nrhs, int where,
                             void* stream);
RTM_API int rtm_preconditioner_destroy(rtm_preconditioner* pc);

/* Solve (Solver.solve / IterativeMethod.solve) ------------------------------------------------ */

typedef struct rtm_solve_config {
    int method;            /* RTM_METHOD_CG (COCG), RTM_METHOD_GMRES, RTM_METHOD_FGMRES_IR */
    double tolerance;      /* relative residual to stop at (Solver.m:29, default 1e-6) */
    int max_iterations;    /* Solver.m:30, default 1000 */
    int restart;           /* GMRES cycle length (Solver.m:31, default 50); FGMRES inner cycle. At most 344
                              in FP64 and 638 in FP32 (RTM_ERR_UNSUPPORTED above): longer bases do not fit
                              the orthogonalisation's shared-memory tile */
    double inner_tolerance;/* FGMRES_IR: the tightest relative residual one FP32 inner solve aims at. Each inner
                              solve stops as soon as its right-hand side's outer tolerance is met in this
                              refinement step (at 0.5 tolerance ||b|| / ||r||), but not below this floor */
    int max_refinements;   /* FGMRES_IR: bound on the FP64 outer refinement steps */
    int check_every;       /* iterations between host convergence checks (0: library default) */
    int right_preconditioned; /* GMRES: 0 left preconditioning (GeneralizedMinimumResidual.m:2-5), 1 right
                                 (x = x0 + M V y at the end of each cycle: the monitored residual is that
                                 of op * x = b) */
    int gram_schmidt_passes;  /* classical Gram-Schmidt passes of each Arnoldi step: 2 (CGS2, the
                                 reference's orthogonalize_.m:15-23) or 1. GMRES: 0 selects 2. FGMRES_IR applies
                                 it to its FP32 inner solves, where 0 selects 1: the FP64 refinement measures
                                 the true residual, so orthogonality lost in one pass costs inner iterations,
                                 never accuracy */
} rtm_solve_config;

typedef struct rtm_solve_stats {
    int converged;         /* Output.converged */
    int iteration_count;   /* Output.iterationCount (inner iterations for FGMRES_IR) */
    double residual_norm;  /* Output.residualNorm, the true relative residual in FP64 */
    double time_s;         /* Output.time, device time of the whole solve */
    int refinements;       /* FGMRES_IR outer steps */
    int matvecs;           /* products applied */
} rtm_solve_stats;

/* Solves op * x = b for nrhs right-hand sides of length n (replaces IterativeMethod.solve,
 * src/+rooftopMoM/+solver/IterativeMethod.m:27-70, with ConjugateGradient.iterate_,
 * PreconditionedConjugateGradient.precondition_ and GeneralizedMinimumResidual.iterate_).
 * pc may be NULL; x0 may be NULL (zeros). history may be NULL, otherwise it receives
 * nrhs x (max_iterations+1) relative residuals (NaN after the last iteration). stats has nrhs
 * entries. The FP64 operator gives the true residual; FGMRES_IR needs op FP64 and uses inner_op
 * (FP32) and inner_pc for the inner solves. */
RTM_API int rtm_solve(rtm_operator* op, rtm_preconditioner* pc, const rtm_solve_config* config, const void* b,
              const void* x0, void* x, int64_t n, int nrhs, int where, double* history, rtm_solve_stats* stats,
              void* stream);
RTM_API int rtm_solve_mixed(rtm_operator* op, rtm_operator* inner_op, rtm_preconditioner* inner_pc,
                    const rtm_solve_config* config, const void* b, const void* x0, void* x, int64_t n, int nrhs,
                    int where, double* history, rtm_solve_stats* stats, void* stream);

/* Plate batches (not in the reference) ------------------------------------------------------- */

/* A batch of count entries, entry k one right-hand side on the plate of ops[k]: plates of uneven size
 * (and several right-hand sides of one plate, as entries that share its operator) solved together. The
 * vectors of a batch hold count entries of `stride` elements, the largest entry's unknowns; entry k's own
 * n_k unknowns come first, the elements after them are ignored on input and zero on output. The operators
 * have one precision; split products that share their transform grid on the power-of-two path
 * (rtm_tune_product chooses such grids) run as one launch of each of their kernels for the whole batch
 * (`fused` of rtm_plate_batch_info), any others one entry after another. pcs is NULL or count
 * preconditioners, one per entry. The operators and preconditioners must outlive the batch. */
typedef struct rtm_plate_batch rtm_plate_batch;
RTM_API int rtm_plate_batch_create(rtm_operator* const* ops, rtm_preconditioner* const* pcs, int count,
                                   rtm_plate_batch** out);
/* fused: the products share each kernel launch; fused_preconditioner: so do the block-Jacobi preconditioners
 * (circulant preconditioners, whose transforms follow each face grid, run entry by entry). */
RTM_API int rtm_plate_batch_info(const rtm_plate_batch* batch, int64_t* stride, int* count, int* fused,
                                 int* fused_preconditioner);
/* y = A x (preconditioner 0) or y = M x (preconditioner 1, a batch created with preconditioners), entry
 * by entry; x and y are count x stride elements. */
RTM_API int rtm_plate_batch_apply(rtm_plate_batch* batch, int preconditioner, const void* x, void* y, int where,
                                  void* stream);
/* rtm_solve over the batch (method RTM_METHOD_CG or RTM_METHOD_GMRES): every entry stops on its own
 * tolerance; history (count x (max_iterations+1)) and stats (count) as rtm_solve's. */
RTM_API int rtm_plate_batch_solve(rtm_plate_batch* batch, const rtm_solve_config* config, const void* b,
                                  const void* x0, void* x, int where, double* history, rtm_solve_stats* stats,
                                  void* stream);
RTM_API int rtm_plate_batch_destroy(rtm_plate_batch* batch);

/* Excitation and results (src/+rooftopMoM/+operator) ------------------------------------------ */

/* generatePlaneWave.m:18-42 on the device, for nrhs waves: direction and polarization are 3*nrhs
 * unit vectors, each pair perpendicular (RTM_ERR_ARG unless within 1e-9 of that), intensity nrhs values.
 * order is the far quadrature order of the rooftops. */
RTM_API int rtm_plane_wave(int count_x, int count_y, double size_x, double size_y, int order, double wavenumber,
                   const double* directions, const double* polarizations, const double* intensities, int nrhs,
                   void* out, int where, void* stream);

/* generateDeltaGap.m:13-14 with generateMiddlePort.m:14-28 (port of the given direction, 'x' = 0 or
 * 'y' = 1) or an explicit 0-based port. */
RTM_API int rtm_delta_gap(int count_x, int count_y, double size_x, double size_y, const int64_t* port, int port_count,
                  int direction, double voltage, void* out, int where);

/* computeRadarCrossSection.m:18-19 and computeInputImpedance.m:17 (current on host or device). */
RTM_API int rtm_radar_cross_section(double wavenumber, const void* excitation, const void* current, int64_t n,
                            double intensity, int where, double* out);
RTM_API int rtm_input_impedance(int count_x, int count_y, double size_x, double size_y, const void* current,
                        const int64_t* port, int port_count, double voltage, int where, double* out);
/* (out of rtm_input_impedance: out[0] + i out[1], the complex input impedance in ohms) */

/* Serving: a request loop of plate solves ------------------------------------------------------
 * No counterpart in the reference, whose closest analogue is the admission check of its memory
 * ledger (Budget.require, src/+rooftopMoM/+resources/Budget.m:82-106, fed by the byte models
 * estimate*.m). A server admits submitted requests first-fit in arrival order while a slot is free
 * and their estimated device bytes fit under the budget; each admitted request runs the whole
 * pipeline (assembly, split-FFT product, preconditioner, excitation, solve, RCS or input impedance)
 * on its own worker thread and CUDA streams, so the device work of admitted requests overlaps, and
 * requests that arrive meanwhile are admitted as slots and bytes free up. A request's result does not
 * depend on what else runs: every kernel's launch shape follows from the request alone. */
typedef struct rtm_server rtm_server;

typedef enum rtm_transform_sizes {
    RTM_SIZES_REFERENCE = 0,    /* the reference's 7-smooth transform sizes (generateFastFFTSize.m) */
    RTM_SIZES_POWER_OF_TWO = 1, /* plates: the next powers of two where the power-of-two kernels take them */
    RTM_SIZES_AUTOTUNE = 2      /* plates: rtm_tune_product on the first request of each face grid */
} rtm_transform_sizes;

typedef struct rtm_server_config {
    double budget_bytes;   /* device bytes the admitted requests may hold together (<= 0: 150e9) */
    int max_active;        /* requests admitted at once, one worker thread each (<= 0: 8) */
    int precision;         /* RTM_FP64, or RTM_FP32 for the mixed form (FP32 inner FGMRES, FP64 refinement) */
    int device;            /* CUDA device of the workers */
    int transform_sizes;   /* rtm_transform_sizes of the requests' split products (any size at least the face
                              count gives the same product up to rounding) */
    int max_batch;         /* 0 or 1: every request solves alone on its worker. Above 1 (FP64, power-of-two
                              sizes): max_active / max_batch workers (at least one), each taking up to
                              max_batch admitted requests at once whose 2-D plates share their transform grid,
                              method, preconditioner, restart and iteration bound, solved as one plate batch
                              (rtm_plate_batch_solve), each on its own tolerance. A request cancelled while its
                              batch runs is discarded when the batch ends. */
} rtm_server_config;

typedef enum rtm_excitation { RTM_EXCITE_PLANE_WAVE = 0, RTM_EXCITE_DELTA_GAP = 1 } rtm_excitation;
typedef enum rtm_request_state {
    RTM_REQUEST_QUEUED = 0,
    RTM_REQUEST_RUNNING = 1,
    RTM_REQUEST_DONE = 2,
    RTM_REQUEST_FAILED = 3,
    RTM_REQUEST_CANCELLED = 4
} rtm_request_state;

typedef struct rtm_request {
    int count_x, count_y;       /* faces of the plate (count_y = 1: a strip) */
    double size_x, size_y;      /* face sizes in metres */
    double wavenumber;          /* k = 2 pi f / c */
    int excitation;             /* rtm_excitation */
    double direction[3];        /* plane wave: unit propagation direction */
    double polarization[3];     /* plane wave: unit polarisation perpendicular to it (intensity 1); submit
                                   rejects the pair unless both hold to within 1e-9 */
    int port_direction;         /* delta gap: middle port across x (0) or y (1) rooftops */
    double voltage;             /* delta gap: gap voltage */
    int method;                 /* RTM_METHOD_CG or RTM_METHOD_GMRES (right-preconditioned) */
    int preconditioner;         /* 0 none, 1 block-Jacobi over 2 x 2 faces, 2 rChan circulant (partwise) */
    double tolerance;
    int max_iterations;
    int restart;
    int keep_current;           /* nonzero: keep the solution for rtm_server_poll to copy out */
} rtm_request;

typedef struct rtm_request_result {
    int state;                  /* rtm_request_state */
    int status;                 /* rtm_status of a failed request */
    int converged, iteration_count;
    double residual_norm;       /* true FP64 relative residual */
    double rcs;                 /* plane wave: monostatic radar cross section (m^2) */
    double impedance[2];        /* delta gap: input impedance, re and im (ohm) */
    int64_t unknowns;
    double bytes;               /* estimated device bytes the request held */
    double submitted_s, started_s, finished_s; /* host clock, seconds since the server was created */
    double solve_s;             /* device time of the solve */
} rtm_request_result;

RTM_API int rtm_server_create(const rtm_server_config* config, rtm_server** out);
/* Queues a request; *id identifies it. A request whose estimate alone exceeds the budget fails at once
 * with RTM_ERR_OOM_BUDGET (rooftopMoM:resources:insufficientMemory). */
RTM_API int rtm_server_submit(rtm_server* server, const rtm_request* request, uint64_t* id);
/* Copies the request's state and result, waiting up to wait_ms for it to finish (0: no wait, < 0:
 * until it finishes). current (host, n complex doubles) receives the solution of a finished request
 * that kept it; release != 0 forgets a finished request afterwards. */
RTM_API int rtm_server_poll(rtm_server* server, uint64_t id, int wait_ms, rtm_request_result* out, double* current,
                            int64_t n, int release);
/* Cancels a queued request at once, a running one at its solver's next host check. */
RTM_API int rtm_server_cancel(rtm_server* server, uint64_t id);
/* Cancels what is queued, lets running requests stop, joins the workers and frees the server. */
RTM_API int rtm_server_destroy(rtm_server* server);

#ifdef __cplusplus
}
#endif

#endif /* RTM_H */
