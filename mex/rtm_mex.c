/*
 * rtm_mex.c - the MEX gateway that binds librtm.so (include/rtm.h) under the +rooftopMoM MATLAB classes.
 *
 * Build on a MATLAB host:  mex -R2018a -I<repo>/include rtm_mex.c -L<repo>/rooftop_mom_b200 -lrtm
 *
 * MATLAB R2018a+ stores complex arrays interleaved (re, im), the layout of rtm.h, so
 * mxGetComplexDoubles is passed through without repacking. Handles travel as uint64 scalars. Each
 * operation of the MATLAB glue (GpuMomentAssembler < Assembler, GpuSplitFFTApplicator < Applicator,
 * GpuIterativeMethod < IterativeMethod) has a branch; the seams it binds are Assembler.m:4-7,
 * Applicator.m:38-46 and IterativeMethod.m:27-70.
 */
#include "mex.h"
#include "rtm.h"
#include <math.h>
#include <string.h>

static void check(int status, const char* id_default) {
    if (status == RTM_OK) return;
    char msg[1024];
    rtm_last_error(msg, sizeof msg);
    const char* id = status == RTM_ERR_SIZE ? "rooftopMoM:product:sizeMismatch"
                   : status == RTM_ERR_OOM_BUDGET ? "rooftopMoM:resources:insufficientMemory"
                   : status == RTM_ERR_SINGULAR ? "rooftopMoM:preconditioner:singular" : id_default;
    mexErrMsgIdAndTxt(id, "%s", msg);
}

static void* handle_in(const mxArray* a) { return (void*)(uintptr_t)(*(uint64_t*)mxGetData(a)); }
static mxArray* handle_out(void* h) {
    mxArray* a = mxCreateNumericMatrix(1, 1, mxUINT64_CLASS, mxREAL);
    *(uint64_t*)mxGetData(a) = (uint64_t)(uintptr_t)h;
    return a;
}

/* A generator argument: interleaved complex doubles, or NULL for the empty generator of a missing direction. */
static const double* generator_in(const mxArray* a) {
    if (mxIsEmpty(a)) return NULL;
    if (!mxIsComplex(a)) mexErrMsgIdAndTxt("rooftopMoM:gpu:realGenerator", "pass complex(generator)");
    return (const double*)mxGetComplexDoubles(a);
}

/* Generators from the MATLAB arrays (electric is countX x countY); the caller destroys them. */
static rtm_generators* generators_in(const mxArray* xx, const mxArray* yy, const mxArray* e) {
    rtm_generators* g = NULL;
    check(rtm_generators_create((int)mxGetM(e), (int)mxGetN(e), generator_in(xx), generator_in(yy), generator_in(e),
                                RTM_HOST, &g), "rooftopMoM:gpu:generators");
    return g;
}

static int product_in(const mxArray* a) {
    char name[32];
    mxGetString(a, name, sizeof name);
    if (!strcmp(name, "fft")) return RTM_PRODUCT_FFT;
    if (!strcmp(name, "splitFFT")) return RTM_PRODUCT_SPLIT;
    if (!strcmp(name, "leanSplitFFT")) return RTM_PRODUCT_LEAN;
    mexErrMsgIdAndTxt("rooftopMoM:operator:invalidProduct", "unknown product %s", name);
    return -1;
}

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    char op[64];
    (void)nrhs;
    mxGetString(prhs[0], op, sizeof op);
    if (!strcmp(op, "assemble")) {
        /* countX, countY, sizeX, sizeY, wavenumber, near order, far order -> generators handle */
        rtm_generators* g = NULL;
        check(rtm_generators_assemble((int)mxGetScalar(prhs[1]), (int)mxGetScalar(prhs[2]), mxGetScalar(prhs[3]),
                                      mxGetScalar(prhs[4]), mxGetScalar(prhs[5]), (int)mxGetScalar(prhs[6]),
                                      (int)mxGetScalar(prhs[7]), NULL, &g), "rooftopMoM:gpu:assemble");
        plhs[0] = handle_out(g);
    } else if (!strcmp(op, "generators_read")) {
        /* handle -> magneticXX, magneticYY, electric (empty for a missing direction) */
        rtm_generators* g = handle_in(prhs[1]);
        int cx = 0, cy = 0, content = 0;
        check(rtm_generators_info(g, &cx, &cy, &content), "rooftopMoM:gpu:generators");
        plhs[0] = mxCreateDoubleMatrix(cx > 1 ? cx - 1 : 0, cx > 1 ? cy : 0, mxCOMPLEX);
        plhs[1] = mxCreateDoubleMatrix(cy > 1 ? cx : 0, cy > 1 ? cy - 1 : 0, mxCOMPLEX);
        plhs[2] = mxCreateDoubleMatrix(cx, cy, mxCOMPLEX);
        check(rtm_generators_read(g, cx > 1 ? (double*)mxGetComplexDoubles(plhs[0]) : NULL,
                                  cy > 1 ? (double*)mxGetComplexDoubles(plhs[1]) : NULL,
                                  (double*)mxGetComplexDoubles(plhs[2]), RTM_HOST), "rooftopMoM:gpu:generators");
    } else if (!strcmp(op, "generators_destroy")) {
        rtm_generators_destroy(handle_in(prhs[1]));
    } else if (!strcmp(op, "operator_create")) {
        /* magneticXX, magneticYY, electric, sizeX, sizeY, product -> operator handle */
        rtm_generators* g = generators_in(prhs[1], prhs[2], prhs[3]);
        rtm_operator* h = NULL;
        const int status = rtm_operator_create(g, mxGetScalar(prhs[4]), mxGetScalar(prhs[5]), product_in(prhs[6]),
                                               RTM_FP64, 1, &h);
        rtm_generators_destroy(g); /* the operator holds its spectra, built before the call returned */
        check(status, "rooftopMoM:gpu:operator");
        plhs[0] = handle_out(h);
    } else if (!strcmp(op, "operator_destroy")) {
        rtm_operator_destroy(handle_in(prhs[1]));
    } else if (!strcmp(op, "operator_apply")) {
        rtm_operator* h = handle_in(prhs[1]);
        const mwSize n = mxGetNumberOfElements(prhs[2]);
        plhs[0] = mxCreateDoubleMatrix(n, 1, mxCOMPLEX);
        check(rtm_operator_apply(h, mxGetComplexDoubles(prhs[2]), mxGetComplexDoubles(plhs[0]), (int64_t)n, 1,
                                 RTM_HOST, NULL), "rooftopMoM:product:sizeMismatch");
    } else if (!strcmp(op, "preconditioner_create")) {
        /* magneticXX, magneticYY, electric, sizeX, sizeY, kernel (rtm_kernel), builder (rtm_builder),
           bandwidth ([] or [bx, by] for Huckle) -> preconditioner handle */
        rtm_generators* g = generators_in(prhs[1], prhs[2], prhs[3]);
        int bandwidth[2] = {0, 0};
        const int has_bandwidth = !mxIsEmpty(prhs[8]);
        if (has_bandwidth) {
            const double* bw = mxGetDoubles(prhs[8]);
            bandwidth[0] = (int)bw[0];
            bandwidth[1] = (int)bw[1];
        }
        rtm_preconditioner* pc = NULL;
        const int status = rtm_preconditioner_create(g, mxGetScalar(prhs[4]), mxGetScalar(prhs[5]),
                                                     (int)mxGetScalar(prhs[6]), (int)mxGetScalar(prhs[7]),
                                                     has_bandwidth ? bandwidth : NULL, RTM_FP64, &pc);
        rtm_generators_destroy(g);
        check(status, "rooftopMoM:gpu:preconditioner");
        plhs[0] = handle_out(pc);
    } else if (!strcmp(op, "preconditioner_apply")) {
        rtm_preconditioner* pc = handle_in(prhs[1]);
        const mwSize n = mxGetNumberOfElements(prhs[2]);
        plhs[0] = mxCreateDoubleMatrix(n, 1, mxCOMPLEX);
        check(rtm_preconditioner_apply(pc, mxGetComplexDoubles(prhs[2]), mxGetComplexDoubles(plhs[0]), (int64_t)n, 1,
                                       RTM_HOST, NULL), "rooftopMoM:product:sizeMismatch");
    } else if (!strcmp(op, "preconditioner_destroy")) {
        rtm_preconditioner_destroy(handle_in(prhs[1]));
    } else if (!strcmp(op, "plane_wave")) {
        /* countX, countY, sizeX, sizeY, far order, wavenumber, direction (3), polarization (3), intensity */
        const int cx = (int)mxGetScalar(prhs[1]), cy = (int)mxGetScalar(prhs[2]);
        const double intensity = mxGetScalar(prhs[9]);
        plhs[0] = mxCreateDoubleMatrix((mwSize)(cx - 1) * cy + (mwSize)cx * (cy - 1), 1, mxCOMPLEX);
        check(rtm_plane_wave(cx, cy, mxGetScalar(prhs[3]), mxGetScalar(prhs[4]), (int)mxGetScalar(prhs[5]),
                             mxGetScalar(prhs[6]), mxGetDoubles(prhs[7]), mxGetDoubles(prhs[8]), &intensity, 1,
                             mxGetComplexDoubles(plhs[0]), RTM_HOST, NULL), "rooftopMoM:gpu:planeWave");
    } else if (!strcmp(op, "solve")) {
        /* operator, preconditioner ([] for none), method (0 cg, 1 gmres), tolerance, maxIterationCount, restart,
           right-hand side, initial guess ([] for zero) -> solution, residual norms, output struct */
        rtm_operator* A = handle_in(prhs[1]);
        rtm_preconditioner* P = mxIsEmpty(prhs[2]) ? NULL : handle_in(prhs[2]);
        rtm_solve_config c = {0};
        c.method = (int)mxGetScalar(prhs[3]);
        c.tolerance = mxGetScalar(prhs[4]);
        c.max_iterations = (int)mxGetScalar(prhs[5]);
        const double restart = mxGetScalar(prhs[6]); /* Solver.m:31: Inf means no restart */
        c.restart = isinf(restart) || restart > c.max_iterations ? c.max_iterations : (int)restart;
        const mwSize n = mxGetNumberOfElements(prhs[7]);
        plhs[0] = mxCreateDoubleMatrix(n, 1, mxCOMPLEX);
        plhs[1] = mxCreateDoubleMatrix(c.max_iterations + 1, 1, mxREAL);
        rtm_solve_stats s;
        check(rtm_solve(A, P, &c, mxGetComplexDoubles(prhs[7]),
                        mxIsEmpty(prhs[8]) ? NULL : mxGetComplexDoubles(prhs[8]), mxGetComplexDoubles(plhs[0]),
                        (int64_t)n, 1, RTM_HOST, mxGetDoubles(plhs[1]), &s, NULL), "rooftopMoM:solver:sizeMismatch");
        if (nlhs > 2) {
            const char* f[] = {"converged", "iterationCount", "residualNorm", "time"};
            plhs[2] = mxCreateStructMatrix(1, 1, 4, f);
            mxSetField(plhs[2], 0, "converged", mxCreateLogicalScalar(s.converged));
            mxSetField(plhs[2], 0, "iterationCount", mxCreateDoubleScalar(s.iteration_count));
            mxSetField(plhs[2], 0, "residualNorm", mxCreateDoubleScalar(s.residual_norm));
            mxSetField(plhs[2], 0, "time", mxCreateDoubleScalar(s.time_s));
        }
    } else {
        mexErrMsgIdAndTxt("rooftopMoM:gpu:unknownOperation", "unknown operation %s", op);
    }
}
