// MATLAB MEX gateway of the B200 transform, with the calling convention of
// the reference's gateway (src/MEX/fcwtmex.cpp of fastlib/fCWT):
//
//   [tfm, freqs] = fcwt(x, c0, fs, f0, f1, fn, nthreads)
//
// x: single, real row vector (n samples); c0: Morlet bandwidth; fs: sample
// rate; f0, f1, fn: LOGSCALES grid; nthreads: accepted for compatibility.
// tfm: n x fn single complex (MATLAB column-major, so column i holds scale i:
// the same memory as the library's row-major [fn][n] output); freqs: 1 x fn
// single, fs / scale. Like the reference gateway the transform runs with
// threads = 1 (which also fixes the truncation rule) and normalisation on.
// Build (R2018a+ interleaved complex API), e.g.:
//   mex -R2018a fcwt_b200/mex/fcwtmex.cpp -Iinclude -Lfcwt_b200/lib -lfcwt_b200
#include "mex.h"
#include "matrix.h"

#include <cstdio>
#include <string>

#include "fcwt_b200.h"

namespace {

bool is_real_scalar(const mxArray* a) { return mxIsDouble(a) && !mxIsComplex(a) && mxGetNumberOfElements(a) == 1; }

fcwt_context* g_ctx = nullptr;  // one context for the MATLAB session (device 0)

void release_context() {
    if (g_ctx) fcwt_context_destroy(g_ctx);
    g_ctx = nullptr;
}

void check(int rc, const char* what) {
    if (rc != FCWT_OK) {
        std::string msg = std::string(what) + ": " + fcwt_last_error();
        mexErrMsgIdAndTxt("fCWT:library", "%s", msg.c_str());
    }
}

}  // namespace

void mexFunction(int nlhs, mxArray* plhs[], int nrhs, const mxArray* prhs[]) {
    if (nrhs != 7)
        mexErrMsgIdAndTxt("fCWT:nrhs", "Seven inputs required. (inputArray, c0, fs, f0, f1, fn, nthreads)");
    if (nlhs != 2)
        mexErrMsgIdAndTxt("fCWT:nlhs", "Two outputs are required. (time-frequency matrix, frequencies)");
    if (!mxIsSingle(prhs[0]) || mxIsComplex(prhs[0]))
        mexErrMsgIdAndTxt("fCWT:notSingle", "Input matrix must be type float (single).");
    if (mxGetM(prhs[0]) != 1) mexErrMsgIdAndTxt("fCWT:notRowVector", "Input must be a row vector.");
    static const char* names[6] = {"Wavelet coefficient", "Sampling frequency", "Starting frequency",
                                   "Ending frequency", "Number of frequencies", "Number of threads"};
    for (int k = 1; k < 7; k++)
        if (!is_real_scalar(prhs[k])) mexErrMsgIdAndTxt("fCWT:notScalar", "%s must be a scalar.", names[k - 1]);

    const float* x = mxGetSingles(prhs[0]);
    const int n = (int)mxGetN(prhs[0]);
    const float c0 = (float)mxGetScalar(prhs[1]);
    const int fs = (int)mxGetScalar(prhs[2]);
    const float f0 = (float)mxGetScalar(prhs[3]);
    const float f1 = (float)mxGetScalar(prhs[4]);
    const int fn = (int)mxGetScalar(prhs[5]);
    if (fn < 1 || !(f0 > 0.0f) || !(f1 > 0.0f)) mexErrMsgIdAndTxt("fCWT:range", "f0, f1 and fn must be positive.");

    mwSize dims[2] = {(mwSize)n, (mwSize)fn};
    plhs[0] = mxCreateNumericArray(2, dims, mxSINGLE_CLASS, mxCOMPLEX);
    float* tfm = reinterpret_cast<float*>(mxGetComplexSingles(plhs[0]));
    mwSize fdims[2] = {1, (mwSize)fn};
    plhs[1] = mxCreateNumericArray(2, fdims, mxSINGLE_CLASS, mxREAL);
    float* freqs = mxGetSingles(plhs[1]);

    if (!g_ctx) {
        check(fcwt_context_create(0, &g_ctx), "fcwt_context_create");
        mexAtExit(release_context);
    }
    // Scales(Morlet, FCWT_LOGSCALES, fs, f0, f1, fn) and fs / scale, as the reference gateway
    check(fcwt_scales(FCWT_LOGSCALES, fs, f0, f1, fn, freqs), "fcwt_scales");
    float* scales = static_cast<float*>(mxMalloc(sizeof(float) * (size_t)fn));
    for (int i = 0; i < fn; i++) scales[i] = freqs[i];
    check(fcwt_frequencies(scales, fn, fs, freqs), "fcwt_frequencies");
    // host buffers: the call copies in and out and returns when tfm is written
    const int rc = fcwt_cwt(g_ctx, x, n, c0, scales, fn, 1, FCWT_NORM, tfm, FCWT_OUT_C64);
    mxFree(scales);
    check(rc, "fcwt_cwt");
}
