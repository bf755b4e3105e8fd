// Heap-backed implementation of the mx/mex functions declared in
// tests/mex/mex.h, and a driver that calls the gateway like MATLAB would:
//   fake_mex <in.f32> <n> <c0> <fs> <f0> <f1> <fn> <out.bin>
// writes the n x fn complex single output (column-major) and the 1 x fn
// frequencies. TEST INFRASTRUCTURE.
#include "mex.h"

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

struct mxArray_tag {
    mxClassID cls;
    bool cplx;
    size_t m, n;
    void* data;
};

extern "C" {
bool mxIsSingle(const mxArray* a) { return a->cls == mxSINGLE_CLASS; }
bool mxIsDouble(const mxArray* a) { return a->cls == mxDOUBLE_CLASS; }
bool mxIsComplex(const mxArray* a) { return a->cplx; }
size_t mxGetNumberOfElements(const mxArray* a) { return a->m * a->n; }
size_t mxGetM(const mxArray* a) { return a->m; }
size_t mxGetN(const mxArray* a) { return a->n; }
double mxGetScalar(const mxArray* a) {
    return a->cls == mxDOUBLE_CLASS ? *(double*)a->data : (double)*(float*)a->data;
}
float* mxGetSingles(const mxArray* a) { return (float*)a->data; }
mxComplexSingle* mxGetComplexSingles(const mxArray* a) { return (mxComplexSingle*)a->data; }
mxArray* mxCreateNumericArray(mwSize ndim, const mwSize* dims, mxClassID cls, mxComplexity cplx) {
    mxArray* a = new mxArray_tag{cls, cplx == mxCOMPLEX, dims[0], ndim > 1 ? dims[1] : 1, nullptr};
    const size_t esz = (cls == mxDOUBLE_CLASS ? 8 : 4) * (a->cplx ? 2 : 1);
    a->data = std::calloc(a->m * a->n, esz);
    return a;
}
void* mxMalloc(size_t n) { return std::malloc(n); }
void mxFree(void* p) { std::free(p); }
void mexErrMsgIdAndTxt(const char* id, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::fprintf(stderr, "%s: ", id);
    std::vfprintf(stderr, fmt, ap);
    std::fprintf(stderr, "\n");
    va_end(ap);
    std::exit(3);
}
void mexWarnMsgIdAndTxt(const char*, const char*, ...) {}
static void (*g_atexit)(void) = nullptr;
int mexAtExit(void (*fn)(void)) {
    g_atexit = fn;
    return 0;
}
}

static mxArray* scalar(double v) {
    mwSize d[2] = {1, 1};
    mxArray* a = mxCreateNumericArray(2, d, mxDOUBLE_CLASS, mxREAL);
    *(double*)a->data = v;
    return a;
}

int main(int argc, char** argv) {
    if (argc != 9) return 2;
    const size_t n = std::strtoul(argv[2], nullptr, 10);
    mwSize d[2] = {1, n};
    mxArray* x = mxCreateNumericArray(2, d, mxSINGLE_CLASS, mxREAL);
    FILE* f = std::fopen(argv[1], "rb");
    if (!f || std::fread(x->data, 4, n, f) != n) return 2;
    std::fclose(f);
    const mxArray* in[7] = {x, scalar(std::atof(argv[3])), scalar(std::atof(argv[4])), scalar(std::atof(argv[5])),
                            scalar(std::atof(argv[6])), scalar(std::atof(argv[7])), scalar(8)};
    mxArray* out[2] = {nullptr, nullptr};
    mexFunction(2, out, 7, in);
    FILE* o = std::fopen(argv[8], "wb");
    std::fwrite(out[0]->data, 8, out[0]->m * out[0]->n, o);
    std::fwrite(out[1]->data, 4, out[1]->m * out[1]->n, o);
    std::fclose(o);
    if (g_atexit) g_atexit();
    return 0;
}
