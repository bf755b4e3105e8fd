// C++ drop-in classes (include/fcwt.h) over the C ABI (include/fcwt_b200.h).
#include "fcwt.h"

#include <cstdlib>
#include <cstring>
#include <iostream>
#include <stdexcept>
#include <string>

#include "fcwt_b200.h"

namespace {

// One context per calling thread, created on first use on device 0 (or the
// device named by FCWT_DEVICE).
struct ThreadContext {
    fcwt_context* ctx = nullptr;
    ~ThreadContext() {
        if (ctx) fcwt_context_destroy(ctx);
    }
    fcwt_context* get() {
        if (!ctx) {
            const char* d = std::getenv("FCWT_DEVICE");
            int dev = d ? std::atoi(d) : 0;
            if (fcwt_context_create(dev, &ctx) != FCWT_OK) {
                ctx = nullptr;
                throw std::runtime_error(std::string("fcwt: ") + fcwt_last_error());
            }
        }
        return ctx;
    }
};

thread_local ThreadContext t_ctx;

// FCWT_STRICT=1 in the environment turns on the Nyquist checks the reference
// makes with (release-disabled) asserts, src/fcwt/fcwt.cpp:148,167,184.
unsigned strict_flag() {
    const char* v = std::getenv("FCWT_STRICT");
    return (v && v[0] && v[0] != '0') ? FCWT_STRICT : 0u;
}

void check(int rc) {
    if (rc != FCWT_OK) throw std::runtime_error(std::string("fcwt: ") + fcwt_last_error());
}

}  // namespace

// ---- Wavelet base: the reference prints an error for the unimplemented virtuals
void Wavelet::generate(float*, float*, int, float) { std::printf("ERROR [generate time complex]: Override this virtual class"); }
void Wavelet::generate(int) { std::printf("ERROR [generate freq]: Override this virtual class"); }
int Wavelet::getSupport(float) {
    std::printf("ERROR [getsupport]: Override this virtual class");
    return 0;
}
void Wavelet::getWavelet(float, std::complex<float>*, int) { std::printf("ERROR [getsupport]: Override this virtual class"); }

// ---- Morlet (src/fcwt/fcwt.cpp:41-105)
Morlet::Morlet(float bandwidth) {
    four_wavelen = 0.9876f;
    fb = bandwidth;
    fb2 = 2.0f * fb * fb;
    ifb = 1.0f / fb;
    imag_frequency = false;
    doublesided = false;
    mother = nullptr;
}

Morlet::~Morlet() { std::free(mother); }

void Morlet::generate(int size) {
    width = size;
    std::free(mother);
    mother = (float*)std::malloc(sizeof(float) * (size_t)(size > 0 ? size : 1));
    if (!mother) throw std::bad_alloc();
    if (size > 0) check(fcwt_morlet_mother(t_ctx.get(), fb, size, mother));
}

void Morlet::generate(float* real, float* imag, int size, float scale) {
    width = getSupport(scale);
    check(fcwt_morlet_time(fb, scale, size, real, imag));
}

int Morlet::getSupport(float scale) { return fcwt_morlet_support(fb, scale); }

void Morlet::getWavelet(float scale, std::complex<float>* pwav, int pn) {
    check(fcwt_morlet_wavelet(fb, scale, reinterpret_cast<float*>(pwav), pn));
}

// ---- Scales (src/fcwt/fcwt.cpp:111-137)
Scales::Scales(Wavelet* wav, SCALETYPE st, int afs, float af0, float af1, int afn) {
    fs = afs;
    fourwavl = wav ? wav->four_wavelen : 0.9876f;
    nscales = afn;
    scales = (float*)std::malloc(sizeof(float) * (size_t)(afn > 0 ? afn : 1));
    if (!scales) throw std::bad_alloc();
    const int rc = fcwt_scales_checked((int)st, afs, af0, af1, afn, strict_flag(), scales);
    if (rc == FCWT_ERR_INVALID) {
        std::free(scales);
        throw std::invalid_argument(std::string("fcwt: ") + fcwt_last_error());
    }
    check(rc);
}

Scales::~Scales() { std::free(scales); }

void Scales::getScales(float* pfreqs, int pnf) {
    for (int i = 0; i < pnf; i++) pfreqs[i] = scales[i];
}

void Scales::getFrequencies(float* pfreqs, int pnf) { check(fcwt_frequencies(scales, pnf, fs, pfreqs)); }

// ---- FCWT (src/fcwt/fcwt.h:114-152, src/fcwt/fcwt.cpp:313-548)
FCWT::FCWT(Wavelet* pwav, int pthreads, bool puse_optimalization_schemes, bool puse_normalization)
    : wavelet(pwav),
      threads(pthreads),
      use_optimalization_schemes(puse_optimalization_schemes),
      use_normalization(puse_normalization) {}

void FCWT::create_FFT_optimization_plan(int pmaxsize, int flags) {
    // FFTW flag values: ESTIMATE 1<<6, MEASURE 0, PATIENT 1<<5, EXHAUSTIVE 1<<3.
    int level = 1;
    if (flags & (1 << 6))
        level = 0;
    else if (flags & (1 << 3))
        level = 3;
    else if (flags & (1 << 5))
        level = 2;
    if (find2power(pmaxsize) <= 10)
        std::cerr << "Maxsize is too small (<=1024)... please use a larger number" << std::endl;
    check(fcwt_create_optimization_plan(t_ctx.get(), pmaxsize, threads, level, nullptr));
}

void FCWT::create_FFT_optimization_plan(int pmaxsize, std::string flags) {
    int flag;
    if (flags == "FFTW_MEASURE")
        flag = 0;
    else if (flags == "FFTW_PATIENT")
        flag = 1 << 5;
    else if (flags == "FFTW_EXHAUSTIVE")
        flag = 1 << 3;
    else if (flags == "FFTW_ESTIMATE")
        flag = 1 << 6;
    else {
        std::cerr << "Unknown flag: " << flags << std::endl;
        return;
    }
    create_FFT_optimization_plan(pmaxsize, flag);
}

void FCWT::run(const void* input, bool complexinput, int psize, std::complex<float>* poutput, Scales* scales) {
    Morlet* m = dynamic_cast<Morlet*>(wavelet);
    if (!wavelet) throw std::runtime_error("fcwt: null Wavelet");
    if (!scales) throw std::runtime_error("fcwt: null Scales");
    fcwt_context* ctx = t_ctx.get();
    if (use_optimalization_schemes) {
        const int N = 1 << find2power(psize);
        if (N <= 1024) {
            std::cout << "Inputsize is too small (N <= 1024) to use optimization." << std::endl;
        } else if (fcwt_load_optimization_plan(ctx, psize, threads, nullptr) != FCWT_OK) {
            std::cout << "WARNING: Optimization scheme 'n" << N << "_t" << threads
                      << ".wis' was not found, fallback to calculation without optimization." << std::endl;
        }
    }
    const unsigned flags = (use_normalization ? FCWT_NORM : 0u) | strict_flag();
    const float* in = reinterpret_cast<const float*>(input);
    if (!m) {
        // any other Wavelet: the table its generate(N) fills and its imag_frequency /
        // doublesided fields, as the reference uses them (src/fcwt/fcwt.cpp:396-429, 504-505)
        const int N = 1 << find2power(psize);
        wavelet->generate(N);
        if (!wavelet->mother) throw std::runtime_error("fcwt: Wavelet::generate(N) left mother empty");
        const unsigned kind = (wavelet->imag_frequency ? FCWT_IMAG_FREQUENCY : 0u) |
                              (wavelet->doublesided ? FCWT_DOUBLESIDED : 0u);
        check(fcwt_cwt_mother(ctx, input, psize, complexinput ? 1 : 0, wavelet->mother, N, scales->scales,
                              scales->nscales, threads, flags | kind, poutput, FCWT_OUT_C64));
        check(fcwt_synchronize(ctx));
        return;
    }
    int rc = complexinput
                 ? fcwt_ccwt(ctx, in, psize, m->fb, scales->scales, scales->nscales, threads, flags, poutput, FCWT_OUT_C64)
                 : fcwt_cwt(ctx, in, psize, m->fb, scales->scales, scales->nscales, threads, flags, poutput, FCWT_OUT_C64);
    check(rc);
    check(fcwt_synchronize(ctx));
}

void FCWT::cwt(float* pinput, int psize, std::complex<float>* poutput, Scales* scales) {
    run(pinput, false, psize, poutput, scales);
}

void FCWT::cwt(std::complex<float>* pinput, int psize, std::complex<float>* poutput, Scales* scales) {
    run(pinput, true, psize, poutput, scales);
}

void FCWT::cwt(float* pinput, int psize, Scales* scales, std::complex<float>* poutput, int pn1, int pn2) {
    if ((long long)psize * scales->nscales != (long long)pn1 * pn2)
        throw std::runtime_error("fcwt: output shape does not match n * nscales");
    run(pinput, false, psize, poutput, scales);
}

void FCWT::cwt(std::complex<float>* pinput, int psize, Scales* scales, std::complex<float>* poutput, int pn1,
               int pn2) {
    if ((long long)psize * scales->nscales != (long long)pn1 * pn2)
        throw std::runtime_error("fcwt: output shape does not match n * nscales");
    run(pinput, true, psize, poutput, scales);
}
