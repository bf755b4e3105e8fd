// C entry points over the reference fCWT C++ classes, so that Python (ctypes)
// can drive the reference's own CPU path (FFTW + AVX) as the parity oracle and
// as the timed CPU baseline.
//
// This file is test infrastructure. It is compiled together with the
// reference's src/fcwt/fcwt.cpp (never copied) by oracle/build_ref.sh into
// oracle/_ref/libfcwt_ref.so. Nothing in the product links or loads it.
//
// Each function mirrors one reference call sequence:
//   ref_scales      -> Scales::Scales + Scales::getScales      (src/fcwt/fcwt.cpp:111-158)
//   ref_frequencies -> Scales::getFrequencies                  (src/fcwt/fcwt.cpp:133-137)
//   ref_mother      -> Morlet::generate(int)                   (src/fcwt/fcwt.cpp:51-67)
//   ref_wavelet     -> Morlet::getWavelet                      (src/fcwt/fcwt.cpp:86-105)
//   ref_cwt         -> FCWT::cwt (real or complex input)       (src/fcwt/fcwt.cpp:447-548)
//   ref_create_plan -> FCWT::create_FFT_optimization_plan      (src/fcwt/fcwt.cpp:313-374)
//   ref_cwt_table   -> FCWT::cwt with a Wavelet subclass whose generate(N)
//                      fills `mother` from a caller table (the reference's
//                      Wavelet interface, src/fcwt/fcwt.h:67-79)
//   ref_daughter    -> FCWT::daughter_wavelet_multiplication, the per-scale
//                      product into the reused O1 buffer (src/fcwt/fcwt.cpp:197-311),
//                      row after row like FCWT::cwt (fcwt.cpp:514-518)
//
// daughter_wavelet_multiplication is a private member of FCWT. To call it, the
// reference header is included with `private` defined as `public` (the
// standard and FFTW headers it includes are included first, untouched).
#include <complex>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <string>
#include <unistd.h>
#include <omp.h>
#include <immintrin.h>
#include "fftw3.h"

#define private public
#include "fcwt.h"
#undef private

extern "C" {

int ref_find2power(int n) { return find2power(n); }

void ref_scales(float fb, int scaletype, int fs, float f0, float f1, int fn, float* out) {
    Morlet m(fb);
    Scales s(&m, (SCALETYPE)scaletype, fs, f0, f1, fn);
    s.getScales(out, fn);
    free(s.scales);
}

void ref_frequencies(float fb, int scaletype, int fs, float f0, float f1, int fn, float* out) {
    Morlet m(fb);
    Scales s(&m, (SCALETYPE)scaletype, fs, f0, f1, fn);
    s.getFrequencies(out, fn);
    free(s.scales);
}

void ref_mother(float fb, int N, float* out) {
    Morlet m(fb);
    m.generate(N);
    std::memcpy(out, m.mother, sizeof(float) * (size_t)N);
}

int ref_support(float fb, float scale) {
    Morlet m(fb);
    return m.getSupport(scale);
}

void ref_wavelet(float fb, float scale, float* out_interleaved, int pn) {
    Morlet m(fb);
    m.getWavelet(scale, reinterpret_cast<std::complex<float>*>(out_interleaved), pn);
}

// Runs the reference transform with an explicit scales array. The Scales
// object is built with LOGSCALES and its public `scales` array is then
// overwritten, which is how the reference API lets a caller pass any grid.
void ref_cwt(const void* input, int n, int is_complex, float fb, const float* scales, int fn,
             int fs, int threads, int optplans, int norm, void* output) {
    Morlet m(fb);
    Scales s(&m, FCWT_LOGSCALES, fs, 1.0f, 2.0f, fn);
    std::memcpy(s.scales, scales, sizeof(float) * (size_t)fn);
    FCWT f(&m, threads, optplans != 0, norm != 0);
    if (is_complex) {
        f.cwt((std::complex<float>*)input, n, (std::complex<float>*)output, &s);
    } else {
        f.cwt((float*)input, n, (std::complex<float>*)output, &s);
    }
    free(s.scales);
}

// A wavelet given by its frequency-domain table (single-sided, real), as a
// user subclass of the reference's Wavelet would provide it.
class TableWavelet : public Wavelet {
public:
    TableWavelet(const float* t, int n, int kind) : table(t), size(n) {
        imag_frequency = (kind & 1) != 0;
        doublesided = (kind & 2) != 0;
        four_wavelen = 1.0f;
        mother = nullptr;
    }
    ~TableWavelet() { free(mother); }
    void generate(int n) override {
        free(mother);
        mother = (float*)malloc(sizeof(float) * (size_t)n);
        for (int i = 0; i < n; i++) mother[i] = i < size ? table[i] : 0.0f;
        width = n;
    }
    const float* table;
    int size;
};

// kind: bit 0 imag_frequency, bit 1 doublesided (the Wavelet fields the
// reference's product reads, src/fcwt/fcwt.cpp:396-429)
void ref_cwt_table(const void* input, int n, int is_complex, const float* table, int table_size,
                   const float* scales, int fn, int threads, int norm, int kind, void* output) {
    TableWavelet w(table, table_size, kind);
    Morlet m(2.0f);
    Scales s(&m, FCWT_LOGSCALES, 1000, 1.0f, 2.0f, fn);
    std::memcpy(s.scales, scales, sizeof(float) * (size_t)fn);
    FCWT f(&w, threads, false, norm != 0);
    if (is_complex) {
        f.cwt((std::complex<float>*)input, n, (std::complex<float>*)output, &s);
    } else {
        f.cwt((float*)input, n, (std::complex<float>*)output, &s);
    }
    free(s.scales);
}

// Runs FCWT(threads)::daughter_wavelet_multiplication for scales[0..fn) in
// order on one O1 buffer of N bins, with input `in` (N interleaved complex)
// and table `mother` (N floats), and stores O1 after each row into out[i]
// (N interleaved complex). reset != 0 fills O1 with NaN before every row (so
// bins the row does not write stay NaN); reset == 0 starts from zeros and keeps
// O1 across rows, as FCWT::cwt does.
void ref_daughter(int N, const float* scales, int fn, int threads, int imaginary, int doublesided, int reset,
                  const float* in, const float* mother, float* out) {
    Morlet m(2.0f);
    FCWT f(&m, threads, false, true);
    const size_t bytes = sizeof(fftwf_complex) * (size_t)N;
    fftwf_complex* I = (fftwf_complex*)aligned_alloc(32, (bytes + 31) & ~(size_t)31);
    fftwf_complex* O = (fftwf_complex*)aligned_alloc(32, (bytes + 31) & ~(size_t)31);
    std::memcpy(I, in, bytes);
    std::memset(O, 0, bytes);
    for (int i = 0; i < fn; i++) {
        if (reset)
            for (int q = 0; q < N; q++) O[q][0] = O[q][1] = __builtin_nanf("");
        f.daughter_wavelet_multiplication(I, O, mother, scales[i], N, imaginary != 0, doublesided != 0);
        std::memcpy(out + 2 * (size_t)N * (size_t)i, O, bytes);
    }
    free(I);
    free(O);
}

void ref_create_plan(float fb, int threads, int maxsize, const char* flag) {
    Morlet m(fb);
    FCWT f(&m, threads, true, true);
    f.create_FFT_optimization_plan(maxsize, std::string(flag));
}

}  // extern "C"
