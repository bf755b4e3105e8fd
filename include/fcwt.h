// fcwt.h — C++ drop-in API of the B200 fCWT transform path.
//
// Same classes, public members and member-function signatures as the
// reference's public header (src/fcwt/fcwt.h:65-165 of fastlib/fCWT), so code
// written against the reference compiles and links against libfcwt_b200.so
// unchanged. The transform runs on the GPU through the C ABI in fcwt_b200.h;
// input and output pointers may be host or device memory.
//
// Like the reference header it defines PI, sqrt2PI and IPI4 and brings
// namespace std into scope (src/fcwt/fcwt.h:59-63), which code written
// against it relies on (e.g. `complex<float>` unqualified).
//
// Differences a caller can observe:
//   - Any Wavelet subclass works: FCWT::cwt runs on the table its
//     generate(N) fills, as the reference does (src/fcwt/fcwt.cpp:504-505);
//     Morlet tables are generated on the GPU.
//   - Errors (bad sizes, CUDA failures) throw std::runtime_error instead of
//     being ignored; with FCWT_STRICT=1 in the environment, frequencies above
//     fs/2 throw std::invalid_argument (the reference's asserts,
//     src/fcwt/fcwt.cpp:148,167,184, compiled out of its release builds).
//   - create_FFT_optimization_plan writes tuning files of the GPU engine under
//     the reference's file names (n<N>_t<threads>.wis).
#ifndef FCWT_H
#define FCWT_H

#include <complex>
#include <iostream>
#include <memory>
#include <string>

#define FCWT_LIBRARY_API

#define PI 3.14159265358979323846264338327950288f
#define sqrt2PI 2.50662827463100050241576528f
#define IPI4 0.75112554446f

using namespace std;

enum SCALETYPE { FCWT_LINSCALES, FCWT_LOGSCALES, FCWT_LINFREQS };

class Wavelet {
public:
    Wavelet() : width(0), four_wavelen(0.0f), imag_frequency(false), doublesided(false), mother(nullptr) {}
    virtual ~Wavelet() {}
    virtual void generate(float* real, float* imag, int size, float scale);
    virtual void generate(int size);
    virtual int getSupport(float scale);
    virtual void getWavelet(float scale, std::complex<float>* pwav, int pn);

    int width;
    float four_wavelen;
    bool imag_frequency, doublesided;
    float* mother;
};

class Morlet : public Wavelet {
public:
    FCWT_LIBRARY_API Morlet(float bandwidth);
    ~Morlet();

    void generate(int size);                                         // frequency domain, on the GPU
    void generate(float* real, float* imag, int size, float scale);  // time domain
    int getSupport(float scale);
    void getWavelet(float scale, std::complex<float>* pwav, int pn);
    float fb;

private:
    float ifb, fb2;
};

class Scales {
public:
    FCWT_LIBRARY_API Scales(Wavelet* pwav, SCALETYPE st, int fs, float f0, float f1, int fn);
    ~Scales();
    Scales(const Scales&) = delete;
    Scales& operator=(const Scales&) = delete;

    void FCWT_LIBRARY_API getScales(float* pfreqs, int pnf);
    void FCWT_LIBRARY_API getFrequencies(float* pfreqs, int pnf);

    float* scales;
    int fs;
    float fourwavl;
    int nscales;
};

class FCWT {
public:
    FCWT_LIBRARY_API FCWT(Wavelet* pwav, int pthreads, bool puse_optimalization_schemes,
                          bool puse_normalization);

    void FCWT_LIBRARY_API create_FFT_optimization_plan(int pmaxsize, int poptimizationflags);
    void FCWT_LIBRARY_API create_FFT_optimization_plan(int pmaxsize, std::string poptimizationflags);
    void FCWT_LIBRARY_API cwt(float* pinput, int psize, std::complex<float>* poutput, Scales* scales);
    void FCWT_LIBRARY_API cwt(std::complex<float>* pinput, int psize, std::complex<float>* poutput,
                              Scales* scales);
    void FCWT_LIBRARY_API cwt(float* pinput, int psize, Scales* scales, std::complex<float>* poutput,
                              int pn1, int pn2);
    void FCWT_LIBRARY_API cwt(std::complex<float>* pinput, int psize, Scales* scales,
                              std::complex<float>* poutput, int pn1, int pn2);

    Wavelet* wavelet;

private:
    void run(const void* input, bool complexinput, int psize, std::complex<float>* poutput, Scales* scales);
    int threads;
    bool use_optimalization_schemes;
    bool use_normalization;
};

inline int find2power(int n) {
    int m = 0, m2 = 1;
    while (m2 - n < 0) {
        m++;
        m2 <<= 1;
    }
    return m;
}

#endif
