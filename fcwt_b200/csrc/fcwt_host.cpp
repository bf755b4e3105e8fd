// Host-side arithmetic of the fCWT transform path: scale grids, the Morlet
// mother table and time-domain wavelet, and the per-row truncation rule.
//
// Every function keeps the reference's float/double operation order so that
// the results are bit-identical to the reference CPU build (compiled with
// -ffp-contract=off; the reference is built with -mavx and no FMA, so no
// contraction happens there either). Citations are to src/fcwt/fcwt.cpp and
// src/fcwt/fcwt.h of the reference.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fcwt_internal.h"

namespace fcwt {
namespace host {

// Same float literals as the reference's PI and IPI4 macros (fcwt.h:59-61).
static const float kPi = 3.14159265358979323846f;
static const float kIpi4 = 0.75112554446f;

// Smallest m with 2^m >= n (fcwt.h:154-165).
int find2power(int n) {
    int m = 0, m2 = 1;
    while (m2 - n < 0) {
        m++;
        m2 <<= 1;
    }
    return m;
}

// Scales::calculate_{log,lin}scale_array / calculate_linfreq_array
// (fcwt.cpp:139-190). scaletype: 0 LINSCALES, 1 LOGSCALES, 2 LINFREQS.
void scales(int scaletype, int fs, float f0, float f1, int fn, float* out) {
    if (scaletype == 1) {
        const float base = 2.0f;
        float s0 = (fs / f1);
        float s1 = (fs / f0);
        float power0 = std::log(s0) / std::log(base);
        float power1 = std::log(s1) / std::log(base);
        float dpower = power1 - power0;
        for (int i = 0; i < fn; i++) {
            float power = power0 + (dpower / (fn - 1)) * i;
            out[i] = std::pow(base, power);
        }
    } else if (scaletype == 0) {
        float s0 = fs / f1;
        float s1 = fs / f0;
        float ds = s1 - s0;
        for (int i = 0; i < fn; i++) out[i] = (s0 + (ds / fn) * i);
    } else {
        float df = f1 - f0;
        for (int i = 0; i < fn; i++) out[fn - i - 1] = (((float)fs) / (f0 + (df / fn) * (float)i));
    }
}

// Scales::getFrequencies (fcwt.cpp:133-137).
void frequencies(const float* sc, int fn, int fs, float* out) {
    for (int i = 0; i < fn; i++) out[i] = ((float)fs) / sc[i];
}

// norm factor of Morlet::generate(int) (fcwt.cpp:57): sqrt(2*PI)*IPI4 in float.
float mother_norm() { return std::sqrt(2 * kPi) * kIpi4; }

// Morlet::generate(int) (fcwt.cpp:51-67), frequency-domain mother table.
void mother_table(float fb, int N, float* out) {
    float toradians = (2 * kPi) / (float)N;
    float norm = mother_norm();
    for (int w = 0; w < N; w++) {
        float tmp1 = (2.0f * ((float)w * toradians) * fb - 2.0f * kPi * fb);
        tmp1 = -(tmp1 * tmp1) / 2;
        out[w] = (norm * std::exp(tmp1));
    }
}

// Morlet::getSupport (fcwt.h:88).
int morlet_support(float fb, float scale) { return (int)(fb * scale * 3.0f); }

// Morlet::generate(real, imag, size, scale) (fcwt.cpp:68-84): 2*width+1 taps.
void morlet_time(float fb, float scale, int size, float* real, float* imag) {
    float ifb = 1.0f / fb;
    float fb2 = 2.0f * fb * fb;
    int width = morlet_support(fb, scale);
    float norm = (float)size * ifb * kIpi4;
    for (int t = 0; t < width * 2 + 1; t++) {
        float tmp1 = (float)(t - width) / scale;
        float tmp2 = std::exp(-(tmp1 * tmp1) / (fb2));
        real[t] = norm * tmp2 * std::cos(tmp1 * 2.0f * kPi) / scale;
        imag[t] = norm * tmp2 * std::sin(tmp1 * 2.0f * kPi) / scale;
    }
}

// Morlet::getWavelet (fcwt.cpp:86-105): pn interleaved complex taps.
void morlet_wavelet(float fb, float scale, int pn, float* out_interleaved) {
    int w = morlet_support(fb, scale);
    int len = (w * 2 + 1) > pn ? (w * 2 + 1) : pn;
    std::vector<float> re((size_t)len, 0.0f), im((size_t)len, 0.0f);
    morlet_time(fb, scale, pn, re.data(), im.data());
    for (int t = 0; t < pn; t++) {
        out_interleaved[2 * t] = re[(size_t)t];
        out_interleaved[2 * t + 1] = im[(size_t)t];
    }
}

// Truncation length of one scale in daughter_wavelet_multiplication
// (fcwt.cpp:199-203 and 213-214 for the AVX build, 277-278 for the scalar
// build): the number of leading bins the reference multiplies for this scale.
int row_proc(int N, float scale, int threads, bool avx) {
    float isizef = ((float)(N));
    float endpointf = std::fmin(isizef / 2.0, ((isizef * 2.0) / scale));
    int endpoint = ((int)endpointf);
    if (avx) {
        int endpoint4 = endpoint >> 2;
        int a = endpoint4 / 16;
        int athreads = threads < (a > 1 ? a : 1) ? threads : (a > 1 ? a : 1);
        int batchsize = (endpoint4 / athreads);
        return 4 * batchsize * athreads;
    }
    int a = endpoint / 16;
    int athreads = threads < (a > 1 ? a : 1) ? threads : (a > 1 ? a : 1);
    int batchsize = (endpoint / athreads);
    return batchsize * athreads;
}

// `float step = (scale/2.0)` (fcwt.cpp:201).
float row_step(float scale) { return (float)(scale / 2.0); }

// Mother-table index of bin q (fcwt.cpp:225-240, 290-293):
// (int)min((float)(N-1), step * (float)q).
int row_index(int N, float step, int q) {
    float maximum = (float)N - 1;
    float t = step * (float)q;
    return (int)(maximum < t ? maximum : t);
}

}  // namespace host
}  // namespace fcwt
