/*
 * fcwt_oracle.c — CPU restatement of the reference fCWT transform semantics.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker: only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it. The
 * product (fcwt_b200) never links, loads or calls it.
 *
 * It restates, in plain C with the reference's float/double operation order
 * (compile with -O2 -ffp-contract=off; the reference is built with -mavx and
 * no FMA, so no contraction happens there either):
 *   - find2power                         src/fcwt/fcwt.h:154-165
 *   - Scales: LOG / LIN / LINFREQ arrays src/fcwt/fcwt.cpp:139-190
 *   - Scales::getFrequencies             src/fcwt/fcwt.cpp:133-137
 *   - Morlet::generate(int)              src/fcwt/fcwt.cpp:51-67
 *   - Morlet::generate(re,im,size,scale) src/fcwt/fcwt.cpp:68-84
 *   - Morlet::getWavelet / getSupport    src/fcwt/fcwt.cpp:86-105, fcwt.h:88
 *   - daughter_wavelet_multiplication: truncation length `proc` and the
 *     mother-table index of every bin, AVX path (the one the reference ships,
 *     CMakeLists.txt:56, setup.py:45) and scalar path   src/fcwt/fcwt.cpp:197-311
 *   - the O1 buffer reuse across scales (bins >= proc keep the previous
 *     scale's product; fcwt.cpp:459-467, 514-518), expressed as a per-row
 *     effective weight vector W_i[q] with O1_i[q] = Ihat[q] * W_i[q].
 *
 * The FFTs themselves (FFTW in the reference) are done by the Python side of
 * the oracle in float64 (numpy), see oracle/oracle.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_PI 3.14159265358979323846264338327950288419716939937510582097494459072381640628620899862803482534211706798f
#define OR_IPI4 0.75112554446f

int or_find2power(int n) {
    int m = 0, m2 = 1;
    while (m2 - n < 0) {
        m++;
        m2 <<= 1;
    }
    return m;
}

/* scaletype: 0 = LINSCALES, 1 = LOGSCALES, 2 = LINFREQS (enum order, fcwt.h:65) */
void or_scales(int scaletype, int fs, float f0, float f1, int fn, float* scales) {
    if (scaletype == 1) {
        float base = 2.0f;
        float s0 = (fs / f1);
        float s1 = (fs / f0);
        float power0 = logf(s0) / logf(base);
        float power1 = logf(s1) / logf(base);
        float dpower = power1 - power0;
        for (int i = 0; i < fn; i++) {
            float power = power0 + (dpower / (fn - 1)) * i;
            scales[i] = powf(base, power);
        }
    } else if (scaletype == 0) {
        float s0 = fs / f1;
        float s1 = fs / f0;
        float ds = s1 - s0;
        for (int i = 0; i < fn; i++) scales[i] = (s0 + (ds / fn) * i);
    } else {
        float df = f1 - f0;
        for (int i = 0; i < fn; i++) scales[fn - i - 1] = (((float)fs) / (f0 + (df / fn) * (float)i));
    }
}

void or_frequencies(const float* scales, int fn, int fs, float* freqs) {
    for (int i = 0; i < fn; i++) freqs[i] = ((float)fs) / scales[i];
}

void or_mother(float fb, int size, float* mother) {
    float toradians = (2 * OR_PI) / (float)size;
    float norm = sqrtf(2 * OR_PI) * OR_IPI4;
    for (int w = 0; w < size; w++) {
        float tmp1 = (2.0f * ((float)w * toradians) * fb - 2.0f * OR_PI * fb);
        tmp1 = -(tmp1 * tmp1) / 2;
        mother[w] = (norm * expf(tmp1));
    }
}

int or_support(float fb, float scale) { return (int)(fb * scale * 3.0f); }

/* Morlet::generate(real, imag, size, scale): time-domain wavelet of 2*width+1 taps. */
int or_wavelet_time(float fb, float scale, int size, float* real, float* imag) {
    float ifb = 1.0f / fb;
    float fb2 = 2.0f * fb * fb;
    int width = or_support(fb, scale);
    float norm = (float)size * ifb * OR_IPI4;
    for (int t = 0; t < width * 2 + 1; t++) {
        float tmp1 = (float)(t - width) / scale;
        float tmp2 = expf(-(tmp1 * tmp1) / (fb2));
        real[t] = norm * tmp2 * cosf(tmp1 * 2.0f * OR_PI) / scale;
        imag[t] = norm * tmp2 * sinf(tmp1 * 2.0f * OR_PI) / scale;
    }
    return width;
}

/* Morlet::getWavelet(scale, pwav, pn): interleaved complex output of pn taps. */
void or_get_wavelet(float fb, float scale, int pn, float* out_interleaved) {
    int w = or_support(fb, scale);
    int len = (w * 2 + 1) > pn ? (w * 2 + 1) : pn;
    float* re = (float*)calloc((size_t)len, sizeof(float));
    float* im = (float*)calloc((size_t)len, sizeof(float));
    or_wavelet_time(fb, scale, pn, re, im);
    for (int t = 0; t < pn; t++) {
        out_interleaved[2 * t] = re[t];
        out_interleaved[2 * t + 1] = im[t];
    }
    free(re);
    free(im);
}

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

/* Number of leading bins written for one scale (the truncation length).
 * avx != 0: AVX path, bins handled in groups of 4 per thread batch.
 * avx == 0: scalar path. */
int or_proc(int isize, float scale, int threads, int avx) {
    float isizef = ((float)(isize));
    float endpointf = fmin(isizef / 2.0, ((isizef * 2.0) / scale));
    int endpoint = ((int)endpointf);
    if (avx) {
        int endpoint4 = endpoint >> 2;
        int athreads = imin(threads, imax(1, endpoint4 / 16));
        int batchsize = (endpoint4 / athreads);
        return 4 * batchsize * athreads;
    } else {
        int athreads = imin(threads, imax(1, endpoint / 16));
        int batchsize = (endpoint / athreads);
        return batchsize * athreads;
    }
}

/* Mother-table index of bin q for one scale (AVX and scalar paths agree). */
int or_index(int isize, float scale, int q) {
    float isizef = ((float)(isize));
    float step = (scale / 2.0);
    float maximum = isizef - 1;
    float t = step * (float)q;
    float m = maximum < t ? maximum : t;
    return (int)m;
}

/* Effective weights: W[i*half + q] for rows i < fn and bins q < half, where
 * half = isize/2. Bins >= proc_i keep the weight of the most recent earlier row
 * that wrote them (0 if none), exactly as the reused O1 buffer does. Also
 * returns each row's proc in procs[] (may be NULL). */
void or_weights(int isize, const float* scales, int fn, int threads, int avx, const float* mother,
                float* W, int* procs) {
    int half = isize / 2;
    float* state = (float*)calloc((size_t)(half > 0 ? half : 1), sizeof(float));
    for (int i = 0; i < fn; i++) {
        int p = or_proc(isize, scales[i], threads, avx);
        if (procs) procs[i] = p;
        for (int q = 0; q < p && q < half; q++) state[q] = mother[or_index(isize, scales[i], q)];
        memcpy(W + (size_t)i * half, state, sizeof(float) * (size_t)half);
    }
    free(state);
}

/* Same as or_weights but only materialises the selected rows (sel[k] < fn,
 * ascending): W[k*half + q] is the weight vector of row sel[k]. */
void or_weights_rows(int isize, const float* scales, int fn, int threads, int avx, const float* mother,
                     const int* sel, int nsel, float* W) {
    int half = isize / 2;
    float* state = (float*)calloc((size_t)(half > 0 ? half : 1), sizeof(float));
    int k = 0;
    for (int i = 0; i < fn && k < nsel; i++) {
        int p = or_proc(isize, scales[i], threads, avx);
        for (int q = 0; q < p && q < half; q++) state[q] = mother[or_index(isize, scales[i], q)];
        while (k < nsel && sel[k] == i) {
            memcpy(W + (size_t)k * half, state, sizeof(float) * (size_t)half);
            k++;
        }
    }
    free(state);
}
