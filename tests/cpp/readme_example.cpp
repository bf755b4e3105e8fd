// The reference README's C++ call sequence (fastlib/fCWT README.md:139-214),
// compiled against include/fcwt.h and linked with libfcwt_b200.so by
// tests/test_cpp_dropin.py. Test infrastructure.
//
//   readme_example host <out.bin>   host-only parts: Scales, getFrequencies,
//                                   Morlet time domain, FCWT_STRICT behaviour
//   readme_example gpu <out.bin>    the README transform: 100k samples, 3000
//                                   LINFREQS 1-32 Hz, Morlet(2), 8 threads,
//                                   optplan on, normalisation off
// Writes raw float32 / complex64 arrays the Python side checks.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <fcwt.h>

static void put(FILE* f, const void* p, size_t bytes) {
    if (fwrite(p, 1, bytes, f) != bytes) std::exit(3);
}

int main(int argc, char* argv[]) {
    if (argc < 3) return 2;
    FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 2;
    if (std::strcmp(argv[1], "host") == 0) {
        Morlet morl(2.0f);
        Wavelet* wavelet = &morl;
        Scales scs(wavelet, FCWT_LOGSCALES, 1000, 1.0f, 101.0f, 300);
        std::vector<float> sc(300), fr(300);
        scs.getScales(sc.data(), 300);
        scs.getFrequencies(fr.data(), 300);
        put(f, sc.data(), sizeof(float) * 300);
        put(f, fr.data(), sizeof(float) * 300);
        const int sup = morl.getSupport(10.0f);
        std::vector<float> re(2 * sup + 1), im(2 * sup + 1);
        morl.generate(re.data(), im.data(), 2 * sup + 1, 10.0f);
        put(f, &sup, sizeof(int));
        put(f, re.data(), sizeof(float) * re.size());
        put(f, im.data(), sizeof(float) * im.size());
        // above Nyquist: accepted by default (the release build's behaviour), refused under FCWT_STRICT=1
        int strict_threw = 0;
        try {
            Scales bad(wavelet, FCWT_LINFREQS, 100, 1.0f, 101.0f, 10);
        } catch (const std::invalid_argument&) {
            strict_threw = 1;
        }
        put(f, &strict_threw, sizeof(int));
        std::fclose(f);
        return 0;
    }
    // ---- README.md:146-211, unchanged apart from the output file
    int n = 100000;  // signal length
    const int fs = 1000;
    float twopi = 2.0 * 3.1415;
    const float f0 = 1;
    const float f1 = 32;
    const int fn = 3000;
    const int nthreads = 8;
    std::vector<float> sig(n);
    std::vector<complex<float>> tfm(n * fn);
    for (auto& el : sig) {
        el = cos(twopi * ((float)(&el - &sig[0]) / (float)fs));
    }
    Wavelet* wavelet;
    Morlet morl(2.0f);
    wavelet = &morl;
    FCWT fcwt(wavelet, nthreads, true, false);
    Scales scs(wavelet, FCWT_LINFREQS, fs, f0, f1, fn);
    fcwt.cwt(&sig[0], n, &tfm[0], &scs);
    // sampled rows for the checker
    const int rows[3] = {0, fn / 2, fn - 1};
    put(f, sig.data(), sizeof(float) * n);
    put(f, scs.scales, sizeof(float) * fn);
    for (int r : rows) put(f, &tfm[(size_t)r * n], sizeof(complex<float>) * n);
    std::fclose(f);
    return 0;
}
