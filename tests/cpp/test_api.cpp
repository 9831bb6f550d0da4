// C++ client of the MetalFFT mirror (metalfft_b200/MetalFFT.hpp), written like
// the reference's XCTests (Tests/MetalFFTTests/MetalFFTTests.swift): impulse
// -> all ones, batch == single, round trip, FFTError cases, a delta-kernel
// convolution and an autocorrelation peak.  Prints "OK" and exits 0 on success.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "../../metalfft_b200/MetalFFT.hpp"

#define EXPECT(c)                                                    \
    do {                                                             \
        if (!(c)) {                                                  \
            std::fprintf(stderr, "FAIL %s:%d %s\n", __FILE__, __LINE__, #c); \
            std::exit(1);                                            \
        }                                                            \
    } while (0)

int main() {
    using namespace mfft;
    for (int64_t n : {64, 512, 4096, 16384, 1 << 20}) {
        MetalFFT f(n);
        std::vector<cfloat> x((size_t)n, cfloat(0.f, 0.f));
        x[0] = cfloat(1.f, 0.f);
        auto y = f.forward(x);
        for (auto v : y) EXPECT(std::abs(v - cfloat(1.f, 0.f)) < 1e-5f);
        auto z = f.inverse(y);
        EXPECT(std::abs(z[0] - cfloat(1.f, 0.f)) < 1e-5f && std::abs(z[1]) < 1e-5f);
        // adjoint of the forward: F^H (all ones) = n * impulse
        auto g = f.backward(y, MFFT_FORWARD);
        EXPECT(std::abs(g[0] - cfloat((float)n, 0.f)) < 1e-5f * (float)n && std::abs(g[1]) < 1e-5f * (float)n);
    }
    {
        MetalFFT f(512);
        std::vector<std::vector<cfloat>> xs(2, std::vector<cfloat>(512));
        for (int i = 0; i < 512; ++i) {
            xs[0][i] = cfloat(std::sin(0.1f * i), 0.f);
            xs[1][i] = cfloat(std::cos(0.3f * i), 0.5f);
        }
        auto yb = f.forwardBatch(xs);
        auto y0 = f.forward(xs[0]);
        for (int i = 0; i < 512; ++i) EXPECT(yb[0][i] == y0[i]);
        bool thrown = false;
        try {
            f.forward(std::vector<cfloat>(100));
        } catch (const FFTError& e) {
            thrown = (e.status() == MFFT_ERR_INVALID_INPUT_SIZE && e.expected() == 512 && e.got() == 100);
        }
        EXPECT(thrown);
        thrown = false;
        try {
            xs[1].resize(7);
            f.forwardBatch(xs);
        } catch (const FFTError& e) {
            thrown = (e.status() == MFFT_ERR_BATCH_INPUT_SIZE && e.batchIndex() == 1);
        }
        EXPECT(thrown);
    }
    {
        bool thrown = false;
        try {
            MetalFFT bad(100);
        } catch (const FFTError& e) {
            thrown = std::string(e.caseName()) == "unsupportedFFTSize";
        }
        EXPECT(thrown);
    }
    {
        std::vector<float> delta(64, 0.f);
        delta[0] = 1.f;
        Convolver c(delta, 4096);
        std::vector<float> s((size_t)c.hopSize());
        for (size_t i = 0; i < s.size(); ++i) s[i] = std::sin(0.01f * (float)i);
        auto y = c.apply(s);
        EXPECT(y.size() == s.size() + 63);
        for (size_t i = 0; i < s.size(); ++i) EXPECT(std::fabs(y[i] - s[i]) < 1e-5f);
        EXPECT(Convolver::recommendedFFTSize(100) == 128);
    }
    {
        Correlator corr(256);
        std::vector<float> x(100);
        double e = 0;
        for (int i = 0; i < 100; ++i) {
            x[i] = std::sin(0.37f * i) + 0.1f * (float)(i % 7);
            e += (double)x[i] * x[i];
        }
        auto r = corr.autocorrelation(x);
        EXPECT(std::fabs(r[0] - e) < 1e-3 * e);
        for (size_t i = 1; i < r.size(); ++i) EXPECT(r[i] <= r[0]);
    }
    {
        FFTAnalyzer an(1024, 1024.0, MFFT_WINDOW_RECTANGULAR);
        std::vector<float> s(1024);
        for (int i = 0; i < 1024; ++i) s[i] = std::cos(2.0 * M_PI * 100 * i / 1024.0);
        auto X = an.analyze(s);
        int peak = 0;
        for (int i = 1; i < 512; ++i)
            if (std::norm(X[i]) > std::norm(X[peak])) peak = i;
        EXPECT(peak == 100);
    }
    std::printf("OK\n");
    return 0;
}
