// MetalFFT.hpp -- C++ mirror of the reference's Swift API over the C ABI of
// libmfft.so (include/mfft.h).  Header-only; link with -lmfft.
//
// Reference types (docs/MetalFFT.swiftinterface:12-266) and their mirrors:
//   FFTError        -> mfft::FFTError (exception; case() names the Swift case)
//   MetalFFT        -> mfft::MetalFFT: forward, forward(input, output),
//                      forwardBatch, inverse, backward (adjoint, no
//                      counterpart)
//   MultiChannelFFT -> mfft::MultiChannelFFT
//   Convolver       -> mfft::Convolver: apply, blockSize, hopSize,
//                      recommendedFFTSize
//   Correlator      -> mfft::Correlator: cross, autocorrelation
//   FFTAnalyzer     -> mfft::FFTAnalyzer: analyze(samples[, offset])
// Arrays are std::vector<std::complex<float>> / std::vector<float>, copied in
// and out like the Swift arrays (host-memory calls).
#pragma once

#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../include/mfft.h"

namespace mfft {

using cfloat = std::complex<float>;

class FFTError : public std::runtime_error {
   public:
    FFTError(int status, const std::string& msg, int64_t expected, int64_t got, int64_t index)
        : std::runtime_error(msg), status_(status), expected_(expected), got_(got), index_(index) {}
    int status() const { return status_; }
    int64_t expected() const { return expected_; }
    int64_t got() const { return got_; }
    int64_t batchIndex() const { return index_; }
    // the FFTError case of Sources/MetalFFT/Internal/MetalContext.swift:6-30
    const char* caseName() const {
        switch (status_) {
            case MFFT_ERR_NO_DEVICE: return "noMetalDevice";
            case MFFT_ERR_NO_STREAM: return "noCommandQueue";
            case MFFT_ERR_LIBRARY_BUILD: return "libraryBuildFailed";
            case MFFT_ERR_KERNEL_NOT_FOUND: return "kernelNotFound";
            case MFFT_ERR_EXEC_FAILED: return "commandBufferFailed";
            case MFFT_ERR_INVALID_INPUT_SIZE: return "invalidInputSize";
            case MFFT_ERR_BATCH_INPUT_SIZE: return "batchInputSize";
            case MFFT_ERR_UNSUPPORTED_SIZE: return "unsupportedFFTSize";
            case MFFT_ERR_ALLOCATION: return "bufferAllocationFailed";
            case MFFT_ERR_INVALID_ARGUMENT: return "invalidArgument";
            case MFFT_ERR_TIMEOUT: return "timeout";
            default: return "unknown";
        }
    }

   private:
    int status_;
    int64_t expected_, got_, index_;
};

inline void check(int status) {
    if (status == MFFT_SUCCESS) return;
    char buf[512];
    mfft_last_error(buf, sizeof(buf));
    int64_t e = -1, g = -1, i = -1;
    mfft_last_error_detail(&e, &g, &i);
    throw FFTError(status, buf, e, g, i);
}

inline mfft_ctx* sharedContext() {
    mfft_ctx* c = nullptr;
    check(mfft_context_shared(&c));
    return c;
}

class MetalFFT {
   public:
    explicit MetalFFT(int64_t size) : size_(size) { check(mfft_plan_create(sharedContext(), size, &plan_)); }
    ~MetalFFT() { mfft_plan_destroy(plan_); }
    MetalFFT(const MetalFFT&) = delete;
    MetalFFT& operator=(const MetalFFT&) = delete;
    int64_t size() const { return size_; }

    std::vector<cfloat> forward(const std::vector<cfloat>& x) { return run(x, MFFT_FORWARD); }
    void forward(const cfloat* input, int64_t count, std::vector<cfloat>& output) {
        if (count != size_) throw FFTError(MFFT_ERR_INVALID_INPUT_SIZE, "Input size mismatch", size_, count, -1);
        output.resize((size_t)size_);
        check(mfft_exec_c2c(plan_, input, output.data(), 1, MFFT_FORWARD, MFFT_HOST_MEMORY, nullptr));
    }
    std::vector<cfloat> inverse(const std::vector<cfloat>& x) { return run(x, MFFT_INVERSE); }
    // Gradient with respect to the input of forward (direction MFFT_FORWARD)
    // or inverse (MFFT_INVERSE), given the gradient of a real loss with
    // respect to its output (mfft_exec_c2c_backward).
    std::vector<cfloat> backward(const std::vector<cfloat>& grad, int direction = MFFT_FORWARD) {
        if ((int64_t)grad.size() != size_)
            throw FFTError(MFFT_ERR_INVALID_INPUT_SIZE, "Input size mismatch", size_, (int64_t)grad.size(), -1);
        std::vector<cfloat> g((size_t)size_);
        check(mfft_exec_c2c_backward(plan_, grad.data(), g.data(), 1, direction, MFFT_HOST_MEMORY, nullptr));
        return g;
    }
    std::vector<std::vector<cfloat>> forwardBatch(const std::vector<std::vector<cfloat>>& xs) {
        if (xs.empty()) return {};
        std::vector<cfloat> flat;
        flat.reserve(xs.size() * (size_t)size_);
        for (size_t i = 0; i < xs.size(); ++i) {
            if ((int64_t)xs[i].size() != size_)
                throw FFTError(MFFT_ERR_BATCH_INPUT_SIZE, "Batch element size mismatch", size_,
                               (int64_t)xs[i].size(), (int64_t)i);
            flat.insert(flat.end(), xs[i].begin(), xs[i].end());
        }
        check(mfft_exec_c2c(plan_, flat.data(), flat.data(), (int64_t)xs.size(), MFFT_FORWARD, MFFT_HOST_MEMORY,
                            nullptr));
        std::vector<std::vector<cfloat>> out(xs.size());
        for (size_t i = 0; i < xs.size(); ++i)
            out[i].assign(flat.begin() + i * size_, flat.begin() + (i + 1) * size_);
        return out;
    }
    mfft_plan* handle() { return plan_; }

   private:
    std::vector<cfloat> run(const std::vector<cfloat>& x, int dir) {
        if ((int64_t)x.size() != size_)
            throw FFTError(MFFT_ERR_INVALID_INPUT_SIZE, "Input size mismatch", size_, (int64_t)x.size(), -1);
        std::vector<cfloat> y((size_t)size_);
        check(mfft_exec_c2c(plan_, x.data(), y.data(), 1, dir, MFFT_HOST_MEMORY, nullptr));
        return y;
    }
    int64_t size_;
    mfft_plan* plan_ = nullptr;
};

class MultiChannelFFT {
   public:
    MultiChannelFFT(int64_t channels, int64_t size) : channels_(channels), fft_(size) {
        if (channels <= 0) throw FFTError(MFFT_ERR_INVALID_ARGUMENT, "channels must be > 0", -1, channels, -1);
    }
    std::vector<std::vector<cfloat>> forward(const std::vector<std::vector<cfloat>>& xs) {
        if ((int64_t)xs.size() != channels_)
            throw FFTError(MFFT_ERR_INVALID_ARGUMENT, "channel count mismatch", channels_, (int64_t)xs.size(), -1);
        return fft_.forwardBatch(xs);
    }

   private:
    int64_t channels_;
    MetalFFT fft_;
};

class Convolver {
   public:
    Convolver(const std::vector<float>& kernel, int64_t fftSize) : K_((int64_t)kernel.size()) {
        check(mfft_conv_create(sharedContext(), kernel.data(), K_, fftSize, &h_));
    }
    ~Convolver() { mfft_conv_destroy(h_); }
    Convolver(const Convolver&) = delete;
    Convolver& operator=(const Convolver&) = delete;
    int64_t blockSize() const { return mfft_conv_block_size(h_); }
    int64_t hopSize() const { return mfft_conv_hop_size(h_); }
    static int64_t recommendedFFTSize(int64_t kernelCount) { return mfft_recommended_fft_size(kernelCount); }
    std::vector<float> apply(const std::vector<float>& signal) {
        std::vector<float> y(signal.size() + (size_t)K_ - 1);
        check(mfft_conv_apply(h_, signal.data(), (int64_t)signal.size(), y.data(), MFFT_HOST_MEMORY, nullptr));
        return y;
    }

   private:
    int64_t K_;
    mfft_conv* h_ = nullptr;
};

class Correlator {
   public:
    explicit Correlator(int64_t fftSize) : n_(fftSize) { check(mfft_corr_create(sharedContext(), fftSize, &h_)); }
    ~Correlator() { mfft_corr_destroy(h_); }
    Correlator(const Correlator&) = delete;
    Correlator& operator=(const Correlator&) = delete;
    std::vector<float> cross(const std::vector<float>& a, const std::vector<float>& b) {
        std::vector<float> r((size_t)n_);
        check(mfft_corr_cross(h_, a.data(), (int64_t)a.size(), b.data(), (int64_t)b.size(), r.data(),
                              MFFT_HOST_MEMORY, nullptr));
        return r;
    }
    std::vector<float> autocorrelation(const std::vector<float>& x) { return cross(x, x); }

   private:
    int64_t n_;
    mfft_corr* h_ = nullptr;
};

class FFTAnalyzer {
   public:
    FFTAnalyzer(int64_t size, double sampleRate, int window = MFFT_WINDOW_HANN, double kaiserBeta = 6.0)
        : size_(size) {
        check(mfft_analyzer_create(sharedContext(), size, sampleRate, window, kaiserBeta, &h_));
    }
    ~FFTAnalyzer() { mfft_analyzer_destroy(h_); }
    FFTAnalyzer(const FFTAnalyzer&) = delete;
    FFTAnalyzer& operator=(const FFTAnalyzer&) = delete;
    std::vector<cfloat> analyze(const std::vector<float>& samples, int64_t offset = 0) {
        std::vector<cfloat> out((size_t)size_);
        check(mfft_analyzer_analyze(h_, samples.data(), (int64_t)samples.size(), offset, out.data(),
                                    MFFT_HOST_MEMORY, nullptr));
        return out;
    }

   private:
    int64_t size_;
    mfft_analyzer* h_ = nullptr;
};

}  // namespace mfft
