// stubs.cu -- entry points whose kernels are not built yet report it.
#include "capi_internal.h"

using namespace mfft;


#define MFFT_NOT_BUILT(name) set_error(MFFT_ERR_KERNEL_NOT_FOUND, -1, -1, -1, "%s: kernel not built", name)

extern "C" int mfft_multi_create(mfft_ctx*, const mfft_multi_desc*, int, mfft_multi**) {
    return MFFT_NOT_BUILT("mfft_multi_create");
}
extern "C" int mfft_multi_destroy(mfft_multi*) { return MFFT_SUCCESS; }
extern "C" int64_t mfft_multi_points(const mfft_multi*) { return 0; }
extern "C" int mfft_multi_exec(mfft_multi*, const void*, void*, int, int, void*) {
    return MFFT_NOT_BUILT("mfft_multi_exec");
}
extern "C" int mfft_conv_create(mfft_ctx*, const float*, int64_t, int64_t, mfft_conv**) {
    return MFFT_NOT_BUILT("mfft_conv_create");
}
extern "C" int mfft_conv_destroy(mfft_conv*) { return MFFT_SUCCESS; }
extern "C" int64_t mfft_conv_block_size(const mfft_conv*) { return 0; }
extern "C" int64_t mfft_conv_hop_size(const mfft_conv*) { return 0; }
extern "C" int64_t mfft_conv_kernel_len(const mfft_conv*) { return 0; }
extern "C" int mfft_conv_apply(mfft_conv*, const float*, int64_t, float*, int, void*) {
    return MFFT_NOT_BUILT("mfft_conv_apply");
}
extern "C" int mfft_conv_backward(mfft_conv*, const float*, int64_t, const float*, float*, float*, int, void*) {
    return MFFT_NOT_BUILT("mfft_conv_backward");
}
extern "C" int mfft_corr_create(mfft_ctx*, int64_t, mfft_corr**) { return MFFT_NOT_BUILT("mfft_corr_create"); }
extern "C" int mfft_corr_destroy(mfft_corr*) { return MFFT_SUCCESS; }
extern "C" int mfft_corr_cross(mfft_corr*, const float*, int64_t, const float*, int64_t, float*, int, void*) {
    return MFFT_NOT_BUILT("mfft_corr_cross");
}
extern "C" int mfft_window(int, int64_t, double, float*) { return MFFT_NOT_BUILT("mfft_window"); }
extern "C" int mfft_analyzer_create(mfft_ctx*, int64_t, double, int, double, mfft_analyzer**) {
    return MFFT_NOT_BUILT("mfft_analyzer_create");
}
extern "C" int mfft_analyzer_destroy(mfft_analyzer*) { return MFFT_SUCCESS; }
extern "C" int mfft_analyzer_analyze(mfft_analyzer*, const float*, int64_t, int64_t, void*, int, void*) {
    return MFFT_NOT_BUILT("mfft_analyzer_analyze");
}
