// Arithmetic-rate probe: eight independent FMA chains per thread in float64, float32 or
// packed float32x2, so that the FMA pipes, not latency, bound the launch.  The simulator's
// two precision forms differ mainly in which of these pipes their per-facet range and
// phase work runs on; the measured ratio is what bounds the mixed form's gain.
#include "common.cuh"

namespace ocs {

constexpr int kRateChains = 8;

template <typename T> struct RateOps;
template <> struct RateOps<double> {
    static OCS_D double fma_(double x, double a, double b) { return fma(x, a, b); }
    static OCS_D double init(int i) { return (double)i * 1e-3; }
    static OCS_D double scalar(double x) { return x; }
};
template <> struct RateOps<float> {
    static OCS_D float fma_(float x, float a, float b) { return fmaf(x, a, b); }
    static OCS_D float init(int i) { return (float)i * 1e-3f; }
    static OCS_D float scalar(float x) { return x; }
};
template <> struct RateOps<float2> {
    static OCS_D float2 fma_(float2 x, float2 a, float2 b) { return __ffma2_rn(x, a, b); }
    static OCS_D float2 init(int i) { return make_float2((float)i * 1e-3f, (float)i * 2e-3f); }
    static OCS_D float scalar(float2 x) { return x.x + x.y; }
};

// The result is stored only when it equals a value the chains cannot reach, which the
// compiler cannot prove: every FMA stays live and nothing is written.
template <typename T>
__global__ void fma_rate_kernel(T a, T b, int iters, float *sink) {
    T x[kRateChains];
#pragma unroll
    for (int k = 0; k < kRateChains; ++k) x[k] = RateOps<T>::init((int)threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kRateChains; ++k) x[k] = RateOps<T>::fma_(x[k], a, b);
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < kRateChains; ++k) s += (float)RateOps<T>::scalar(x[k]);
    if (s == -1234.5f) sink[blockIdx.x] = s;
}

}  // namespace ocs

// kind 0: float64, 1: float32, 2: packed float32x2.  Each thread runs iters x 8 FMAs
// (x 2 lanes for kind 2); sink: at least `blocks` floats, never written in practice.
extern "C" int ocs_fma_rate(int32_t kind, int32_t blocks, int32_t threads, int32_t iters, float *sink, void *stream) {
    if (kind < 0 || kind > 2 || blocks < 1 || threads < 32 || threads > 1024 || iters < 1 || !sink) return OCS_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    // a = 1 - 2^-20, b = 2^-10: the chains converge to b / (1 - a) without overflow
    if (kind == 0)
        ocs::fma_rate_kernel<double><<<blocks, threads, 0, st>>>(1.0 - 0x1p-20, 0x1p-10, iters, sink);
    else if (kind == 1)
        ocs::fma_rate_kernel<float><<<blocks, threads, 0, st>>>(1.f - 0x1p-20f, 0x1p-10f, iters, sink);
    else
        ocs::fma_rate_kernel<float2><<<blocks, threads, 0, st>>>(make_float2(1.f - 0x1p-20f, 1.f - 0x1p-20f),
                                                                 make_float2(0x1p-10f, 0x1p-10f), iters, sink);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}
