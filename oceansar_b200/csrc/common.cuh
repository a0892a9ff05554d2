// Shared device helpers for the OCEANSAR raw-generation kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <utility>

#include "oceansar_b200.h"

#define OCS_HD __host__ __device__ __forceinline__
#define OCS_D __device__ __forceinline__

namespace ocs {

constexpr int kSincTaps = 8;        // n_sinc_samples fixed by sar_raw_nompi.py:119
constexpr int kSincOvs = 20;        // sinc_ovs fixed by sar_raw_nompi.py:120

// ---------------------------------------------------------------------------------------
// Exactly rounded double arithmetic that the compiler may not contract into FMAs.  Used
// wherever the reference's float64 numpy expression must be reproduced bit for bit (slant
// range, range-bin index, LUT index).
OCS_D double dadd(double a, double b) { return __dadd_rn(a, b); }
OCS_D double dsub(double a, double b) { return __dsub_rn(a, b); }
OCS_D double dmul(double a, double b) { return __dmul_rn(a, b); }
OCS_D double ddiv(double a, double b) { return __ddiv_rn(a, b); }
OCS_D float fadd(float a, float b) { return __fadd_rn(a, b); }
OCS_D float fsub(float a, float b) { return __fsub_rn(a, b); }
OCS_D float fmul(float a, float b) { return __fmul_rn(a, b); }

template <typename T> struct cplx { T re, im; };
using c64 = cplx<float>;
using c128 = cplx<double>;

template <typename T> OCS_HD cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T> OCS_HD cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T> OCS_HD cplx<T> cscale(cplx<T> a, T s) { return {a.re * s, a.im * s}; }

OCS_D c128 cexpi(double ph) { double s, c; sincos(ph, &s, &c); return {c, s}; }
OCS_D c64 cexpi(float ph) { float s, c; sincosf(ph, &s, &c); return {c, s}; }

// numpy.sinc: sin(pi*x)/(pi*x) with x == 0 replaced by 1e-20 (numpy/lib/_function_base_impl.py)
OCS_D double np_sinc(double x) {
    double y = dmul(3.141592653589793, (x == 0.0) ? 1.0e-20 : x);
    return sin(y) / y;
}
OCS_D float np_sinc(float x) {
    float y = 3.14159265358979f * ((x == 0.0f) ? 1.0e-20f : x);
    return sinf(y) / y;
}

// Reduce an angle to [-pi, pi) in float64 (Cody-Waite with a two-part 2*pi).
OCS_D double reduce_2pi(double x) {
    const double inv2pi = 0.15915494309189535;
    const double p1 = 6.283185307179586;          // fl(2*pi)
    const double p2 = 2.4492935982947064e-16;     // 2*pi - p1
    double k = rint(x * inv2pi);
    return fma(-k, p2, fma(-k, p1, x));
}

// Range-bin index and LUT index of one facet (range_profile.py:103-108), bit-exact with
// numpy: bin_f = (srg - min_sr) / binsize; bin_d = floor(bin_f);
// lut = round_half_even(ovs * (1 - (bin_f - bin_d))).
OCS_D void bin_and_lut(double srg, double min_sr, double binsize, int ovs, int &bin_d, int &lut) {
    double bin_f = ddiv(dsub(srg, min_sr), binsize);
    double fl = floor(bin_f);
    if (!(fabs(fl) < 1.0e9)) {            // NaN / inf / absurd ranges: every tap is dropped
        bin_d = -(1 << 30);
        lut = 0;
        return;
    }
    bin_d = (int)fl;
    lut = (int)rint(dmul((double)ovs, dsub(1.0, dsub(bin_f, fl))));
}

// Raise a kernel's dynamic shared-memory limit once per (kernel, device): later launches,
// including those recorded into a CUDA graph, then issue no attribute call.
inline cudaError_t ensure_smem(const void *kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(kernel, dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done[key] = bytes;
    return e;
}

// CTAs of `kernel` that fit on the whole device at once (cached per kernel, block size,
// shared memory and device): the grid size of persistent kernels.
inline int resident_ctas(const void *kernel, int threads, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<std::pair<const void *, int>, std::pair<int, size_t>>, int> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    std::lock_guard<std::mutex> lock(mu);
    auto key = std::make_pair(std::make_pair(kernel, dev), std::make_pair(threads, smem));
    auto it = done.find(key);
    if (it != done.end()) return it->second;
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess) return -1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
    int n = per_sm * sms;
    done[key] = n;
    return n;
}

// Mixed-precision form of bin_and_lut: the division becomes a multiplication by the
// reciprocal bin size (a one-ulp difference in bin_f; the floor / round-half-even steps
// are unchanged).
OCS_D void bin_and_lut_fast(double srg, double min_sr, double inv_binsize, int ovs, int &bin_d, int &lut) {
    double bin_f = (srg - min_sr) * inv_binsize;
    double fl = floor(bin_f);
    if (!(fabs(fl) < 1.0e9)) {
        bin_d = -(1 << 30);
        lut = 0;
        return;
    }
    bin_d = (int)fl;
    lut = (int)rint((double)ovs * (1.0 - (bin_f - fl)));
}

}  // namespace ocs
