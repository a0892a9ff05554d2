// Facet-to-range-bin accumulation engine (the body of profile_integrator,
// oceansar/radarsim/range_profile.py:22-49, re-organised for the GPU).
//
// Every facet adds taps * complex values to consecutive range bins:
//     out[bin_d - taps/2 + j] += sinc[lut + j*ovs] * coef,   j = 0 .. taps-1.
// Instead of one atomic per tap, each thread keeps a private S-slot window of bins in
// registers.  A facet whose taps fall inside the window is added with S predicated
// multiply-adds whose weights come from a pre-shifted table in shared memory
// (wtab[off][lut][s] = sinc[lut + (s-off)*ovs] for 0 <= s-off < taps, else 0), so the
// weights of one facet are S/4 vectorised shared loads and no register is indexed
// dynamically.  When a facet falls outside the window (or the thread's facets end) the
// window is flushed into a per-CTA shared-memory copy of the bins it covers, and the CTA
// adds that copy to global memory once at the end.  Bins outside [0, nbins) are dropped,
// exactly like the reference's edge branch.
#pragma once
#include "common.cuh"

namespace ocs {

// Row stride (elements) of the pre-shifted weight table: S slots padded so that rows start
// on 8 different 4-bank groups (a row is read with 16-byte vector loads by lanes whose
// rows differ).
template <typename T, int S> __host__ __device__ constexpr int wtab_stride() {
    return sizeof(T) == 4 ? (S == 16 ? 20 : S) : (S == 12 ? 14 : (S == 16 ? 18 : S));
}

template <typename T, int S> __host__ __device__ constexpr int wtab_len(int taps, int ovs) {
    return (S - taps + 1) * (ovs + 1) * wtab_stride<T, S>();
}

// Pre-shifted weight table: (S - taps + 1) offsets x (ovs + 1) LUT positions x S slots.
template <typename T, int S>
__device__ void build_wtab(T *wtab, const float *sinc, int taps, int ovs) {
    constexpr int W = wtab_stride<T, S>();
    const int total = wtab_len<T, S>(taps, ovs);
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        int s = i % W;
        int lut = (i / W) % (ovs + 1);
        int off = i / (W * (ovs + 1));
        int j = s - off;
        wtab[i] = (s < S && j >= 0 && j < taps) ? (T)sinc[lut + j * ovs] : (T)0;
    }
}

template <typename T> struct vec4_of;
template <> struct vec4_of<float> { using type = float4; };
template <> struct vec4_of<double> { using type = double2; };   // 16-byte loads

// Per-CTA shared accumulator for the bins [cta_base, cta_base + nbw), NOUT outputs,
// interleaved (re, im).
template <typename T, int NOUT>
struct CtaBins {
    T *acc;          // [NOUT][nbw][2]
    int cta_base;
    int nbw;
    int nout;        // outputs in use (<= NOUT); the others are never written
    int nbins;       // valid output bins [0, nbins)
    T *out;          // global output, output o at out + 2*o*out_stride
    long long out_stride;

    __device__ void add(int o, int b, T re, T im) {
        if (o >= nout || b < 0 || b >= nbins) return;
        int lb = b - cta_base;
        if (lb >= 0 && lb < nbw) {
            atomicAdd(&acc[(o * nbw + lb) * 2], re);
            atomicAdd(&acc[(o * nbw + lb) * 2 + 1], im);
        } else {
            atomicAdd(&out[2 * (o * out_stride + b)], re);
            atomicAdd(&out[2 * (o * out_stride + b) + 1], im);
        }
    }

    __device__ void zero() {
        for (int i = threadIdx.x; i < NOUT * nbw * 2; i += blockDim.x) acc[i] = (T)0;
    }

    // After a __syncthreads(): add the CTA's bins to global memory.
    __device__ void flush_to_global() {
        for (int i = threadIdx.x; i < nout * nbw; i += blockDim.x) {
            int o = i / nbw, lb = i % nbw;
            int b = cta_base + lb;
            if (b < 0 || b >= nbins) continue;
            T re = acc[2 * i], im = acc[2 * i + 1];
            if (re != (T)0 || im != (T)0) {
                atomicAdd(&out[2 * (o * out_stride + b)], re);
                atomicAdd(&out[2 * (o * out_stride + b) + 1], im);
            }
        }
    }
};

template <typename T, int S, int NOUT>
struct BinWindow {
    T re[NOUT][S];
    T im[NOUT][S];
    int base;       // bin of slot 0
    int lo, hi;     // touched slot range [lo, hi]
    bool live;

    __device__ void reset() {
#pragma unroll
        for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int s = 0; s < S; ++s) { re[o][s] = (T)0; im[o][s] = (T)0; }
        live = false;
        lo = S;
        hi = -1;
    }

    __device__ void flush(CtaBins<T, NOUT> &cb) {
        if (!live) return;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (s >= lo && s <= hi) {
#pragma unroll
                for (int o = 0; o < NOUT; ++o) cb.add(o, base + s, re[o][s], im[o][s]);
            }
        }
        reset();
    }

    // Add one facet whose first tap lands on bin `first` with LUT index `lut`.
    __device__ void add(int first, int lut, const cplx<T> (&coef)[NOUT], const T *wtab,
                        const float *sinc, int taps, int ovs, CtaBins<T, NOUT> &cb) {
        // one test for all coefficients: a finite sum implies finite terms; a sum that
        // overflows with finite terms takes the exact per-tap path as well
        T sum = (T)0;
#pragma unroll
        for (int o = 0; o < NOUT; ++o) sum += coef[o].re + coef[o].im;
        if (!isfinite(sum)) {
            // Non-finite coefficients touch exactly their own taps, as in the reference.
            for (int j = 0; j < taps; ++j) {
                T w = (T)sinc[lut + j * ovs];
#pragma unroll
                for (int o = 0; o < NOUT; ++o)
                    cb.add(o, first + j, w * coef[o].re - (T)0 * coef[o].im,
                           w * coef[o].im + (T)0 * coef[o].re);
            }
            return;
        }
        const int slack = S - taps;
        int off = first - base;
        if (!live || off < 0 || off > slack) {
            flush(cb);
            base = first - slack / 2;
            off = slack / 2;
            live = true;
        }
        lo = min(lo, off);
        hi = max(hi, off + taps - 1);
        using V = typename vec4_of<T>::type;
        const V *w = reinterpret_cast<const V *>(wtab + (off * (ovs + 1) + lut) * wtab_stride<T, S>());
        constexpr int PER = sizeof(V) / sizeof(T);
#pragma unroll
        for (int v = 0; v < S / PER; ++v) {
            V wv = w[v];
            const T *wp = reinterpret_cast<const T *>(&wv);
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int s = v * PER + k;
#pragma unroll
                for (int o = 0; o < NOUT; ++o) {
                    re[o][s] = fma(wp[k], coef[o].re, re[o][s]);
                    im[o][s] = fma(wp[k], coef[o].im, im[o][s]);
                }
            }
        }
    }
};

}  // namespace ocs
