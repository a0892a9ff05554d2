// Mixed-precision pulse kernel (sm_100a): the body of the azimuth loop of sar_raw
// (oceansar/radarsim/sar_raw_nompi.py:349-535) for SAR scenes with Kodis specular and / or
// Romeiser Bragg scattering, in the split-range precision form:
//
//   float64 only per pulse row and per column (the reference ranges):
//     R_y = az/2 * sin_az (row), sr_c = slant range of the column, both reduced to
//     2 k0 R mod 2 pi and converted to range-bin units, split into a float32 high part on a
//     2^-8-bin grid (so that high parts add exactly) and a float32 low part;
//   float32 per facet (the bulk):
//     delta = -cos_inc Dz + Dx sin_inc + Dy sin_az (the facet's range offset), the bin
//     position hi + (lo + delta / binsize) and the two-way phase
//     phi_col + phi_row - 2 k0 delta, whose large product 2 k0 delta is reduced exactly
//     (an error-free product and a three-part 2 pi), the Kodis field, the Bragg lines,
//     antenna / ATI / XTI factors and the accumulation;
//   float64 only for facets whose float32 decision is within its error bound of a
//     rounding boundary (range bin floor, LUT round-half-even, Kodis facet window), which
//     are re-decided with the float64 drop-in's exact arithmetic: bins, LUT indices and
//     specular facet selection are therefore identical to the float64 form's.
//
// Accumulation: 12-slot register windows per thread (float32 FMA; a window sums at most one
// tile height of facets), flushed into CTA shared bins kept as compensated (hi, lo) float32
// pairs (TwoSum of every shared atomic add), added at the end of a tile into the complex64
// raw row with compensated global atomics whose rounding errors collect in a per-pulse
// float32 compensation row; the next pulse's row-table kernel (or ocs_pulse_flush) folds
// that row into the raw row.
//
// Input staging: the facet inputs of a CTA row (the float32 fields, sqrt(RCS) and
// scatterer start indices of 128 columns) are moved into a four-row shared-memory ring by
// tiled tensor copies (cp.async.bulk.tensor: one three-dimensional box for all fields, one
// per index map and one for the sqrt(RCS) planes) that complete on the slot's mbarrier.
// The warp that finishes reading a row last refills its slot with the row four ahead, so no
// warp ever waits for another, only for data.  Every mbarrier wait is bounded: a wait that
// gives up sets the launch's error flag, lets the copies in flight land and ends the CTA's
// work.
#pragma once
#include <cuda.h>

#include "bulk.cuh"

namespace ocs {

constexpr int kMixCols = 128;       // columns (threads) per CTA, 32 per warp
constexpr int kMixSlots = 4;        // ring rows (three in flight while one is read)
constexpr int kMixArrays = 14;      // staged input arrays per row (see MixArr)
constexpr int kMixRT = 8;           // float row-table entries before the channel factors
constexpr int kMixS = 12;           // register-window slots
constexpr int kMixNbw = 160;        // CTA shared bin window

// staged arrays: fields, Kodis curvatures, scatterer start indices, sqrt(RCS) [pol][line]
enum MixArr { kAdx = 0, kAdy, kAdz, kAdiffx, kAdiffy, kAdxx, kAdyy, kAdxy, kAindm, kAindp, kAscat };

// Tensor maps of one launch's inputs: the fields as one [nf][ny][nx] float32 tensor (the
// surface keeps them in one block, Dx Dy Dz Diffx Diffy [Diffxx Diffyy Diffxy]), the two
// int32 [ny][nx] scatterer index maps and the [2 npol][ny][nx] sqrt(RCS) planes; every box
// is one row of kMixCols columns.
struct alignas(64) MixMaps {
    CUtensorMap fields, indm, indp, scat;
    int nf;                         // fields in the fields map (5, or 8 with the curvatures)
};

// Per-pulse workspace after the float64 row table: float row table [ny][kMixRT + 2 nch]
// (Bh, Bl, phi_y, sin_az, cos_azp, sin_azp, azp, -, then the channel factors), then the
// header {pending raw row, error flag}.
OCS_HD size_t mix_rowtab_offset(int ny, int nch) { return (size_t)ny * (5 + 2 * nch) * sizeof(double); }
OCS_HD size_t mix_hdr_offset(int ny, int nch) {
    return (mix_rowtab_offset(ny, nch) + (size_t)ny * (kMixRT + 2 * nch) * sizeof(float) + 15) & ~(size_t)15;
}
constexpr size_t kMixHdrBytes = 16;

// ---------------------------------------------------------------------------------------
// Split-float helpers.
OCS_D float two_sum_err(float a, float b, float s) {
    const float bp = __fsub_rn(s, a);
    return __fadd_rn(__fsub_rn(a, __fsub_rn(s, bp)), __fsub_rn(b, bp));
}

// Compensated add of v into the shared pair (hi, lo): the atomic returns the old high
// part, from which the exact rounding error of the stored sum follows.
OCS_D void cadd_shared(float *hi, float *lo, float v) {
    if (v == 0.f) return;
    const float old = atomicAdd(hi, v);
    const float err = two_sum_err(old, v, __fadd_rn(old, v));
    if (err != 0.f) atomicAdd(lo, err);
}

// Reduction of a float32 phase p = K_hi * d (plus the exact product error and K_lo * d) to
// about [-pi, pi]: n = rint(p / 2 pi), p - n P1 exactly (P1 has 8 significant bits), then
// the remaining parts of 2 pi.
OCS_D float reduce_prod(float khi, float klo, float d) {
    const float p = __fmul_rn(khi, d);
    const float pe = fmaf(khi, d, -p) + klo * d;
    const float n = rintf(p * 0.15915494309189535f);
    float r = fmaf(-n, 6.28125f, p);                      // exact
    r = fmaf(-n, 1.9353071693331003e-3f, r);              // 2 pi - 6.28125, float part
    r = fmaf(-n, 1.0253376273028358e-11f, r);             // remainder of 2 pi
    return r + pe;
}
OCS_D float wrap_pi(float x) { return fmaf(-rintf(x * 0.15915494309189535f), 6.2831853071795865f, x); }

// Split of a float64 bin position into a float32 part on a 2^-8 grid and a float32 rest.
OCS_HD void split_bins(double v, float &hi, float &lo) {
    const double h = rint(v * 256.0) * (1.0 / 256.0);
    hi = (float)h;
    lo = (float)(v - h);
}

// ---------------------------------------------------------------------------------------
// Per-pulse row tables of the mixed kernel: the float64 table of pulse_row plus the float
// table (split bin position and reduced phase of R_y, sin_az, projected azimuth cos / sin /
// angle, channel factors).  Threads beyond the rows fold the previous pulse's compensation
// row into its raw row.
OCS_D void mix_row(const PulseArgs &a, double az_now, int y) {
    unsigned char *ws = reinterpret_cast<unsigned char *>(a.rowtab);
    pulse_row(a, az_now, y);
    {
        const double az = a.rowtab[y], sin_az = a.rowtab[(long long)a.ny + y];
        const double azp = a.rowtab[2LL * a.ny + y];
        const double ry = dmul(az * 0.5, sin_az);
        float *ft = reinterpret_cast<float *>(ws + mix_rowtab_offset(a.ny, a.nch)) + (long long)y * (kMixRT + 2 * a.nch);
        split_bins(ry * a.inv_binsize, ft[0], ft[1]);
        ft[2] = (float)reduce_2pi((-2.0 * a.k0) * ry);
        ft[3] = (float)sin_az;
        ft[4] = (float)a.rowtab[3LL * a.ny + y];
        ft[5] = (float)a.rowtab[4LL * a.ny + y];
        ft[6] = (float)azp;
        ft[7] = 0.f;
        const double *fac = a.rowtab + 5LL * a.ny + 2LL * y * a.nch;
        for (int c = 0; c < 2 * a.nch; ++c) ft[kMixRT + c] = (float)fac[c];
    }
}

__global__ void pulse_rows_mixed_kernel(const __grid_constant__ PulseArgs a, float *lo_row, int nout_all) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned char *ws = reinterpret_cast<unsigned char *>(a.rowtab);
    int *hdr = reinterpret_cast<int *>(ws + mix_hdr_offset(a.ny, a.nch));
    if (t < a.ny) mix_row(a, a.az_now, t);
    // fold the compensation row of the previous pulse (pending >= 0) into its raw row
    if (lo_row) {
        const int pending = hdr[0];
        const long long nfold = (long long)nout_all * a.nbins;
        if (pending >= 0) {
            float *raw = reinterpret_cast<float *>(a.raw);
            for (long long i = t; i < nfold; i += (long long)gridDim.x * blockDim.x) {
                const long long o = i / a.nbins, b = i - o * a.nbins;
                float *dst = raw + 2 * (o * a.raw_out_stride + (long long)pending * a.nbins + b);
                const float lr = lo_row[2 * i], li = lo_row[2 * i + 1];
                if (lr != 0.f) dst[0] += lr;
                if (li != 0.f) dst[1] += li;
                lo_row[2 * i] = 0.f;
                lo_row[2 * i + 1] = 0.f;
            }
        }
    }
}

// The fold alone (end of a scene, or before the raw cube is read).
__global__ void pulse_flush_kernel(const __grid_constant__ PulseArgs a, float *lo_row, int nout_all) {
    unsigned char *ws = reinterpret_cast<unsigned char *>(a.rowtab);
    int *hdr = reinterpret_cast<int *>(ws + mix_hdr_offset(a.ny, a.nch));
    const int pending = hdr[0];
    const long long nfold = (long long)nout_all * a.nbins;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (pending >= 0) {
        float *raw = reinterpret_cast<float *>(a.raw);
        for (long long i = t; i < nfold; i += (long long)gridDim.x * blockDim.x) {
            const long long o = i / a.nbins, b = i - o * a.nbins;
            float *dst = raw + 2 * (o * a.raw_out_stride + (long long)pending * a.nbins + b);
            const float lr = lo_row[2 * i], li = lo_row[2 * i + 1];
            if (lr != 0.f) dst[0] += lr;
            if (li != 0.f) dst[1] += li;
            lo_row[2 * i] = 0.f;
            lo_row[2 * i + 1] = 0.f;
        }
    }
}

// ---------------------------------------------------------------------------------------
// Shared memory of the mixed kernel.
template <int NOUT> struct MixSmem {
    float *wtab;                    // pre-shifted weights [5][21][12]
    float *bhi, *blo;               // CTA bins [NOUT][kMixNbw][2] (hi, lo)
    float *rt;                      // float row table of the tile [rows][RT]
    double *raz;                    // float64 az, sin_az of the tile's rows [2][rows]
    double *sred;                   // block reduction scratch [32]
    float *stage;                   // [kMixSlots][kMixArrays][kMixCols]
    unsigned long long *bar;        // [kMixSlots] full barriers
    int *cnt;                       // [kMixSlots] warps done with the slot's row
    int rcap;                       // rows the row tables hold (the largest tile height)
};

template <int NOUT> OCS_HD size_t mix_smem_bytes(int nch, int rows_cap) {
    return (size_t)wtab_len<float, kMixS>(kSincTaps, kSincOvs) * 4 + (size_t)NOUT * kMixNbw * 2 * 2 * 4 +
           (size_t)rows_cap * (kMixRT + 2 * nch) * 4 + 2 * (size_t)rows_cap * 8 + 32 * 8 +
           (size_t)kMixSlots * kMixArrays * kMixCols * 4 + kMixSlots * 16 + 256;
}

template <int NOUT> OCS_D MixSmem<NOUT> mix_smem(unsigned char *smem, int nch, int rows_cap) {
    MixSmem<NOUT> sm;
    size_t off = 0;
    auto take = [&](size_t bytes, size_t align) {
        off = (off + align - 1) & ~(align - 1);
        unsigned char *p = smem + off;
        off += bytes;
        return p;
    };
    sm.bar = reinterpret_cast<unsigned long long *>(take(kMixSlots * 8, 8));
    sm.cnt = reinterpret_cast<int *>(take(kMixSlots * 4, 4));
    sm.stage = reinterpret_cast<float *>(take((size_t)kMixSlots * kMixArrays * kMixCols * 4, 128));
    sm.wtab = reinterpret_cast<float *>(take((size_t)wtab_len<float, kMixS>(kSincTaps, kSincOvs) * 4, 16));
    sm.bhi = reinterpret_cast<float *>(take((size_t)NOUT * kMixNbw * 2 * 4, 16));
    sm.blo = reinterpret_cast<float *>(take((size_t)NOUT * kMixNbw * 2 * 4, 16));
    sm.rt = reinterpret_cast<float *>(take((size_t)rows_cap * (kMixRT + 2 * nch) * 4, 16));
    sm.raz = reinterpret_cast<double *>(take(2 * (size_t)rows_cap * 8, 8));
    sm.sred = reinterpret_cast<double *>(take(32 * 8, 8));
    sm.rcap = rows_cap;
    return sm;
}

// Register window of one thread (accum.cuh's BinWindow, flushed into compensated bins).
template <int NOUT> struct MixBins {
    float *hi, *lo;                 // shared [NOUT][kMixNbw][2]
    int cta_base, nout, nbins;
    float *out;                     // raw row of output 0 (complex64 interleaved)
    float *lo_row;                  // compensation row of output 0, or null
    long long out_stride;           // floats between outputs in out

    // bins outside the CTA window: compensated global atomics
    OCS_D void add_global(int o, int b, float re, float im) {
        float *d = out + (long long)o * out_stride + 2 * b;
        if (re != 0.f) {
            const float old = atomicAdd(d, re);
            const float e = two_sum_err(old, re, __fadd_rn(old, re));
            if (lo_row && e != 0.f) atomicAdd(lo_row + (long long)o * 2 * nbins + 2 * b, e);
        }
        if (im != 0.f) {
            const float old = atomicAdd(d + 1, im);
            const float e = two_sum_err(old, im, __fadd_rn(old, im));
            if (lo_row && e != 0.f) atomicAdd(lo_row + (long long)o * 2 * nbins + 2 * b + 1, e);
        }
    }
    OCS_D void add(int o, int b, float re, float im) {
        if (o >= nout || b < 0 || b >= nbins) return;
        const int lb = b - cta_base;
        if (lb >= 0 && lb < kMixNbw) {
            const int i = 2 * (o * kMixNbw + lb);
            cadd_shared(hi + i, lo + i, re);
            cadd_shared(hi + i + 1, lo + i + 1, im);
        } else {
            add_global(o, b, re, im);
        }
    }
};

template <int NOUT> struct MixWindow {
    float re[NOUT][kMixS], im[NOUT][kMixS];
    int base, lo, hi;
    bool live;

    OCS_D void reset() {
#pragma unroll
        for (int o = 0; o < NOUT; ++o)
#pragma unroll
            for (int s = 0; s < kMixS; ++s) { re[o][s] = 0.f; im[o][s] = 0.f; }
        live = false;
        lo = kMixS;
        hi = -1;
    }
    OCS_D void flush(MixBins<NOUT> &cb) {
        if (!live) return;
#pragma unroll
        for (int s = 0; s < kMixS; ++s) {
            if (s >= lo && s <= hi) {
#pragma unroll
                for (int o = 0; o < NOUT; ++o) cb.add(o, base + s, re[o][s], im[o][s]);
            }
        }
        reset();
    }
    // facet whose first tap is bin `first`, LUT index `lut`
    OCS_D void add(int first, int lut, const c64 (&coef)[NOUT], const float *wtab, const float *sinc,
                   MixBins<NOUT> &cb) {
        float sum = 0.f;
#pragma unroll
        for (int o = 0; o < NOUT; ++o) sum += coef[o].re + coef[o].im;
        if (!isfinite(sum)) {
            // non-finite coefficients touch exactly their own taps, as in the reference
            for (int j = 0; j < kSincTaps; ++j) {
                const float w = sinc[lut + j * kSincOvs];
#pragma unroll
                for (int o = 0; o < NOUT; ++o)
                    cb.add(o, first + j, w * coef[o].re - 0.f * coef[o].im, w * coef[o].im + 0.f * coef[o].re);
            }
            return;
        }
        constexpr int slack = kMixS - kSincTaps;
        int off = first - base;
        if (!live || off < 0 || off > slack) {
            flush(cb);
            base = first - slack / 2;
            off = slack / 2;
            live = true;
        }
        lo = min(lo, off);
        hi = max(hi, off + kSincTaps - 1);
        const float4 *w = reinterpret_cast<const float4 *>(wtab + (off * (kSincOvs + 1) + lut) * wtab_stride<float, kMixS>());
#pragma unroll
        for (int v = 0; v < kMixS / 4; ++v) {
            const float4 wv = w[v];
            const float ws[4] = {wv.x, wv.y, wv.z, wv.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int s = 4 * v + k;
#pragma unroll
                for (int o = 0; o < NOUT; ++o) {
                    re[o][s] = fmaf(ws[k], coef[o].re, re[o][s]);
                    im[o][s] = fmaf(ws[k], coef[o].im, im[o][s]);
                }
            }
        }
    }
};

// Tile-end flush of a warp's 32 register windows without contention: every lane writes its
// window (one output at a time) into the warp's scratch, then lane l sums bin lo + l (and
// every 32nd after it) over the lanes whose windows cover it, in lane order, and makes one
// compensated add into the CTA bins -- the lanes of a warp never add to the same bin.
// scr: per-warp [32][kMixS][2] floats; sbase: per-warp [32] ints.  All 32 lanes call it.
template <int NOUT>
OCS_D void warp_flush(MixWindow<NOUT> &win, MixBins<NOUT> &cb, float *scr, int *sbase) {
    const int lane = threadIdx.x & 31;
    int lo = win.live ? win.base + win.lo : 0x3fffffff;
    int hi = win.live ? win.base + win.hi : -0x3fffffff;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (hi < lo) return;                  // no live window in the warp
    sbase[lane] = win.live ? win.base : -0x3fffffff;
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
#pragma unroll
        for (int sl = 0; sl < kMixS; ++sl) {
            scr[(lane * kMixS + sl) * 2] = win.re[o][sl];
            scr[(lane * kMixS + sl) * 2 + 1] = win.im[o][sl];
        }
        __syncwarp();
        for (int b = lo + lane; b <= hi; b += 32) {
            float sr = 0.f, si = 0.f;
            for (int j = 0; j < 32; ++j) {
                const int off = b - sbase[j];
                if (off >= 0 && off < kMixS) {
                    sr += scr[(j * kMixS + off) * 2];
                    si += scr[(j * kMixS + off) * 2 + 1];
                }
            }
            cb.add(o, b, sr, si);
        }
        __syncwarp();
    }
    win.reset();
}

// Float64 slant range of one facet exactly as the drop-in computes it (no contraction).
OCS_D double srs_f64(double sr_c, double cos_i, double sin_i, double az, double sin_az, float dx, float dy,
                     float dz) {
    double srs = dsub(sr_c, dmul(cos_i, (double)dz));
    srs = dadd(srs, dmul(az * 0.5, sin_az));
    srs = dadd(srs, dmul((double)dx, sin_i));
    return dadd(srs, dmul((double)dy, sin_az));
}

// ---------------------------------------------------------------------------------------
// One tile of 128 columns x tile_rows rows.  `rseq` is the warp's running row count (ring
// slot and barrier parity); `bad` becomes true when a bounded wait gave up.
// TMA = false (the scene batch, whose slots keep no tensor maps): every thread stages its
// own column's inputs of each row into the same ring by per-thread asynchronous copies
// (cp.async, one group per row, four rows ahead) and waits only for its own copies, since
// it alone reads that column of a slot.  REFRESH: 0 = a
// pulse that reads the stored sqrt(RCS), 1 = a Bragg-refresh pulse (the Romeiser model is
// compiled only into these), 2 = decided at run time from a.refresh (the scene batch).
template <int NOUT, bool KODIS, bool TMA = true, int REFRESH = 2, int FAST = 0>
OCS_D void mix_tile(const PulseArgs &a, const MixMaps *maps, float *lo_row, int tile, int tile_rows,
                    const MixSmem<NOUT> &sm, unsigned &rseq, bool &bad, double &spec_sum, double (&bragg_sum)[2]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tiles_x = (a.nx + kMixCols - 1) / kMixCols;
    const int x0t = (tile % tiles_x) * kMixCols;
    const int x = x0t + threadIdx.x;
    const int y0 = (tile / tiles_x) * tile_rows;
    const int nrows = min(tile_rows, a.ny - y0);
    const int RT = kMixRT + 2 * a.nch;
    __syncthreads();                      // the previous tile's bins and row tables are consumed
    {
        const float *ft = reinterpret_cast<const float *>(reinterpret_cast<const unsigned char *>(a.rowtab) +
                                                          mix_rowtab_offset(a.ny, a.nch)) + (long long)y0 * RT;
        for (int i = threadIdx.x; i < nrows * RT; i += blockDim.x) sm.rt[i] = ft[i];
        for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
            sm.raz[i] = a.rowtab[y0 + i];
            sm.raz[sm.rcap + i] = a.rowtab[(long long)a.ny + y0 + i];
        }
    }
    MixBins<NOUT> cb;
    cb.hi = sm.bhi;
    cb.lo = sm.blo;
    cb.nout = a.nout;
    cb.nbins = a.nbins;
    cb.out = reinterpret_cast<float *>(a.raw) + 2 * ((long long)a.out0 * a.raw_out_stride + a.raw_row);
    cb.lo_row = lo_row ? lo_row + 2LL * a.out0 * a.nbins : nullptr;
    cb.out_stride = 2 * a.raw_out_stride;
    {
        const int xc = min(x0t, a.nx - 1);
        const double az = (double)a.y[y0] - a.az_now;
        const double srg = a.sr_col[xc] + az * 0.5 * (az / a.sr0);
        cb.cta_base = (int)floor((srg - a.min_sr) / a.binsize) - 24;
    }
    for (int i = threadIdx.x; i < NOUT * kMixNbw * 2; i += blockDim.x) {
        sm.bhi[i] = 0.f;
        sm.blo[i] = 0.f;
    }
    __syncthreads();

    MixWindow<NOUT> win;
    win.reset();
    if (!bad) {
        // every warp takes part in every row (the ring's slots are released per warp);
        // lanes past the last column stage and wait but compute nothing
        const bool col_ok = x < a.nx;
        const int xs = col_ok ? x : a.nx - 1;
        // ---- per-column constants (float64 reference quantities, converted once) ----
        const double sr_c = a.sr_col[xs];
        float Ch, Cl;
        split_bins((sr_c - a.min_sr) * a.inv_binsize, Ch, Cl);
        const float phi_x = (float)reduce_2pi((-2.0 * a.k0) * sr_c);
        const float sin_i = (float)a.sin_inc[xs], cos_i = (float)a.cos_inc[xs];
        const bool kodis = FAST || (KODIS && a.do_kodis);
        const bool bragg = FAST || a.do_bragg;
        const int npol = FAST ? 1 : a.npol;
        const float tan_i = kodis ? (float)a.tan_inc[xs] : 0.f;
        const float dinc0 = (float)(a.inc[xs] - a.inc_angle);
        float cap_r = 0.f;
        if (a.do_bragg) cap_r = (float)reduce_2pi(((2.0 * a.k0) * a.t_step) * a.c_b[xs] * (double)(a.az_step + 1));
        const float inv_bs = (float)a.inv_binsize;
        const float khi = (float)(2.0 * a.k0), klo = (float)(2.0 * a.k0 - (double)khi);
        const float hdx = (float)a.kodis.hdx, hdy = (float)a.kodis.hdy, inv_sr0 = (float)(1.0 / a.sr0);
        const float hr = (float)(0.5 * a.kodis.R_re), hi_ = (float)(0.5 * a.kodis.R_im);   // R / 2
        const long long npix = (long long)a.nx * a.ny;
        float *scat = reinterpret_cast<float *>(a.scat);
        const bool refresh = REFRESH == 2 ? a.refresh != 0 : REFRESH == 1;
        const bool load_scat = a.do_bragg && !refresh;
        // outputs of this pass (5 bits each: channel, polarisation, XTI flag)
        unsigned outs = 0;
        float kxti[NOUT];                 // -k0 b_xti of each output's channel
#pragma unroll
        for (int k = 0; k < NOUT; ++k) {
            const int o = a.out0 + k;
            const int p = o / a.nch, c = o - p * a.nch;
            const bool xti = k < a.nout && a.b_xti[c] != 0.0;
            outs |= (unsigned)(c | (p << 3) | (xti ? 16 : 0)) << (5 * k);
            kxti[k] = k < a.nout ? (float)(-a.k0 * a.b_xti[c]) : 0.f;
        }
        // ---- staging: tensor copies of whole CTA rows into the ring ----
        const int nf = TMA ? maps->nf : 0;
        const unsigned row_bytes = (unsigned)(nf + (a.do_bragg ? 2 : 0) + (load_scat ? 2 * a.npol : 0)) * kMixCols * 4u;
        const unsigned first = rseq;      // ring position of this tile's row 0
        auto slot_of = [&](int r) { return (int)((first + (unsigned)r) % kMixSlots); };
        auto issue = [&](int r) {         // TMA: one thread; the slot of row r is free
            if constexpr (!TMA) {
                // every thread: its column's words of row r, one copy group per row (empty
                // past the tile, so that every thread counts the same groups)
                if (r < nrows) {
                    float *dst = sm.stage + (size_t)slot_of(r) * kMixArrays * kMixCols + threadIdx.x;
                    const long long g = (long long)(y0 + r) * a.nx + xs;
                    cp_async(dst + kAdx * kMixCols, a.dx_f + g, 4);
                    cp_async(dst + kAdy * kMixCols, a.dy_f + g, 4);
                    cp_async(dst + kAdz * kMixCols, a.dz_f + g, 4);
                    cp_async(dst + kAdiffx * kMixCols, a.diffx + g, 4);
                    cp_async(dst + kAdiffy * kMixCols, a.diffy + g, 4);
                    if (kodis) {
                        cp_async(dst + kAdxx * kMixCols, a.diffxx + g, 4);
                        cp_async(dst + kAdyy * kMixCols, a.diffyy + g, 4);
                        cp_async(dst + kAdxy * kMixCols, a.diffxy + g, 4);
                    }
                    if (bragg) {
                        cp_async(dst + kAindm * kMixCols, a.ind0_m + g, 4);
                        cp_async(dst + kAindp * kMixCols, a.ind0_p + g, 4);
                    }
                    if (load_scat) {
                        cp_async(dst + kAscat * kMixCols, scat + g, 4);
                        cp_async(dst + (kAscat + 1) * kMixCols, scat + npix + g, 4);
                        if (npol == 2) {
                            cp_async(dst + (kAscat + 2) * kMixCols, scat + 2 * npix + g, 4);
                            cp_async(dst + (kAscat + 3) * kMixCols, scat + 3 * npix + g, 4);
                        }
                    }
                }
                cp_async_commit();
                return;
            }
            const int slot = slot_of(r);
            float *dst = sm.stage + (size_t)slot * kMixArrays * kMixCols;
            unsigned long long *bar = sm.bar + slot;
            fence_proxy_async();
            mbar_expect_tx(bar, row_bytes);
            const int yy = y0 + r;
            tma_load_3d(dst + kAdx * kMixCols, &maps->fields, x0t, yy, 0, bar);
            if (bragg) {
                tma_load_2d(dst + kAindm * kMixCols, &maps->indm, x0t, yy, bar);
                tma_load_2d(dst + kAindp * kMixCols, &maps->indp, x0t, yy, bar);
            }
            if (load_scat) tma_load_3d(dst + kAscat * kMixCols, &maps->scat, x0t, yy, 0, bar);
        };
        auto wait_row = [&](int r) -> bool {
            if constexpr (!TMA) {
                // rows up to r + 3 are issued: row 0 waits with 3 groups pending, row r > 0
                // (waited at the top of row r - 1, with rows r + 1 and r + 2 issued) with 2
                if (r == 0) cp_async_wait<3>();
                else cp_async_wait<2>();
                return true;
            }
            const unsigned q = first + (unsigned)r;
            return mbar_wait(sm.bar + (q % kMixSlots), (q / kMixSlots) & 1u);
        };
        if (TMA && threadIdx.x == 0)
            for (int r = 0; r < kMixSlots && r < nrows; ++r) issue(r);
        if (!TMA)
            for (int r = 0; r < kMixSlots; ++r) issue(r);
        // gathers of the scatterer series, one row ahead
        float2 gm = {0.f, 0.f}, gp = {0.f, 0.f};
        const float2 *sm32 = reinterpret_cast<const float2 *>(a.s_m32);
        const float2 *sp32 = reinterpret_cast<const float2 *>(a.s_p32);
        auto gather = [&](int r, float2 &m, float2 &p) {
            const float *src = sm.stage + (size_t)slot_of(r) * kMixArrays * kMixCols;
            int i0 = __float_as_int(src[kAindm * kMixCols + threadIdx.x]);
            int i1 = __float_as_int(src[kAindp * kMixCols + threadIdx.x]);
            i0 += a.tmod_m;
            i0 = i0 >= a.n_m ? i0 - a.n_m : i0;
            i1 += a.tmod_p;
            i1 = i1 >= a.n_p ? i1 - a.n_p : i1;
            if (col_ok) {
                m = __ldg(sm32 + i0);
                p = __ldg(sp32 + i1);
            }
        };
        // every lane waits (acquiring the copied data), the warp agrees on the outcome
        int fail_row = -1;
        bool ok = __all_sync(0xffffffffu, wait_row(0));
        if (!ok) fail_row = 0;
        if (ok && bragg) gather(0, gm, gp);
        for (int i = 0; i < nrows && ok; ++i) {
            // rows i and i + 1 have landed
            if (i + 1 < nrows) {
                ok = __all_sync(0xffffffffu, wait_row(i + 1));
                if (!ok) { fail_row = i + 1; break; }
            }
            const int slot = slot_of(i);
            float dx, dy, dz, diffx, diffy, dxx = 0.f, dyy = 0.f, dxy = 0.f;
            float sc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
            {
                const float *src = sm.stage + (size_t)slot * kMixArrays * kMixCols;
                const int t = threadIdx.x;
                dx = src[kAdx * kMixCols + t]; dy = src[kAdy * kMixCols + t]; dz = src[kAdz * kMixCols + t];
                diffx = src[kAdiffx * kMixCols + t]; diffy = src[kAdiffy * kMixCols + t];
                if (kodis) {
                    dxx = src[kAdxx * kMixCols + t];
                    dyy = src[kAdyy * kMixCols + t];
                    dxy = src[kAdxy * kMixCols + t];
                }
                if (load_scat) {
                    sc[0][0] = src[kAscat * kMixCols + t];
                    sc[0][1] = src[(kAscat + 1) * kMixCols + t];
                    if (npol == 2) {
                        sc[1][0] = src[(kAscat + 2) * kMixCols + t];
                        sc[1][1] = src[(kAscat + 3) * kMixCols + t];
                    }
                }
            }
            const float2 cm = gm, cp = gp;
            if (bragg && i + 1 < nrows) gather(i + 1, gm, gp);
            // release the slot of row i; the last of the four warps refills it with row i + 4
            __syncwarp();
            if (TMA && lane == 0) {
                __threadfence_block();
                if (atomicAdd(sm.cnt + slot, 1) == 3) {
                    sm.cnt[slot] = 0;
                    __threadfence_block();
                    if (i + kMixSlots < nrows) issue(i + kMixSlots);
                }
            }
            if constexpr (!TMA) issue(i + kMixSlots);  // this thread's column of the slot is read
            if (!col_ok) continue;

            const float *rt = sm.rt + i * RT;
            const float sin_az = rt[3];
            // ---- range offset, bin and LUT index ----
            const float delta = fmaf(dy, sin_az, fmaf(dx, sin_i, -(cos_i * dz)));
            const float S = Ch + rt[0];                                   // exact
            const float r = fmaf(delta, inv_bs, Cl + rt[1]);
            float fl = floorf(S + r);
            float frac = (S - fl) + r;
            if (frac < 0.f) { fl -= 1.f; frac += 1.f; }
            else if (frac >= 1.f) { fl += 1.f; frac -= 1.f; }
            const float x20 = fmaf(-20.f, frac, 20.f);
            float lutf = rintf(x20);
            // error bound of frac (float32 delta and rounding), with a wide margin
            const float eb = 4.76837158e-7f * ((fabsf(dz) + fabsf(dx) + fabsf(dy)) * inv_bs + fabsf(r) + 2.f);
            int bin_d, lut;
            const bool finite = fabsf(fl) < 1.0e9f;
            if (!finite || frac < eb || frac > 1.f - eb || fabsf(fabsf(x20 - lutf) - 0.5f) < 20.f * eb + 1e-6f) {
                // near a rounding boundary (or not finite): the float64 drop-in's decision
                const double srs = srs_f64(a.sr_col[x], a.cos_inc[x], a.sin_inc[x], sm.raz[i], sm.raz[sm.rcap + i],
                                           dx, dy, dz);
                bin_and_lut(srs, a.min_sr, a.binsize, kSincOvs, bin_d, lut);
            } else {
                bin_d = (int)fl;
                lut = (int)lutf;
            }
            // ---- two-way phase of the facet: phi_x + phi_y - 2 k0 delta ----
            const float th = wrap_pi((phi_x + rt[2]) - reduce_prod(khi, klo, delta));

            c64 scene[2] = {{0.f, 0.f}, {0.f, 0.f}};
            if (kodis) {
                // Kodis stationary point of the facet (kodis.py:38-73) in float32
                const float J = __fsub_rn(__fmul_rn(dxx, dyy), __fmul_rn(dxy, dxy));
                if (J != 0.f) {
                    const float Ja = fabsf(J);
                    const float inv_j = __fdividef(1.f, Ja);
                    const float cos_azp = rt[4], sin_azp = rt[5];
                    const float ty = diffy - tan_i * sin_azp;
                    const float tx = diffx - tan_i * cos_azp;
                    const float ddx = inv_j * (dxy * ty - dyy * tx);
                    const float ddy = inv_j * (dxy * tx - dxx * ty);
                    const float keb = 7.62939453e-6f * inv_j * (fabsf(dxx) + fabsf(dyy) + 2.f * fabsf(dxy)) *
                                      (fabsf(tx) + fabsf(ty) + fabsf(diffx) + fabsf(diffy) + tan_i) + 1e-30f;
                    bool inside = (fabsf(ddx) < hdx) && (fabsf(ddy) < hdy);
                    if (fabsf(fabsf(ddx) - hdx) < keb || fabsf(fabsf(ddy) - hdy) < keb) {
                        // near the facet window: the float64 drop-in's test
                        const double ij = (double)(1.f / Ja);
                        const double tan_d = a.tan_inc[x];
                        const double tyd = (double)diffy - tan_d * a.rowtab[4LL * a.ny + y0 + i];
                        const double txd = (double)diffx - tan_d * a.rowtab[3LL * a.ny + y0 + i];
                        const double dxd = ij * ((double)dxy * tyd - (double)dyy * txd);
                        const double dyd = ij * ((double)dxy * txd - (double)dxx * tyd);
                        inside = (-a.kodis.hdx < dxd) && (dxd < a.kodis.hdx) && (-a.kodis.hdy < dyd) &&
                                 (dyd < a.kodis.hdy);
                    }
                    if (inside) {
                        const float ddz = ddx * diffx + ddy * diffy;
                        const float off = sin_i * cos_azp * ddx + sin_i * sin_azp * ddy - cos_i * ddz;
                        const float ph = wrap_pi((phi_x + rt[2]) - reduce_prod(khi, klo, delta + off));
                        float s, c;
                        __sincosf(ph, &s, &c);
                        const float sgn = J > 0.f ? (float)((dxx > 0.f) - (dxx < 0.f)) : 0.f;
                        const float fac = __fadd_rn(__fadd_rn(__fmul_rn(diffx, diffx), __fmul_rn(diffy, diffy)), 1.f);
                        const float amp = fac * 3.5449077018110318f / sqrtf(Ja);    // sqrt(4 pi)
                        // (R/2) eps fac e^{i ph} / sqrt|J|, eps = sign(Dxx) or 1j
                        const c64 re = J > 0.f ? c64{hr * sgn, hi_ * sgn} : c64{-hi_, hr};
                        const c64 e = cmul(re, c64{c * amp, s * amp});
                        spec_sum += (double)e.re * e.re + (double)e.im * e.im;
                        scene[0] = e;
                        scene[1] = e;
                    }
                }
            }
            if (bragg) {
                if (REFRESH != 0 && refresh) {
                    float hh[2], vv[2];
                    const int y = y0 + i;
                    if (!FAST && a.lut) {
                        const int ai = lut_az_index(a, a.rowtab[2LL * a.ny + y]);
                        float r0[2], r1[2];
                        romeiser_lut<float>(a, ai, diffx, diffy, 0, r0);
                        if (npol == 2) romeiser_lut<float>(a, ai, diffx, diffy, 1, r1);
                        else { r1[0] = r0[0]; r1[1] = r0[1]; }
                        const bool vv_first = a.rom.pol == POL_VV;
                        hh[0] = vv_first ? r1[0] : r0[0]; hh[1] = vv_first ? r1[1] : r0[1];
                        vv[0] = vv_first ? r0[0] : r1[0]; vv[1] = vv_first ? r0[1] : r1[1];
                    } else {
                        romeiser_facet<float>(a.rom, (float)a.inc[x], rt[6], rt[4], rt[5], diffx, diffy, hh, vv);
                    }
                    if (!FAST && a.use_hmtf) {
                        float hm = a.hmtf[(long long)y * a.nx + x];
                        hm = hm < -1.f ? -1.f : hm;
                        const float f = 1.f + hm;
                        hh[0] *= f; hh[1] *= f; vv[0] *= f; vv[1] *= f;
                    }
                    const long long idx = (long long)y * a.nx + x;
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        if (p < npol) {
                            const bool use_vv = a.rom.pol == POL_VV || (a.rom.pol == POL_DP && p == 1);
                            const float r0 = use_vv ? vv[0] : hh[0], r1 = use_vv ? vv[1] : hh[1];
                            bragg_sum[p] += (double)r0 + (double)r1;
                            sc[p][0] = sqrtf(r0);
                            sc[p][1] = sqrtf(r1);
                            if (a.out0 == 0) {
                                scat[(2 * p) * npix + idx] = sc[p][0];
                                scat[(2 * p + 1) * npix + idx] = sc[p][1];
                            }
                        }
                    }
                }
                // Bragg phases -2 k0 r -/+ 2 k0 t_step c_b (az_step + 1)
                float s0, c0, s1, c1;
                __sincosf(th - cap_r, &s0, &c0);
                __sincosf(th + cap_r, &s1, &c1);
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    if (p < npol) {
                        const c64 l0 = cmul(c64{sc[p][0] * c0, sc[p][0] * s0}, c64{cm.x, cm.y});
                        const c64 l1 = cmul(c64{sc[p][1] * c1, sc[p][1] * s1}, c64{cp.x, cp.y});
                        scene[p] = cadd(scene[p], cadd(l0, l1));
                    }
                }
            }
            // ---- channels: antenna pattern x ATI phase (row) x XTI phase (facet) ----
            c64 coef[NOUT];
            float wave_dinc = 0.f;
            if (FAST == 2 || (FAST == 0 && a.any_xti)) wave_dinc = (dz * sin_i + dx * sin_i) * inv_sr0;
#pragma unroll
            for (int k = 0; k < NOUT; ++k) {
                if (FAST || k < a.nout) {
                    // fast configurations: one polarisation, output k is channel out0 + k (mode 1:
                    // no XTI phase; mode 2: the XTI flags of the tile's output word)
                    const unsigned okb = FAST == 1 ? (unsigned)(a.out0 + k) : outs >> (5 * k);
                    const int c = okb & 7;
                    const c64 f = {rt[kMixRT + 2 * c], rt[kMixRT + 2 * c + 1]};
                    c64 v = cmul((!FAST && (okb & 8)) ? scene[1] : scene[0], f);
                    if (FAST != 1 && (okb & 16)) {
                        const float ph = wrap_pi(kxti[k] * (dinc0 + wave_dinc));
                        float s, cc;
                        __sincosf(ph, &s, &cc);
                        v = cmul(v, c64{cc, s});
                    }
                    coef[k] = v;
                } else {
                    coef[k] = {0.f, 0.f};
                }
            }
            if (bin_d > -(1 << 29)) win.add(bin_d - kSincTaps / 2, lut, coef, sm.wtab, a.sinc, cb);
        }
        if (!ok) {
            // a wait gave up: record it, and let every copy that may be in flight (rows
            // fail_row .. fail_row + 3, one per slot) land before the shared memory can go away
            bad = true;
            if (lane == 0) {
                atomicOr(reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(a.rowtab) +
                                                 mix_hdr_offset(a.ny, a.nch)) + 1, 1);
                for (int r = fail_row; r < fail_row + kMixSlots && r < nrows; ++r) wait_row(r);
            }
            __syncwarp();
        }
        if constexpr (!TMA) cp_async_wait<0>();  // no copy may land in the ring after the tile
        rseq = first + (unsigned)nrows;
    }
    // every warp is past its last row: the ring holds no live data, its memory is the
    // flush scratch
    __syncthreads();
    {
        float *scr = sm.stage + (size_t)(threadIdx.x >> 5) * 32 * kMixS * 2;
        int *sbase = reinterpret_cast<int *>(sm.stage + (size_t)4 * 32 * kMixS * 2) + 32 * (threadIdx.x >> 5);
        warp_flush<NOUT>(win, cb, scr, sbase);
    }
    __syncthreads();
    // CTA bins -> raw row, compensated: first every returning add of this thread's bins (so
    // that their round trips overlap), then the rounding errors, as plain reductions, into
    // the compensation row
    constexpr int kPer = (NOUT * kMixNbw + kMixCols - 1) / kMixCols;
    float vr[kPer][2], orv[kPer][2], er[kPer][2];
    long long off[kPer];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        const int i = threadIdx.x + k * kMixCols;
        off[k] = -1;
        vr[k][0] = vr[k][1] = orv[k][0] = orv[k][1] = er[k][0] = er[k][1] = 0.f;
        if (i < a.nout * kMixNbw) {
            const int o = i / kMixNbw, lb = i - o * kMixNbw;
            const int b = cb.cta_base + lb;
            if (b >= 0 && b < a.nbins) {
                off[k] = (long long)o * cb.out_stride + 2 * b;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const float h = sm.bhi[2 * i + c], l = sm.blo[2 * i + c];
                    vr[k][c] = __fadd_rn(h, l);
                    er[k][c] = two_sum_err(h, l, vr[k][c]);
                    if (vr[k][c] != 0.f) orv[k][c] = atomicAdd(cb.out + off[k] + c, vr[k][c]);
                }
            }
        }
    }
    if (cb.lo_row) {
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if (off[k] < 0) continue;
            const int i = threadIdx.x + k * kMixCols;
            const int o = i / kMixNbw, b = cb.cta_base + (i - o * kMixNbw);
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                if (vr[k][c] == 0.f) continue;
                const float e = two_sum_err(orv[k][c], vr[k][c], __fadd_rn(orv[k][c], vr[k][c])) + er[k][c];
                if (e != 0.f) atomicAdd(cb.lo_row + (long long)o * 2 * a.nbins + 2 * b + c, e);
            }
        }
    }
}

template <int NOUT> OCS_D void mix_init(const MixSmem<NOUT> &sm) {
    if (threadIdx.x < kMixSlots) {
        mbar_init(sm.bar + threadIdx.x, 1);
        sm.cnt[threadIdx.x] = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();
}

template <int NOUT, bool KODIS, int REFRESH, int FAST = 0>
__global__ void __launch_bounds__(kMixCols, NOUT < 4 ? 4 : 2)
pulse_mixed_kernel(const __grid_constant__ PulseArgs a, const __grid_constant__ MixMaps maps, float *lo_row) {
    extern __shared__ __align__(128) unsigned char smem[];
    const MixSmem<NOUT> sm = mix_smem<NOUT>(smem, a.nch, kPulseRows);
    build_wtab<float, kMixS>(sm.wtab, a.sinc, kSincTaps, kSincOvs);
    mix_init<NOUT>(sm);
    const int tiles = ((a.nx + kMixCols - 1) / kMixCols) * ((a.ny + a.tile_rows - 1) / a.tile_rows);
    double spec_sum = 0.0, bragg_sum[2] = {0.0, 0.0};
    unsigned rseq = 0;
    bool bad = false;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        mix_tile<NOUT, KODIS, true, REFRESH, FAST>(a, &maps, lo_row, tile, a.tile_rows, sm, rseq, bad, spec_sum,
                                                   bragg_sum);
    if (a.out0 == 0) {
        if (KODIS) block_atomic_sum(spec_sum, &a.nrcs_spec[a.az_step], sm.sred);
        if (a.do_bragg && a.refresh)
            for (int p = 0; p < a.npol; ++p)
                block_atomic_sum(bragg_sum[p], &a.nrcs_bragg[(long long)p * a.az_steps + a.az_step], sm.sred);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && lo_row)
        reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(a.rowtab) + mix_hdr_offset(a.ny, a.nch))[0] =
            a.az_step;
}

}  // namespace ocs
