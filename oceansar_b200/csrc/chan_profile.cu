// Standalone facet-to-range-bin accumulation: the drop-in for chan_profile_numba
// (oceansar/radarsim/range_profile.py:83-116 -> profile_integrator :22-49 and
// profile_integrator_1d :52-80).
//
// Facets come in arbitrary order (the caller's flattened slant-range / scene arrays), so
// each thread takes a run of consecutive facets -- consecutive facets of a flattened
// surface row are consecutive ground-range columns, whose bins grow monotonically -- and
// accumulates them through the register window of accum.cuh.  Facets that keep their
// [ny][nx] surface shape go through the fine-grid kernel below (one shared-memory add per
// facet into a (bin, LUT index) histogram, convolved with the pulse once per tile).  Output
// is accumulated in place (+=), never cleared, exactly like the reference.
#include "accum.cuh"

namespace ocs {

constexpr int kProfThreads = 256;

// Dynamic shared memory layout: [wtab | CTA bin accumulator].
template <typename T, int S>
__global__ void __launch_bounds__(kProfThreads)
chan_profile_kernel(const double *__restrict__ srg, const cplx<T> *__restrict__ scene,
                    long long npts, long long row_len, double binsize, double min_sr,
                    const float *__restrict__ sinc, int taps, int ovs, T *__restrict__ out,
                    int nbins, long long out_row_stride, int chunk, int cta_nbw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *wtab = reinterpret_cast<T *>(smem_raw);
    const int wlen = wtab_len<T, S>(taps, ovs);
    T *acc = wtab + ((wlen + 3) & ~3);

    // Row handling (profile_integrator_1d): facets of row r accumulate into out row r.
    // A CTA covers facets [f0, f0 + blockDim*chunk) of one row.
    const long long ctas_per_row = (row_len + (long long)kProfThreads * chunk - 1) /
                                   ((long long)kProfThreads * chunk);
    const long long row = blockIdx.x / ctas_per_row;
    const long long f0 = row * row_len + (blockIdx.x % ctas_per_row) * (long long)kProfThreads * chunk;
    const long long fend = min(row * row_len + row_len, npts);
    if (f0 >= fend) return;

    build_wtab<T, S>(wtab, sinc, taps, ovs);

    CtaBins<T, 1> cb;
    cb.acc = acc;
    cb.nbw = cta_nbw;
    cb.nout = 1;
    cb.nbins = nbins;
    cb.out = out + 2 * row * out_row_stride;
    cb.out_stride = 0;
    if (cta_nbw >= nbins) {
        cb.cta_base = 0;
    } else {
        int b0, l0;
        bin_and_lut(srg[f0], min_sr, binsize, ovs, b0, l0);
        cb.cta_base = b0 - cta_nbw / 2;
    }
    cb.zero();
    __syncthreads();

    BinWindow<T, S, 1> win;
    win.reset();
    const int half = taps / 2;
    const long long my0 = f0 + (long long)threadIdx.x * chunk;
    for (int k = 0; k < chunk; ++k) {
        long long i = my0 + k;
        if (i >= fend) break;
        int bin_d, lut;
        bin_and_lut(srg[i], min_sr, binsize, ovs, bin_d, lut);
        if (bin_d < -(1 << 29)) continue;
        cplx<T> c[1] = {scene[i]};
        win.add(bin_d - half, lut, c, wtab, sinc, taps, ovs, cb);
    }
    win.flush(cb);
    __syncthreads();
    cb.flush_to_global();
}

template <typename T, int S>
static int launch_chan_profile(const double *srg, const void *scene, long long naz, long long npts,
                               double binsize, double min_sr, const float *sinc, int taps, int ovs,
                               T *out, int nbins, cudaStream_t stream) {
    if (taps < 1 || taps > S || ovs < 1 || npts < 0 || naz < 1 || nbins < 0) return OCS_ERR_ARG;
    if (npts == 0 || nbins == 0) return OCS_OK;
    const int wlen = wtab_len<T, S>(taps, ovs);
    const size_t wtab_bytes = (size_t)((wlen + 3) & ~3) * sizeof(T);
    const size_t budget = 96 * 1024;
    if (wtab_bytes > budget / 2) return OCS_ERR_UNSUPPORTED;
    long long cap = (long long)((budget - wtab_bytes) / (2 * sizeof(T)));
    int nbw = (int)(nbins < cap ? nbins : cap);
    if (nbw > 8192) nbw = 8192;
    // Enough CTAs to fill the GPU, but long enough runs per thread to keep the windows warm.
    long long total = naz * npts;
    long long ch = total / (148LL * 8 * kProfThreads);
    int chunk = (int)(ch < 1 ? 1 : (ch > 32 ? 32 : ch));
    long long ctas_per_row = (npts + (long long)kProfThreads * chunk - 1) / ((long long)kProfThreads * chunk);
    long long grid = ctas_per_row * naz;
    if (grid > 0x7fffffffLL) return OCS_ERR_SIZE;
    size_t smem = wtab_bytes + (size_t)nbw * 2 * sizeof(T);
    auto kern = chan_profile_kernel<T, S>;
    if (ensure_smem((const void *)kern, smem) != cudaSuccess)
        return OCS_ERR_CUDA;
    kern<<<(unsigned)grid, kProfThreads, smem, stream>>>(
        srg, reinterpret_cast<const cplx<T> *>(scene), naz * npts, npts, binsize, min_sr, sinc, taps,
        ovs, out, nbins, (long long)nbins, chunk, nbw);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------
// Two-dimensional layout: the facets are a [ny][nx] surface (rows = azimuth, columns =
// ground range), as sar_raw flattens them.  A CTA takes tiles of kC2Cols columns x up to
// kC2Rows rows; a thread owns one column and walks down the rows, so a warp reads 32
// consecutive facets of a row (coalesced) and every thread's range bin drifts only with
// the azimuth curvature and the surface displacement -- its register window almost never
// moves.
constexpr int kC2Cols = 128;
constexpr int kC2Rows = 64;
constexpr int kC2Nbw = 256;

// Register-batched form of the two-dimensional accumulation: persistent CTAs walk tiles
// of kC2Cols columns x tile_rows rows; every thread loads the slant ranges and scene
// values of its column for kRB rows at once (2 kRB independent coalesced loads in flight
// per thread) and then runs them through its register window.  The kernel is bound by
// the latency of each facet's dependent chain (bin -> weight row -> multiply-adds), so
// resident warps count most: single precision runs 4-row batches at 6 CTAs per SM
// (within 80 registers), float64 8-row batches at 4 (its window takes twice the registers).
template <typename T> __host__ __device__ constexpr int rows_per_batch() { return sizeof(T) == 4 ? 4 : 8; }
template <typename T> __host__ __device__ constexpr int ctas_per_sm_2d() { return sizeof(T) == 4 ? 6 : 4; }

template <typename T, int S>
__global__ void __launch_bounds__(kC2Cols, ctas_per_sm_2d<T>())
chan_profile_2d_regs_kernel(const double *__restrict__ srg, const cplx<T> *__restrict__ scene, int ny, int nx,
                            double binsize, double min_sr, const float *__restrict__ sinc, int taps, int ovs,
                            T *__restrict__ out, int nbins, int tile_rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *wtab = reinterpret_cast<T *>(smem_raw);
    const int wlen = wtab_len<T, S>(taps, ovs);
    T *acc = wtab + ((wlen + 3) & ~3);
    build_wtab<T, S>(wtab, sinc, taps, ovs);
    const int tiles_x = (nx + kC2Cols - 1) / kC2Cols;
    const int tiles = tiles_x * ((ny + tile_rows - 1) / tile_rows);
    const double inv_binsize = 1.0 / binsize;
    const int half = taps / 2;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int x0 = (tile % tiles_x) * kC2Cols;
        const int y0 = (tile / tiles_x) * tile_rows;
        const int nrows = min(tile_rows, ny - y0);
        const int x = x0 + threadIdx.x;
        __syncthreads();                  // the previous tile's bins are flushed (and wtab built)
        CtaBins<T, 1> cb;
        cb.acc = acc;
        cb.nbw = kC2Nbw;
        cb.nout = 1;
        cb.nbins = nbins;
        cb.out = out;
        cb.out_stride = 0;
        {
            int b0, l0;
            bin_and_lut(srg[(long long)y0 * nx + x0], min_sr, binsize, ovs, b0, l0);
            cb.cta_base = (b0 > -(1 << 29)) ? b0 - kC2Nbw / 4 : 0;
        }
        cb.zero();
        __syncthreads();
        BinWindow<T, S, 1> win;
        win.reset();
        if (x < nx) {
            const long long g0 = (long long)y0 * nx + x;
            constexpr int kRB = rows_per_batch<T>();
            for (int i0 = 0; i0 < nrows; i0 += kRB) {
                double sr[kRB];
                cplx<T> c[kRB];
#pragma unroll
                for (int k = 0; k < kRB; ++k) {
                    if (i0 + k < nrows) {
                        const long long g = g0 + (long long)(i0 + k) * nx;
                        sr[k] = __ldg(srg + g);
                        c[k] = scene[g];
                    }
                }
#pragma unroll
                for (int k = 0; k < kRB; ++k) {
                    if (i0 + k >= nrows) break;
                    int bin_d, lut;
                    // FP64: IEEE division, bin / LUT bit-identical with numpy; single
                    // precision: reciprocal multiply (a one-ulp difference in the bin coordinate)
                    if (sizeof(T) == 8) bin_and_lut(sr[k], min_sr, binsize, ovs, bin_d, lut);
                    else bin_and_lut_fast(sr[k], min_sr, inv_binsize, ovs, bin_d, lut);
                    if (bin_d < -(1 << 29)) continue;
                    cplx<T> cc[1] = {c[k]};
                    win.add(bin_d - half, lut, cc, wtab, sinc, taps, ovs, cb);
                }
            }
        }
        win.flush(cb);
        __syncthreads();
        cb.flush_to_global();
    }
}

template <typename T, int S>
static int launch_chan_profile_2d_regs(const double *srg, const void *scene, long long ny, long long nx,
                                       double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                       int nbins, cudaStream_t stream) {
    if (taps < 1 || taps > S || ovs < 1) return OCS_ERR_ARG;
    if (ny > 0x7fffffffLL || nx > 0x7fffffffLL) return OCS_ERR_SIZE;
    const int wlen = wtab_len<T, S>(taps, ovs);
    const size_t smem = (size_t)((wlen + 3) & ~3) * sizeof(T) + (size_t)kC2Nbw * 2 * sizeof(T);
    auto kern = chan_profile_2d_regs_kernel<T, S>;
    if (ensure_smem((const void *)kern, smem) != cudaSuccess) return OCS_ERR_CUDA;
    const int resident = resident_ctas((const void *)kern, kC2Cols, smem);
    if (resident <= 0) return OCS_ERR_CUDA;
    const long long tiles_x = (nx + kC2Cols - 1) / kC2Cols;
    const long long want = (long long)resident * ((tiles_x * ((ny + kC2Rows - 1) / kC2Rows) + resident - 1) / resident);
    long long per_col = want / tiles_x;
    if (per_col < 1) per_col = 1;
    long long rows = (ny + per_col - 1) / per_col;
    rows = rows < 8 ? (ny < 8 ? ny : 8) : (rows > kC2Rows ? kC2Rows : rows);
    const long long tiles = tiles_x * ((ny + rows - 1) / rows);
    const long long grid = tiles < resident ? tiles : resident;
    kern<<<(unsigned)grid, kC2Cols, smem, stream>>>(srg, reinterpret_cast<const cplx<T> *>(scene), (int)ny, (int)nx,
                                                      binsize, min_sr, sinc, taps, ovs, out, nbins, (int)rows);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------
// Fine-grid form of the two-dimensional accumulation.  A facet's taps depend only on its
// range bin and LUT index, so with H[bin][l] = the sum of the coefficients of the facets
// whose bin is `bin` and whose LUT index is l,
//     out[b] = sum over facets of sinc[lut + j ovs] c,  j = b - (bin - taps/2)
//            = sum_{j < taps} sum_{l <= ovs} sinc[l + j ovs] H[b + taps/2 - j][l].
// A CTA adds each facet's coefficient once into a shared-memory H that spans kHB bins
// around its tile of 128 columns x tile_rows rows (two shared atomic adds per facet into
// separate real and imaginary planes, instead of a multiply-add per tap and window slot; no
// register window, so 8 to 12 CTAs fit per SM), then convolves H with the oversampled pulse
// once per tile and adds the result to the output with global atomics.  A tile whose first
// and last rows span more bins than H holds is walked in narrower column groups (64 or 32
// columns, two or four rows per step, one H each); facets whose bin still falls outside H,
// and facets with non-finite coefficients (which must touch exactly their own taps, with
// the reference's complex product), take the direct path of per-tap global atomics.  Bins
// outside [0, nbins) are dropped, as the reference's edge branch does.
constexpr int kHThreads = 128;
constexpr int kHRB = 4;             // rows of loads in flight per thread
constexpr int kHB = 64;             // bins held by H
// Resident CTAs per SM: single precision fits twelve within 40 registers; float64 keeps
// eight (its division and 16-byte loads need the registers).
template <typename T> __host__ __device__ constexpr int hist_ctas_per_sm() { return sizeof(T) == 4 ? 12 : 8; }

// floor(bin_f) and round_half_even(ovs (1 - frac)) without conversion instructions: adding
// M = 1.5 * 2^52 rounds a value below 2^51 in magnitude to an integer held in the low word
// of the sum (rounded down, or to nearest even), exactly what floor and numpy's rint give.
// Ranges whose floor is not below 1e9 in magnitude (NaN, inf, absurd) get the invalid
// marker bin, as bin_and_lut does.
OCS_D void bin_lut_magic(double bin_f, double dovs, int &bin_d, int &lut) {
    constexpr double M = 6755399441055744.0;
    const double t = __dadd_rd(bin_f, M);
    const double fl = __dsub_rn(t, M);
    if (!(fabs(fl) < 1.0e9)) {
        bin_d = -(1 << 30);
        lut = 0;
        return;
    }
    bin_d = __double2loint(t);
    lut = __double2loint(__dadd_rn(__dmul_rn(dovs, __dsub_rn(1.0, __dsub_rn(bin_f, fl))), M));
}

template <typename T>
OCS_D void direct_taps(int bin_d, int lut, cplx<T> c, const float *sinc, int taps, int ovs, T *out, int nbins) {
    const int first = bin_d - taps / 2;
    for (int j = 0; j < taps; ++j) {
        const int b = first + j;
        if (b < 0 || b >= nbins) continue;
        const T w = (T)sinc[lut + j * ovs];
        atomicAdd(out + 2 * b, w * c.re - (T)0 * c.im);
        atomicAdd(out + 2 * b + 1, w * c.im + (T)0 * c.re);
    }
}

// Scene value of one facet: one vector load when the scene is aligned to its element pair.
template <typename T, bool VEC> OCS_D cplx<T> load_scene(const cplx<T> *p) {
    if constexpr (VEC) {
        if constexpr (sizeof(T) == 4) {
            const float2 v = __ldg(reinterpret_cast<const float2 *>(p));
            return {v.x, v.y};
        } else {
            const double2 v = __ldg(reinterpret_cast<const double2 *>(p));
            return {v.x, v.y};
        }
    } else {
        return {__ldg(&p->re), __ldg(&p->im)};
    }
}

template <typename T> OCS_HD size_t hist_smem_bytes(int taps, int ovs) {
    return (((size_t)taps * (ovs + 1) * sizeof(T) + 15) & ~(size_t)15) + (size_t)kHB * (ovs + 1) * sizeof(cplx<T>) +
           16 * sizeof(int);
}

template <typename T, bool VEC>
__global__ void __launch_bounds__(kHThreads, hist_ctas_per_sm<T>())
chan_profile_2d_hist_kernel(const double *__restrict__ srg, const cplx<T> *__restrict__ scene, int ny, int nx,
                            double binsize, double min_sr, const float *__restrict__ sinc, int taps, int ovs,
                            T *__restrict__ out, int nbins, int tile_rows) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = ovs + 1;
    T *w = reinterpret_cast<T *>(smem_raw);                                   // [taps][L]
    // H as two planes (real, imaginary) of [kHB][L]: the lanes of one atomic add spread
    // over all 32 banks
    T *Hre = reinterpret_cast<T *>(smem_raw + (((size_t)taps * L * sizeof(T) + 15) & ~(size_t)15));
    T *Him = Hre + kHB * L;
    int *s_lo = reinterpret_cast<int *>(Him + kHB * L);                       // [4] per-warp bin estimates
    int *s_hi = s_lo + 4;
    int *s_tlo = s_lo + 8;                                                    // [4] per-warp touched cells
    int *s_thi = s_lo + 12;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    for (int i = t; i < taps * L; i += kHThreads) {
        const int j = i / L, l = i - j * L;
        w[i] = (T)sinc[l + j * ovs];
    }
    const int tiles_x = (nx + kHThreads - 1) / kHThreads;
    const int tiles = tiles_x * ((ny + tile_rows - 1) / tile_rows);
    const double inv_binsize = 1.0 / binsize;
    const double dovs = (double)ovs;
    const int half = taps / 2;
    auto bin_of = [&](double s, int &bin_d, int &lut) {
        // float64: IEEE division (bins and LUT indices bit-identical with numpy); single
        // precision: reciprocal multiply (a one-ulp difference in the bin coordinate)
        const double bin_f = sizeof(T) == 8 ? ddiv(dsub(s, min_sr), binsize) : (s - min_sr) * inv_binsize;
        bin_lut_magic(bin_f, dovs, bin_d, lut);
    };
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int x0 = (tile % tiles_x) * kHThreads;
        const int y0 = (tile / tiles_x) * tile_rows;
        const int nrows = min(tile_rows, ny - y0);
        __syncthreads();                  // the previous tile's convolution has read H (and w is built)
        // ---- bins of the tile's first and last rows, per warp of 32 columns ----
        {
            int lo = 0x3fffffff, hi = -0x3fffffff;
            const int x = x0 + t;
            if (x < nx) {
                int b, l;
                bin_of(__ldg(srg + (long long)y0 * nx + x), b, l);
                if (b > -(1 << 29)) { lo = min(lo, b); hi = max(hi, b); }
                bin_of(__ldg(srg + (long long)(y0 + nrows - 1) * nx + x), b, l);
                if (b > -(1 << 29)) { lo = min(lo, b); hi = max(hi, b); }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
                hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            }
            if (lane == 0) { s_lo[warp] = lo; s_hi[warp] = hi; }
        }
        for (int i = t; i < kHB * L; i += kHThreads) { Hre[i] = (T)0; Him[i] = (T)0; }
        __syncthreads();
        // column groups: 128 columns when the tile's bins fit H with room for the jitter
        // between its first and last rows, else 64 or 32
        int gw = kHThreads;
        {
            const int lo = min(min(s_lo[0], s_lo[1]), min(s_lo[2], s_lo[3]));
            const int hi = max(max(s_hi[0], s_hi[1]), max(s_hi[2], s_hi[3]));
            const int lo01 = min(s_lo[0], s_lo[1]), hi01 = max(s_hi[0], s_hi[1]);
            const int lo23 = min(s_lo[2], s_lo[3]), hi23 = max(s_hi[2], s_hi[3]);
            if (hi - lo > kHB - 16) gw = (max(hi01 - lo01, hi23 - lo23) > kHB - 16) ? 32 : 64;
        }
        const int ngroups = kHThreads / gw;
        const int rstep = kHThreads / gw;
        for (int g = 0; g < ngroups; ++g) {
            const int xg0 = x0 + g * gw;
            if (xg0 >= nx) break;         // uniform: the tile's remaining groups lie past the surface
            if (g > 0) {
                __syncthreads();          // the previous group's convolution has read H
                for (int i = t; i < kHB * L; i += kHThreads) { Hre[i] = (T)0; Him[i] = (T)0; }
                __syncthreads();
            }
            int base;
            {
                const int w0 = g * gw / 32, w1 = w0 + gw / 32;
                int lo = 0x3fffffff, hi = -0x3fffffff;
                for (int k = w0; k < w1; ++k) { lo = min(lo, s_lo[k]); hi = max(hi, s_hi[k]); }
                base = hi >= lo ? lo - (kHB - (hi - lo + 1)) / 2 : 0;
            }
            const int x = xg0 + t % gw;
            int tlo = kHB, thi = -1;
            if (x < nx) {
                const long long g0 = (long long)y0 * nx + x;
                // one facet: into H, or (outside H, non-finite, or an invalid range whose
                // marker bin puts every tap below 0) by the direct path
                auto facet = [&](double s, cplx<T> c) {
                    int bin_d, lut;
                    bin_of(s, bin_d, lut);
                    const int cb = (int)((unsigned)bin_d - (unsigned)base);
                    if ((unsigned)cb < (unsigned)kHB && isfinite(c.re + c.im)) {
                        const int cell = cb * L + lut;
                        atomicAdd(Hre + cell, c.re);
                        atomicAdd(Him + cell, c.im);
                        tlo = min(tlo, cb);
                        thi = max(thi, cb);
                    } else {
                        direct_taps<T>(bin_d, lut, c, sinc, taps, ovs, out, nbins);
                    }
                };
                int r0 = t / gw;
                for (; r0 + (kHRB - 1) * rstep < nrows; r0 += kHRB * rstep) {      // full batches
                    double sr[kHRB];
                    cplx<T> c[kHRB];
#pragma unroll
                    for (int k = 0; k < kHRB; ++k) {
                        const long long gi = g0 + (long long)(r0 + k * rstep) * nx;
                        sr[k] = __ldg(srg + gi);
                        c[k] = load_scene<T, VEC>(scene + gi);
                    }
#pragma unroll
                    for (int k = 0; k < kHRB; ++k) facet(sr[k], c[k]);
                }
                for (; r0 < nrows; r0 += rstep) {                                   // the rest
                    const long long gi = g0 + (long long)r0 * nx;
                    facet(__ldg(srg + gi), load_scene<T, VEC>(scene + gi));
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                tlo = min(tlo, __shfl_xor_sync(0xffffffffu, tlo, o));
                thi = max(thi, __shfl_xor_sync(0xffffffffu, thi, o));
            }
            if (lane == 0) { s_tlo[warp] = tlo; s_thi[warp] = thi; }
            __syncthreads();
            const int clo = min(min(s_tlo[0], s_tlo[1]), min(s_tlo[2], s_tlo[3]));
            const int chi = max(max(s_thi[0], s_thi[1]), max(s_thi[2], s_thi[3]));
            if (chi < clo) continue;      // uniform: nothing landed in H
            // ---- convolution: output bin base + clo - half + m, m < chi - clo + taps; four
            // lanes per output bin, each a quarter of the taps, summed by shuffles ----
            const int nob = chi - clo + taps;
            const int tq = (taps + 3) / 4;
            const int items = nob * 4;
            for (int i0 = 0; i0 < items; i0 += kHThreads) {
                const int i = i0 + t;
                const int m = i >> 2, jq = i & 3;
                T sre = (T)0, sim = (T)0;
                if (i < items) {
                    const int ja = jq * tq, jb = min(taps, ja + tq);
                    for (int j = ja; j < jb; ++j) {
                        const int cell = clo + m - j;          // H bin feeding output m through tap j
                        if (cell < clo || cell > chi) continue;
                        const T *hr = Hre + cell * L, *hi = Him + cell * L;
                        const T *wj = w + j * L;
                        for (int l = 0; l < L; ++l) {
                            sre = fma(wj[l], hr[l], sre);
                            sim = fma(wj[l], hi[l], sim);
                        }
                    }
                }
                sre += __shfl_xor_sync(0xffffffffu, sre, 1);
                sim += __shfl_xor_sync(0xffffffffu, sim, 1);
                sre += __shfl_xor_sync(0xffffffffu, sre, 2);
                sim += __shfl_xor_sync(0xffffffffu, sim, 2);
                const int b = base + clo - half + m;
                if (i < items && jq == 0 && b >= 0 && b < nbins) {
                    if (sre != (T)0) atomicAdd(out + 2 * b, sre);
                    if (sim != (T)0) atomicAdd(out + 2 * b + 1, sim);
                }
            }
        }
    }
}

template <typename T, bool VEC>
static int launch_chan_profile_2d_hist_v(const double *srg, const void *scene, long long ny, long long nx,
                                         double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                         int nbins, cudaStream_t stream) {
    const size_t smem = hist_smem_bytes<T>(taps, ovs);
    auto kern = chan_profile_2d_hist_kernel<T, VEC>;
    if (ensure_smem((const void *)kern, smem) != cudaSuccess) return OCS_ERR_CUDA;
    const int resident = resident_ctas((const void *)kern, kHThreads, smem);
    if (resident <= 0) return OCS_ERR_CUDA;
    // about one tile per resident CTA: tall tiles amortise the convolution and the global
    // adds of a tile over more facets
    const long long tiles_x = (nx + kHThreads - 1) / kHThreads;
    long long per_col = resident / tiles_x;
    if (per_col < 1) per_col = 1;
    long long rows = (ny + per_col - 1) / per_col;
    if (rows > 1024) rows = 1024;
    if (rows < 1) rows = 1;
    const long long tiles = tiles_x * ((ny + rows - 1) / rows);
    if (tiles > 0x7fffffffLL) return OCS_ERR_SIZE;
    kern<<<(unsigned)tiles, kHThreads, smem, stream>>>(srg, reinterpret_cast<const cplx<T> *>(scene), (int)ny,
                                                        (int)nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                                        (int)rows);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <typename T>
static int launch_chan_profile_2d_hist(const double *srg, const void *scene, long long ny, long long nx,
                                       double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                       int nbins, cudaStream_t stream) {
    if (ny > 0x7fffffffLL || nx > 0x7fffffffLL) return OCS_ERR_SIZE;
    if (((uintptr_t)scene & (2 * sizeof(T) - 1)) == 0)
        return launch_chan_profile_2d_hist_v<T, true>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out,
                                                      nbins, stream);
    return launch_chan_profile_2d_hist_v<T, false>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                                   stream);
}

template <typename T>
static int launch_chan_profile_2d_any(const double *srg, const void *scene, long long ny, long long nx,
                                      double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                      int nbins, cudaStream_t stream) {
    if (taps >= 1 && taps <= 16 && ovs >= 1 && hist_smem_bytes<T>(taps, ovs) <= 40 * 1024)
        return launch_chan_profile_2d_hist<T>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                              stream);
    if (taps <= 8)
        return launch_chan_profile_2d_regs<T, 12>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                                  stream);
    return launch_chan_profile_2d_regs<T, 16>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins, stream);
}

}  // namespace ocs

extern "C" int ocs_chan_profile_f64(const double *srg, const double *scene, int64_t npts,
                                    double binsize, double min_sr, const float *sinc_vec,
                                    int n_sinc_samples, int sinc_ovs, double *output, int64_t nbins,
                                    void *stream) {
    if (npts < 0 || nbins < 0) return OCS_ERR_ARG;
    if (npts == 0 || nbins == 0) return OCS_OK;
    if (!srg || !scene || !sinc_vec || !output) return OCS_ERR_ARG;
    if (nbins > 0x3fffffff) return OCS_ERR_SIZE;
    return ocs::launch_chan_profile<double, 16>(srg, scene, 1, npts, binsize, min_sr, sinc_vec,
                                                n_sinc_samples, sinc_ovs, output, (int)nbins,
                                                (cudaStream_t)stream);
}

extern "C" int ocs_chan_profile_rows_f64(const double *srg, const double *scene, int64_t naz,
                                         int64_t npts, double binsize, double min_sr,
                                         const float *sinc_vec, int n_sinc_samples, int sinc_ovs,
                                         double *output, int64_t nbins, void *stream) {
    if (naz < 0 || npts < 0 || nbins < 0) return OCS_ERR_ARG;
    if (naz == 0 || npts == 0 || nbins == 0) return OCS_OK;
    if (!srg || !scene || !sinc_vec || !output) return OCS_ERR_ARG;
    if (nbins > 0x3fffffff) return OCS_ERR_SIZE;
    return ocs::launch_chan_profile<double, 16>(srg, scene, naz, npts, binsize, min_sr, sinc_vec,
                                                n_sinc_samples, sinc_ovs, output, (int)nbins,
                                                (cudaStream_t)stream);
}

extern "C" int ocs_chan_profile_c64(const double *srg, const float *scene, int64_t npts,
                                    double binsize, double min_sr, const float *sinc_vec,
                                    int n_sinc_samples, int sinc_ovs, float *output, int64_t nbins,
                                    void *stream) {
    if (npts < 0 || nbins < 0) return OCS_ERR_ARG;
    if (npts == 0 || nbins == 0) return OCS_OK;
    if (!srg || !scene || !sinc_vec || !output) return OCS_ERR_ARG;
    if (nbins > 0x3fffffff) return OCS_ERR_SIZE;
    return ocs::launch_chan_profile<float, 16>(srg, scene, 1, npts, binsize, min_sr, sinc_vec,
                                               n_sinc_samples, sinc_ovs, output, (int)nbins,
                                               (cudaStream_t)stream);
}

extern "C" int ocs_chan_profile_2d_f64(const double *srg, const double *scene, int64_t ny, int64_t nx,
                                       double binsize, double min_sr, const float *sinc_vec, int n_sinc_samples,
                                       int sinc_ovs, double *output, int64_t nbins, void *stream) {
    if (ny < 0 || nx < 0 || nbins < 0) return OCS_ERR_ARG;
    if (ny == 0 || nx == 0 || nbins == 0) return OCS_OK;
    if (!srg || !scene || !sinc_vec || !output) return OCS_ERR_ARG;
    if (nbins > 0x3fffffff) return OCS_ERR_SIZE;
    return ocs::launch_chan_profile_2d_any<double>(srg, scene, ny, nx, binsize, min_sr, sinc_vec, n_sinc_samples,
                                                   sinc_ovs, output, (int)nbins, (cudaStream_t)stream);
}

extern "C" int ocs_chan_profile_2d_c64(const double *srg, const float *scene, int64_t ny, int64_t nx,
                                       double binsize, double min_sr, const float *sinc_vec, int n_sinc_samples,
                                       int sinc_ovs, float *output, int64_t nbins, void *stream) {
    if (ny < 0 || nx < 0 || nbins < 0) return OCS_ERR_ARG;
    if (ny == 0 || nx == 0 || nbins == 0) return OCS_OK;
    if (!srg || !scene || !sinc_vec || !output) return OCS_ERR_ARG;
    if (nbins > 0x3fffffff) return OCS_ERR_SIZE;
    return ocs::launch_chan_profile_2d_any<float>(srg, scene, ny, nx, binsize, min_sr, sinc_vec, n_sinc_samples,
                                                  sinc_ovs, output, (int)nbins, (cudaStream_t)stream);
}

