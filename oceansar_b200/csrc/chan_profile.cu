// Standalone facet-to-range-bin accumulation: the drop-in for chan_profile_numba
// (oceansar/radarsim/range_profile.py:83-116 -> profile_integrator :22-49 and
// profile_integrator_1d :52-80).
//
// Facets come in arbitrary order (the caller's flattened slant-range / scene arrays), so
// each thread takes a run of consecutive facets -- consecutive facets of a flattened
// surface row are consecutive ground-range columns, whose bins grow monotonically -- and
// accumulates them through the register window of accum.cuh.  Output is accumulated in
// place (+=), never cleared, exactly like the reference.
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

template <typename T>
static int launch_chan_profile_2d_any(const double *srg, const void *scene, long long ny, long long nx,
                                      double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                      int nbins, cudaStream_t stream) {
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

