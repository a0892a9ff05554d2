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
#include "bulk.cuh"

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
// ground range), as sar_raw flattens them.  A CTA takes a tile of kC2Cols columns x
// kC2Rows rows; a thread owns one column and walks down the rows, so a warp reads 32
// consecutive facets of a row (coalesced) and every thread's range bin drifts only with
// the azimuth curvature and the surface displacement -- its register window almost never
// moves.  The inputs of each row are staged in shared memory two rows ahead with cp.async
// (each thread copies, and later reads, only its own words).
constexpr int kC2Cols = 128;
constexpr int kC2Rows = 64;
constexpr int kC2Stage = 3;
constexpr int kC2Nbw = 256;

template <typename T> OCS_HD constexpr size_t c2_stage_bytes() {
    return (size_t)kC2Stage * kC2Cols * (sizeof(double) + sizeof(cplx<T>));
}

template <typename T, int S>
__global__ void __launch_bounds__(kC2Cols, 4)
chan_profile_2d_kernel(const double *__restrict__ srg, const cplx<T> *__restrict__ scene, int ny, int nx,
                       double binsize, double min_sr, const float *__restrict__ sinc, int taps, int ovs,
                       T *__restrict__ out, int nbins) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *wtab = reinterpret_cast<T *>(smem_raw);
    const int wlen = wtab_len<T, S>(taps, ovs);
    T *acc = wtab + ((wlen + 3) & ~3);
    double *st_srg = reinterpret_cast<double *>(
        (reinterpret_cast<size_t>(acc + 2 * kC2Nbw) + 15) & ~(size_t)15);          // [kC2Stage][kC2Cols]
    cplx<T> *st_sc = reinterpret_cast<cplx<T> *>(st_srg + kC2Stage * kC2Cols);      // [kC2Stage][kC2Cols]

    const int tiles_x = (nx + kC2Cols - 1) / kC2Cols;
    const int x0 = (blockIdx.x % tiles_x) * kC2Cols;
    const int y0 = (blockIdx.x / tiles_x) * kC2Rows;
    const int x = x0 + threadIdx.x;
    const int nrows = min(kC2Rows, ny - y0);
    const double inv_binsize = 1.0 / binsize;

    build_wtab<T, S>(wtab, sinc, taps, ovs);
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
        const long long idx0 = (long long)y0 * nx + x;
        auto issue = [&](int r) {
            if (r < nrows) {
                const long long g = idx0 + (long long)r * nx;
                const int slot = (r % kC2Stage) * kC2Cols + threadIdx.x;
                const unsigned d0 = (unsigned)__cvta_generic_to_shared(st_srg + slot);
                const unsigned d1 = (unsigned)__cvta_generic_to_shared(st_sc + slot);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d0), "l"(srg + g) : "memory");
                if (sizeof(cplx<T>) == 8)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d1), "l"(scene + g) : "memory");
                else
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d1), "l"(scene + g) : "memory");
            }
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        };
        for (int r = 0; r < kC2Stage - 1; ++r) issue(r);
        const int half = taps / 2;
        for (int i = 0; i < nrows; ++i) {
            issue(i + kC2Stage - 1);
            asm volatile("cp.async.wait_group %0;\n" ::"n"(kC2Stage - 1) : "memory");
            const int slot = (i % kC2Stage) * kC2Cols + threadIdx.x;
            int bin_d, lut;
            // FP64: IEEE division, bin / LUT bit-identical with numpy; single precision:
            // reciprocal multiply (a one-ulp difference in the bin coordinate)
            if (sizeof(T) == 8) bin_and_lut(st_srg[slot], min_sr, binsize, ovs, bin_d, lut);
            else bin_and_lut_fast(st_srg[slot], min_sr, inv_binsize, ovs, bin_d, lut);
            if (bin_d < -(1 << 29)) continue;
            cplx<T> c[1] = {st_sc[slot]};
            win.add(bin_d - half, lut, c, wtab, sinc, taps, ovs, cb);
        }
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    }
    win.flush(cb);
    __syncthreads();
    cb.flush_to_global();
}

template <typename T, int S>
static int launch_chan_profile_2d(const double *srg, const void *scene, long long ny, long long nx, double binsize,
                                  double min_sr, const float *sinc, int taps, int ovs, T *out, int nbins,
                                  cudaStream_t stream) {
    if (taps < 1 || taps > S || ovs < 1 || ny < 0 || nx < 0 || nbins < 0) return OCS_ERR_ARG;
    if (ny == 0 || nx == 0 || nbins == 0) return OCS_OK;
    if (ny > 0x7fffffffLL || nx > 0x7fffffffLL) return OCS_ERR_SIZE;
    const int wlen = wtab_len<T, S>(taps, ovs);
    const size_t smem = (size_t)((wlen + 3) & ~3) * sizeof(T) + (size_t)kC2Nbw * 2 * sizeof(T) + 16 +
                        c2_stage_bytes<T>();
    const long long grid = ((nx + kC2Cols - 1) / kC2Cols) * ((ny + kC2Rows - 1) / kC2Rows);
    if (grid > 0x7fffffffLL) return OCS_ERR_SIZE;
    auto kern = chan_profile_2d_kernel<T, S>;
    if (ensure_smem((const void *)kern, smem) != cudaSuccess) return OCS_ERR_CUDA;
    kern<<<(unsigned)grid, kC2Cols, smem, stream>>>(srg, reinterpret_cast<const cplx<T> *>(scene), (int)ny, (int)nx,
                                                      binsize, min_sr, sinc, taps, ovs, out, nbins);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// Bulk-staged form of the two-dimensional accumulation (the default when nx is even and the
// inputs are 16-byte aligned).  Persistent CTAs walk tiles of kC2Cols columns x tile_rows
// rows; each warp moves its 32 columns' slant ranges and scene values of a row into a
// four-row shared-memory ring with two one-dimensional bulk copies (cp.async.bulk, issued by
// lane 0, completing on the slot's mbarrier), so the per-facet work is two shared loads,
// the bin / LUT index and the register-window update.  Waits are bounded: a wait that
// gives up sets g_chan_profile_err (read by ocs_chan_profile_status), lets the warp's
// copies in flight land and ends the warp's work.
constexpr int kB2Slots = 4;
__device__ int g_chan_profile_err = 0;

template <typename T> OCS_HD constexpr size_t b2_slot_bytes() { return 32 * (sizeof(double) + sizeof(cplx<T>)); }

template <typename T, int S> OCS_HD size_t b2_smem_bytes(int taps, int ovs) {
    return (size_t)((wtab_len<T, S>(taps, ovs) + 3) & ~3) * sizeof(T) + (size_t)kC2Nbw * 2 * sizeof(T) + 128 +
           (size_t)4 * kB2Slots * b2_slot_bytes<T>() + 4 * kB2Slots * 8;
}

template <typename T, int S>
__global__ void __launch_bounds__(kC2Cols, 4)
chan_profile_2d_bulk_kernel(const double *__restrict__ srg, const cplx<T> *__restrict__ scene, int ny, int nx,
                            double binsize, double min_sr, const float *__restrict__ sinc, int taps, int ovs,
                            T *__restrict__ out, int nbins, int tile_rows) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(smem_raw);            // [4][kB2Slots]
    unsigned char *stage = smem_raw + 128;                                                   // [4][kB2Slots] slots
    T *wtab = reinterpret_cast<T *>(stage + 4 * kB2Slots * b2_slot_bytes<T>());
    const int wlen = wtab_len<T, S>(taps, ovs);
    T *acc = wtab + ((wlen + 3) & ~3);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    build_wtab<T, S>(wtab, sinc, taps, ovs);
    if (lane == 0)
        for (int k = 0; k < kB2Slots; ++k) mbar_init(bars + warp * kB2Slots + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    __syncthreads();

    const int tiles_x = (nx + kC2Cols - 1) / kC2Cols;
    const int tiles = tiles_x * ((ny + tile_rows - 1) / tile_rows);
    const double inv_binsize = 1.0 / binsize;
    const int half = taps / 2;
    unsigned rseq = 0;
    bool bad = false;
    unsigned char *wst = stage + (size_t)warp * kB2Slots * b2_slot_bytes<T>();
    unsigned long long *wbar = bars + warp * kB2Slots;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int x0 = (tile % tiles_x) * kC2Cols;
        const int y0 = (tile / tiles_x) * tile_rows;
        const int nrows = min(tile_rows, ny - y0);
        __syncthreads();                  // the previous tile's bins are flushed
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
        const int xw = x0 + 32 * warp;
        if (xw < nx && !bad) {
            const int ncw = min(32, nx - xw);
            const bool col_ok = xw + lane < nx;
            const unsigned first = rseq;
            unsigned issued = 0, waited = 0;
            auto issue = [&](int r) {
                if (lane == 0 && r < nrows) {
                    const unsigned q = first + (unsigned)r;
                    unsigned char *dst = wst + (size_t)(q % kB2Slots) * b2_slot_bytes<T>();
                    unsigned long long *bar = wbar + (q % kB2Slots);
                    const long long g = (long long)(y0 + r) * nx + xw;
                    fence_proxy_async();
                    mbar_expect_tx(bar, (unsigned)ncw * (unsigned)(sizeof(double) + sizeof(cplx<T>)));
                    bulk_g2s(dst, srg + g, (unsigned)ncw * 8u, bar);
                    bulk_g2s(dst + 32 * sizeof(double), scene + g, (unsigned)ncw * (unsigned)sizeof(cplx<T>), bar);
                    issued = (unsigned)r + 1;
                }
            };
            auto wait_row = [&](int r) -> bool {
                const unsigned q = first + (unsigned)r;
                return mbar_wait(wbar + (q % kB2Slots), (q / kB2Slots) & 1u);
            };
            issue(0);
            issue(1);
            issue(2);
            bool ok = true;
            for (int i = 0; i < nrows; ++i) {
                ok = __all_sync(0xffffffffu, wait_row(i));
                if (!ok) break;
                waited = (unsigned)i + 1;
                const unsigned char *src = wst + (size_t)((first + (unsigned)i) % kB2Slots) * b2_slot_bytes<T>();
                const double sr = reinterpret_cast<const double *>(src)[lane];
                const cplx<T> c = reinterpret_cast<const cplx<T> *>(src + 32 * sizeof(double))[lane];
                __syncwarp();
                issue(i + 3);             // into the slot of row i - 1
                if (!col_ok) continue;
                int bin_d, lut;
                // FP64: IEEE division, bin / LUT bit-identical with numpy; single precision:
                // reciprocal multiply (a one-ulp difference in the bin coordinate)
                if (sizeof(T) == 8) bin_and_lut(sr, min_sr, binsize, ovs, bin_d, lut);
                else bin_and_lut_fast(sr, min_sr, inv_binsize, ovs, bin_d, lut);
                if (bin_d < -(1 << 29)) continue;
                cplx<T> cc[1] = {c};
                win.add(bin_d - half, lut, cc, wtab, sinc, taps, ovs, cb);
            }
            if (!ok) {
                bad = true;
                if (lane == 0) {
                    atomicOr(&g_chan_profile_err, 1);
                    for (unsigned r = waited; r < issued; ++r) wait_row((int)r);
                }
                __syncwarp();
            }
            rseq = first + (unsigned)nrows;
        }
        win.flush(cb);
        __syncthreads();
        cb.flush_to_global();
    }
}

template <typename T, int S>
static int launch_chan_profile_2d_bulk(const double *srg, const void *scene, long long ny, long long nx,
                                       double binsize, double min_sr, const float *sinc, int taps, int ovs, T *out,
                                       int nbins, cudaStream_t stream) {
    if (taps < 1 || taps > S || ovs < 1) return OCS_ERR_ARG;
    if (ny > 0x7fffffffLL || nx > 0x7fffffffLL) return OCS_ERR_SIZE;
    const size_t smem = b2_smem_bytes<T, S>(taps, ovs);
    auto kern = chan_profile_2d_bulk_kernel<T, S>;
    if (ensure_smem((const void *)kern, smem) != cudaSuccess) return OCS_ERR_CUDA;
    const int resident = resident_ctas((const void *)kern, kC2Cols, smem);
    if (resident <= 0) return OCS_ERR_CUDA;
    // tile height: the tallest (<= kC2Rows) that fills the last wave of resident CTAs
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
    const bool bulk_ok = nx % 2 == 0 && ((((uintptr_t)srg) | ((uintptr_t)scene)) & 15) == 0;
    if (bulk_ok && taps <= 8)
        return launch_chan_profile_2d_bulk<T, 12>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                                  stream);
    if (taps <= 8)
        return launch_chan_profile_2d<T, 12>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins,
                                             stream);
    return launch_chan_profile_2d<T, 16>(srg, scene, ny, nx, binsize, min_sr, sinc, taps, ovs, out, nbins, stream);
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

extern "C" int ocs_chan_profile_status(void) {
    int flag = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&flag, ocs::g_chan_profile_err, sizeof(int)) != cudaSuccess) return OCS_ERR_CUDA;
    if (flag && cudaMemcpyToSymbol(ocs::g_chan_profile_err, &zero, sizeof(int)) != cudaSuccess) return OCS_ERR_CUDA;
    return flag ? OCS_ERR_TIMEOUT : OCS_OK;
}
