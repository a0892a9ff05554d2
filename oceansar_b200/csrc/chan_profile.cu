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
