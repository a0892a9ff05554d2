// Range-Doppler focusing (oceansar/radarsim/sar_processor.py:30-274): the two phase
// multiplications between the FFTs, fused and evaluated on the fly (no phase screens in
// memory).  The FFTs themselves are plain library transforms.
//
//   RCMC (:170-176):  D[p][a][r] *= exp(1j ((4 pi rcmc[a]) / c) fr[r])    (range-frequency ramp)
//   azimuth filter (:213-217):  D[p][a][r] *= h[a]                        (complex per azimuth)
//
// complex128 data [npol][naz][nrg]; the phase is formed in float64 in numpy's order and
// the products use numpy's complex multiplication.
#include "common.cuh"

namespace ocs {

__global__ void rd_rcmc_kernel(double2 *data, long long npol, int naz, int nrg, const double *rcmc,
                               const double *fr, double c) {
    const long long n = npol * naz * (long long)nrg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i % nrg);
        const int a = (int)((i / nrg) % naz);
        const double th = dmul(ddiv(dmul(4.0 * 3.141592653589793, rcmc[a]), c), fr[r]);
        double s, co;
        sincos(th, &s, &co);
        const double2 v = data[i];
        data[i] = make_double2(dsub(dmul(v.x, co), dmul(v.y, s)), dadd(dmul(v.x, s), dmul(v.y, co)));
    }
}

__global__ void rd_azfilter_kernel(double2 *data, long long npol, int naz, int nrg, const double2 *h) {
    const long long n = npol * naz * (long long)nrg;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int a = (int)((i / nrg) % naz);
        const double2 v = data[i], w = h[a];
        data[i] = make_double2(dsub(dmul(v.x, w.x), dmul(v.y, w.y)), dadd(dmul(v.x, w.y), dmul(v.y, w.x)));
    }
}

static unsigned rd_grid(long long n) {
    long long b = (n + 255) / 256;
    return (unsigned)(b > 148 * 32 ? 148 * 32 : (b < 1 ? 1 : b));
}

}  // namespace ocs

using namespace ocs;

extern "C" int ocs_rd_rcmc(double *data_d, int64_t npol, int32_t naz, int32_t nrg, const double *rcmc_d,
                           const double *fr_d, double c, void *stream) {
    if (!data_d || !rcmc_d || !fr_d || npol < 0 || naz < 0 || nrg < 0) return OCS_ERR_ARG;
    const long long n = npol * naz * (long long)nrg;
    if (n == 0) return OCS_OK;
    rd_rcmc_kernel<<<rd_grid(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double2 *>(data_d), npol, naz,
                                                                  nrg, rcmc_d, fr_d, c);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

extern "C" int ocs_rd_azfilter(double *data_d, int64_t npol, int32_t naz, int32_t nrg, const double *h_d,
                               void *stream) {
    if (!data_d || !h_d || npol < 0 || naz < 0 || nrg < 0) return OCS_ERR_ARG;
    const long long n = npol * naz * (long long)nrg;
    if (n == 0) return OCS_OK;
    rd_azfilter_kernel<<<rd_grid(n), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<double2 *>(data_d), npol, naz,
                                                                      nrg, reinterpret_cast<const double2 *>(h_d));
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}
