// SKIM two-scale Doppler: up-sampling of the step profiles and the geometric Doppler of
// each row group (the operation of upsample_and_dopplerize, oceansar/radarsim/skim_raw.py:
// 51-81), written as one band-limited interpolation per output sample instead of FFTs.
//
// The reference zero-pads the N-point azimuth spectrum of every row group to M = N n_up
// points (positive frequencies 0 .. ceil(N/2)-1 first, the others at the end) and
// transforms back, scaled by 1/N.  That is exactly the convolution of the N step samples
// with the M-periodic Dirichlet kernel
//     D(d) = (1/N) sum_{f = f0}^{f0 + N - 1} exp(2 pi i f d / M),  f0 = -floor(N/2),
//          = (1/N) sinpi(d / n_up) / sinpi(d / M) * (exp(-i pi d / M) if N is even),  D(0) = 1,
// evaluated at d = m - n n_up.  So, for output sample m and range bin r,
//     y[m][r] = sum_g exp(2 pi i dop[g][r] m / prf) * sum_n D(m - n n_up) x[n][g][r],
// all in float64 (the reference's spectra are complex64, its result complex128).
#include "common.cuh"

namespace ocs {

// D(d) for d in [0, M)
__global__ void dirichlet_kernel(double2 *D, int M, int N, int n_up) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= M) return;
    if (d == 0) {
        D[0] = make_double2(1.0, 0.0);
        return;
    }
    const double u = (double)d / (double)M;
    const double a = sinpi((double)d / (double)n_up) / (sinpi(u) * (double)N);
    if (N % 2 == 0) {
        double s, c;
        sincospi(-u, &s, &c);
        D[d] = make_double2(a * c, a * s);
    } else {
        D[d] = make_double2(a, 0.0);
    }
}

// One CTA per output sample m; the CTA's threads walk the range bins.
__global__ void skim_upsample_kernel(const double2 *__restrict__ x, const double *__restrict__ dop,
                                     const double2 *__restrict__ D, double2 *__restrict__ y, int N, int G, int R,
                                     int M, int n_up, double two_pi_over_prf) {
    extern __shared__ double2 dm[];                  // D(m - n n_up) for n = 0 .. N-1
    const int m = blockIdx.x;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        long long d = (long long)m - (long long)n * n_up;
        d %= M;
        if (d < 0) d += M;
        dm[n] = D[d];
    }
    __syncthreads();
    const double tm = two_pi_over_prf * (double)m;   // 2 pi t_m
    for (int r = threadIdx.x; r < R; r += blockDim.x) {
        double yr = 0.0, yi = 0.0;
        for (int g = 0; g < G; ++g) {
            double ar = 0.0, ai = 0.0;
            const double2 *xg = x + (long long)g * R + r;
            for (int n = 0; n < N; ++n) {
                const double2 v = xg[(long long)n * G * R];
                const double2 w = dm[n];
                ar = fma(w.x, v.x, fma(-w.y, v.y, ar));
                ai = fma(w.x, v.y, fma(w.y, v.x, ai));
            }
            double s, c;
            sincos(tm * dop[(long long)g * R + r], &s, &c);
            yr += ar * c - ai * s;
            yi += ar * s + ai * c;
        }
        y[(long long)m * R + r] = make_double2(yr, yi);
    }
}

}  // namespace ocs

using namespace ocs;

// x_d: complex128 [N][G][R] step profiles; dop_d: float64 [G][R] Doppler of each row group;
// y_d: complex128 [N * n_up][R]; D_d: complex128 [N * n_up] scratch (the kernel table).
extern "C" int ocs_skim_upsample(const double *x_d, const double *dop_d, double *y_d, double *D_d, int32_t N,
                                 int32_t G, int32_t R, int32_t n_up, double prf, void *stream) {
    if (!x_d || !dop_d || !y_d || !D_d || N < 1 || G < 1 || R < 1 || n_up < 1 || !(prf > 0.0)) return OCS_ERR_ARG;
    const long long M = (long long)N * n_up;
    if (M > (1 << 30) || (size_t)N * sizeof(double2) > 200 * 1024) return OCS_ERR_SIZE;
    cudaStream_t st = (cudaStream_t)stream;
    double2 *D = reinterpret_cast<double2 *>(D_d);
    dirichlet_kernel<<<(unsigned)((M + 255) / 256), 256, 0, st>>>(D, (int)M, N, n_up);
    if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    const size_t smem = (size_t)N * sizeof(double2);
    if (ensure_smem((const void *)skim_upsample_kernel, smem) != cudaSuccess) return OCS_ERR_CUDA;
    const int threads = R >= 256 ? 256 : ((R + 31) / 32) * 32;
    skim_upsample_kernel<<<(unsigned)M, threads, smem, st>>>(reinterpret_cast<const double2 *>(x_d), dop_d, D,
                                                             reinterpret_cast<double2 *>(y_d), N, G, R, (int)M,
                                                             n_up, 2.0 * 3.141592653589793 / prf);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}
