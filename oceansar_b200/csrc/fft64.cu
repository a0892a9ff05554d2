// Complex128 power-of-two FFTs of the SAR processor (the 2-D transforms of sar_focus,
// oceansar/radarsim/sar_processor.py:170, 176, 217, where optimize_fftsize pads both
// dimensions to powers of two).
//
// * Rows of length n <= 8192 (kFft64Smem): one CTA per row, the row and a table of the n/2
//   twiddles in shared memory; iterative decimation in time after a bit-reversed load,
//   three radix-2 levels per pass held in registers (a thread owns whole groups of 8
//   elements, so a pass reads and writes only its own elements and one barrier separates
//   passes).
// * Longer rows, n = n1 n2: the four-step decomposition through global memory: each row
//   viewed as [n1][n2] is transposed, its n2 columns transformed (length n1), multiplied
//   by W_n^(n2 k1), transposed back, its n1 rows transformed (length n2), and transposed
//   once more into natural order.
// * Transforms along a strided dimension (the azimuth of a [pol][az][rg] cube) go through
//   a tiled transpose (ocs_transpose_c128).
// Forward: exp(-2 pi i k n / N); inverse: exp(+2 pi i k n / N) and 1/N, as numpy.fft.
#include "common.cuh"

namespace ocs {

constexpr int kFft64Smem = 8192;

OCS_D double2 z_mul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// In-place transform of one row of length n = 2^logn in shared memory.
__global__ void __launch_bounds__(1024, 1)
fft64_rows_kernel(double2 *__restrict__ data, int n, int logn, int inverse, double scale) {
    extern __shared__ __align__(16) double2 fsm[];
    double2 *buf = fsm, *tw = fsm + n;
    double2 *x = data + (long long)blockIdx.x * n;
    const int T = blockDim.x;
    // twiddles exp(-+2 pi i k / n), k < n/2 (2k/n is exact for a power-of-two n): the first
    // octant from sincospi, the rest by the exact symmetries of cos and sin about pi/4,
    // pi/2 and pi (n >= 8)
    const double sg = inverse ? 1.0 : -1.0;
    if (n < 8) {
        for (int k = threadIdx.x; k < n / 2; k += T) {
            double s, c;
            sincospi(2.0 * (double)k / (double)n, &s, &c);
            tw[k] = make_double2(c, sg * s);
        }
    } else {
        const int q = n / 4;
        for (int k = threadIdx.x; k <= n / 8; k += T) {
            double s, c;
            sincospi(2.0 * (double)k / (double)n, &s, &c);
            tw[k] = make_double2(c, sg * s);                  // theta
            tw[q - k] = make_double2(s, sg * c);              // pi/2 - theta
            if (k > 0) tw[q + k] = make_double2(-s, sg * c);                 // pi/2 + theta
            if (k > 0 && 8 * k < n) tw[2 * q - k] = make_double2(-c, sg * s);  // pi - theta
        }
    }
    for (int j = threadIdx.x; j < n; j += T) buf[__brev((unsigned)j) >> (32 - logn)] = x[j];
    __syncthreads();
    for (int s = 1, done = 0; done < logn;) {
        const int levels = min(3, logn - done);
        const int r = 1 << levels;
        for (int g = threadIdx.x; g < n / r; g += T) {
            const int j = g & (s - 1);
            const int base = (g >> done) * r * s + j;     // g / s with s = 2^done
            double2 v[8];
#pragma unroll
            for (int m = 0; m < 8; ++m)
                if (m < r) v[m] = buf[base + m * s];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                if (q < levels) {
                    const int h = 1 << q;
                    // twiddle index (j + (m mod h) s) n / (2 s h)
                    const int step = n >> (done + q + 1);
#pragma unroll
                    for (int m = 0; m < 8; ++m) {
                        if (m < r && (m & h) == 0) {
                            const double2 w = tw[(j + (m & (h - 1)) * s) * step];
                            const double2 b = z_mul(v[m + h], w);
                            const double2 a = v[m];
                            v[m] = make_double2(a.x + b.x, a.y + b.y);
                            v[m + h] = make_double2(a.x - b.x, a.y - b.y);
                        }
                    }
                }
            }
#pragma unroll
            for (int m = 0; m < 8; ++m)
                if (m < r) buf[base + m * s] = v[m];
        }
        __syncthreads();
        s <<= levels;
        done += levels;
    }
    for (int j = threadIdx.x; j < n; j += T) {
        const double2 v = buf[j];
        x[j] = make_double2(v.x * scale, v.y * scale);
    }
}

// dst[b][c][r] = src[b][r][c] for a batch of rows x cols complex128 matrices.
__global__ void transpose_c128_kernel(const double2 *__restrict__ src, double2 *__restrict__ dst, int rows, int cols) {
    __shared__ double2 tile[32][33];
    const long long b = blockIdx.z;
    const double2 *s = src + b * rows * cols;
    double2 *d = dst + b * rows * cols;
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int r = r0 + i, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[i][threadIdx.x] = s[(long long)r * cols + c];
    }
    __syncthreads();
    for (int i = threadIdx.y; i < 32; i += blockDim.y) {
        const int c = c0 + i, r = r0 + threadIdx.x;
        if (r < rows && c < cols) d[(long long)c * rows + r] = tile[threadIdx.x][i];
    }
}

// Four-step twiddle: a[b][i2][k1] *= exp(-+2 pi i (i2 k1 mod n) / n) on [batch][n2][n1].
__global__ void fft64_twiddle_kernel(double2 *a, long long total, int n1, int n2, int inverse) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const long long n = (long long)n1 * n2;
    const int k1 = (int)(i % n1);
    const int i2 = (int)((i / n1) % n2);
    const long long e = ((long long)i2 * k1) % n;
    double s, c;
    sincospi(2.0 * (double)e / (double)n, &s, &c);
    a[i] = z_mul(a[i], make_double2(c, inverse ? s : -s));
}

static int ilog2_exact(long long n) {
    if (n < 1 || (n & (n - 1))) return -1;
    int l = 0;
    while ((1LL << l) < n) ++l;
    return l;
}

static int launch_rows_smem(double2 *d, long long nrows, int n, bool inverse, double scale, cudaStream_t st) {
    const int logn = ilog2_exact(n);
    if (n == 1) {
        if (scale != 1.0) return OCS_ERR_UNSUPPORTED;
        return OCS_OK;
    }
    const size_t smem = (size_t)(n + n / 2) * sizeof(double2);
    if (ensure_smem((const void *)fft64_rows_kernel, smem) != cudaSuccess) return OCS_ERR_CUDA;
    int threads = n / 8;
    threads = threads < 32 ? 32 : (threads > 1024 ? 1024 : threads);
    for (long long r0 = 0; r0 < nrows; r0 += 0x7fffffffLL) {
        const long long nr = nrows - r0 < 0x7fffffffLL ? nrows - r0 : 0x7fffffffLL;
        fft64_rows_kernel<<<(unsigned)nr, threads, smem, st>>>(d + r0 * n, n, logn, inverse ? 1 : 0, scale);
        if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    }
    return OCS_OK;
}

static int launch_transpose(const double2 *s, double2 *d, long long batch, long long rows, long long cols,
                            cudaStream_t st) {
    if (rows > 0x7fffffffLL || cols > 0x7fffffffLL || (rows + 31) / 32 > 65535) return OCS_ERR_SIZE;
    for (long long b0 = 0; b0 < batch; b0 += 65535) {       // grid z is at most 65535
        const long long nb = batch - b0 < 65535 ? batch - b0 : 65535;
        dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32), (unsigned)nb);
        transpose_c128_kernel<<<grid, dim3(32, 8), 0, st>>>(s + b0 * rows * cols, d + b0 * rows * cols, (int)rows,
                                                            (int)cols);
        if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    }
    return OCS_OK;
}

}  // namespace ocs

using namespace ocs;

// Bytes of scratch ocs_fft64_rows needs: 0 for n <= 8192, else nrows * n complex128.
extern "C" int64_t ocs_fft64_workspace_bytes(int64_t nrows, int64_t n) {
    if (nrows < 0 || ilog2_exact(n) < 0) return -1;
    return n <= kFft64Smem ? 0 : nrows * n * (int64_t)sizeof(double2);
}

// In-place FFT of nrows contiguous complex128 rows of length n (a power of two), forward
// (inverse = 0) or inverse (inverse = 1, scaled by 1/n).  scratch: ocs_fft64_workspace_bytes.
extern "C" int ocs_fft64_rows(double *data, int64_t nrows, int64_t n, int32_t inverse, double *scratch,
                              void *stream) {
    if (nrows < 0 || (nrows > 0 && !data) || ilog2_exact(n) < 0) return OCS_ERR_ARG;
    if (nrows == 0) return OCS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    double2 *d = reinterpret_cast<double2 *>(data);
    if (n <= kFft64Smem) return launch_rows_smem(d, nrows, (int)n, inverse != 0, inverse ? 1.0 / (double)n : 1.0, st);
    if (!scratch) return OCS_ERR_ARG;
    const int logn = ilog2_exact(n);
    const long long n1 = 1LL << (logn / 2 + (logn & 1)), n2 = n / n1;   // n1 >= n2, both <= 8192 up to 2^26
    if (n1 > kFft64Smem) return OCS_ERR_SIZE;
    double2 *w = reinterpret_cast<double2 *>(scratch);
    int s;
    // [rows][n1][n2] -> [rows][n2][n1]; n2 transforms of length n1 per row
    if ((s = launch_transpose(d, w, nrows, n1, n2, st)) != OCS_OK) return s;
    if ((s = launch_rows_smem(w, nrows * n2, (int)n1, inverse != 0, inverse ? 1.0 / (double)n1 : 1.0, st)) != OCS_OK)
        return s;
    const long long total = nrows * n;
    fft64_twiddle_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(w, total, (int)n1, (int)n2, inverse != 0);
    if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    // [rows][n2][n1] -> [rows][n1][n2]; n1 transforms of length n2 per row: [k1][k2]
    if ((s = launch_transpose(w, d, nrows, n2, n1, st)) != OCS_OK) return s;
    if ((s = launch_rows_smem(d, nrows * n1, (int)n2, inverse != 0, inverse ? 1.0 / (double)n2 : 1.0, st)) != OCS_OK)
        return s;
    // X[k1 + n1 k2] at [k1][k2] -> natural order [k2][k1]
    if ((s = launch_transpose(d, w, nrows, n1, n2, st)) != OCS_OK) return s;
    return cudaMemcpyAsync(d, w, (size_t)total * sizeof(double2), cudaMemcpyDeviceToDevice, st) == cudaSuccess
               ? OCS_OK
               : OCS_ERR_CUDA;
}

// dst[b][c][r] = src[b][r][c] for batch complex128 matrices of rows x cols (src != dst).
extern "C" int ocs_transpose_c128(const double *src, double *dst, int64_t batch, int64_t rows, int64_t cols,
                                  void *stream) {
    if (batch < 0 || rows < 0 || cols < 0 || !src || !dst || src == dst) return OCS_ERR_ARG;
    if (batch == 0 || rows == 0 || cols == 0) return OCS_OK;
    return launch_transpose(reinterpret_cast<const double2 *>(src), reinterpret_cast<double2 *>(dst), batch, rows,
                            cols, (cudaStream_t)stream);
}
