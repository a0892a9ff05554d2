// Per-pulse linear-wave surface synthesis: the OceanSurface.t setter
// (oceansar/surfaces/ocean.py:418-526) on sm_100a.
//
// Every field the reference computes is Re(ifft2(M_f(k) * c(t))) (+ a constant / swell
// term), with c(t) = wave_coefs * exp(-i omega t) (ocean.py:427) and M_f a per-field
// spectral multiplier (i kx for Diffx, -kx^2 for Diffxx, i kx/|k| for Dx, ...).  Two real
// fields A, B are packed into ONE complex transform:
//     Z = H(M_A c) + i H(M_B c),  H(X)[k] = (X[k] + conj(X[-k])) / 2,
// so ifft2(Z) = A + iB exactly (H(X) is the Hermitian part whose inverse DFT is Re(ifft2 X)).
// The 2-D inverse DFT runs as two shared-memory passes:
//   pass 1 (rows, x): one CTA per row pair (r, Ny-r).  The phase evolution, multipliers
//          and Hermitian packing are computed on the fly from c and omega (read once per
//          pulse), then each packed row is transformed and written to a scratch plane.
//   pass 2 (columns, y): one CTA per (transform, W-column tile); column transforms, then
//          the 1/(Nx Ny) scale, the additive terms and the unpacking into two float32
//          fields.
// A third, element-wise kernel applies the choppy-wave combinations (ocean.py:451-482).
#include <math.h>
#include <string.h>

#include "batch.cuh"
#include "fft.cuh"

namespace ocs {

constexpr int kMaxPacked = 12;          // transforms per call (24 real fields)

struct MultDesc {
    signed char imag, sign, a, b, c, d, hmtf, pad;
};

struct SurfaceArgs {
    int nx, ny;
    const float2 *coefs;
    const float *omega;
    const float *kx;
    const float *ky;
    float kmin_half;
    float t;
    float inv_n;
    int npair;
    int prog;                         // field program of the row pass (surface_rows_kernel)
    int needs_omega;                  // some field's multiplier involves omega
    int code[2 * kMaxPacked];
    MultDesc mult[2 * kMaxPacked];
    float *dst[2 * kMaxPacked];
    float add[2 * kMaxPacked];
    float2 swm[2 * kMaxPacked];
    const float2 *swell_exp;
    float2 swell_rot;
    float2 *scratch;
    FftPlan px, py;
    const float2 *stw_x, *stw_y;      // stage-major twiddles (power-of-two lengths)
};

// Spectral multiplier M of every field (ocean.py:431-526): Re(ifft2(M c)) is the field.
// Except for the hydrodynamic MTF, M = sign * kx^a * ky^b * kinv^c * omega^d, purely real
// or purely imaginary; MultDesc holds that recipe so the device evaluates it with uniform
// loops (kinv = 1/|k| where |k| > min(kx_res, ky_res)/2, else 0; ocean.py:141-148).
static MultDesc mult_desc(int code) {
    //                                     imag sign a  b  c  d  hmtf
    switch (code) {
        case OCS_FIELD_DZ: return {0, 1, 0, 0, 0, 0, 0, 0};
        case OCS_FIELD_DX: return {1, 1, 1, 0, 1, 0, 0, 0};       // -Im(ifft2(kxn c))
        case OCS_FIELD_DY: return {1, 1, 0, 1, 1, 0, 0, 0};
        case OCS_FIELD_DIFFX: return {1, 1, 1, 0, 0, 0, 0, 0};    // Re(ifft2(i kx c))
        case OCS_FIELD_DIFFY: return {1, 1, 0, 1, 0, 0, 0, 0};
        case OCS_FIELD_DIFFXX: return {0, -1, 2, 0, 0, 0, 0, 0};
        case OCS_FIELD_DIFFYY: return {0, -1, 0, 2, 0, 0, 0, 0};
        case OCS_FIELD_DIFFXY: return {0, -1, 1, 1, 0, 0, 0, 0};
        case OCS_FIELD_VX: return {0, 1, 1, 0, 1, 1, 0, 0};       // -Im(ifft2(kxn (-i w) c))
        case OCS_FIELD_VY: return {0, 1, 0, 1, 1, 1, 0, 0};
        case OCS_FIELD_VZ: return {1, -1, 0, 0, 0, 1, 0, 0};
        case OCS_FIELD_AX: return {1, -1, 1, 0, 1, 2, 0, 0};
        case OCS_FIELD_AY: return {1, -1, 0, 1, 1, 2, 0, 0};
        case OCS_FIELD_AZ: return {0, -1, 0, 0, 0, 2, 0, 0};
        case OCS_FIELD_HMTF: return {0, 1, 0, 0, 0, 0, 1, 0};
        case OCS_FIELD_AUX_XX: return {0, -1, 2, 0, 1, 0, 0, 0};
        case OCS_FIELD_AUX_YY: return {0, -1, 0, 2, 1, 0, 0, 0};
        case OCS_FIELD_AUX_XXX: return {1, -1, 3, 0, 1, 0, 0, 0};
        case OCS_FIELD_AUX_YYY: return {1, -1, 0, 3, 1, 0, 0, 0};
        case OCS_FIELD_AUX_XXY: return {1, -1, 2, 1, 1, 0, 0, 0};
        default: return {0, 0, 0, 0, 0, 0, 0, 0};
    }
}

OCS_D float2 field_mult(const MultDesc &m, float kxv, float kyv, float k, float kinv, float om) {
    if (m.hmtf) {
        // M_h = i k w (w + i mu) / (w^2 + mu^2) * (dlnS/dlnk - Vg/c), zero for k > 2 pi/20
        const float kmax = 0.3141592653589793f, mu = 0.0025f, fac = -3.5f;
        if (k > kmax) return make_float2(0.f, 0.f);
        const float den = om * om + mu * mu;
        return make_float2(-k * om * mu / den * fac, k * om * om / den * fac);
    }
    float v = (float)m.sign;
    for (int i = 0; i < m.a; ++i) v *= kxv;
    for (int i = 0; i < m.b; ++i) v *= kyv;
    if (m.c) v *= kinv;
    for (int i = 0; i < m.d; ++i) v *= om;
    return m.imag ? make_float2(0.f, v) : make_float2(v, 0.f);
}

// c(t) = c * exp(-i fl(omega t)) in complex64 (ocean.py:424-427).
OCS_D float2 phased(const SurfaceArgs &a, int y, int x) {
    size_t i = (size_t)y * a.nx + x;
    float2 c = a.coefs[i];
    float ph = -fmul(a.omega[i], a.t);
    float s, co;
    sincosf(ph, &s, &co);
    return make_float2(fsub(fmul(c.x, co), fmul(c.y, s)), fadd(fmul(c.x, s), fmul(c.y, co)));
}

// c exp(-i fl(omega t)) from values already loaded (the same arithmetic as phased).
OCS_D float2 phased_v(float2 c, float om, float t) {
    float ph = -fmul(om, t);
    float s, co;
    sincosf(ph, &s, &co);
    return make_float2(fsub(fmul(c.x, co), fmul(c.y, s)), fadd(fmul(c.x, s), fmul(c.y, co)));
}

// Threads per CTA of the two passes for a power-of-two length N (0 = any length).
template <int N> __host__ __device__ constexpr int rows_threads() {
    return N == 0 ? 256 : (N / 4 < 64 ? 64 : (N / 4 > 1024 ? 1024 : N / 4));
}
template <int N, int TILE> __host__ __device__ constexpr int cols_threads() {
    return N == 0 ? 256 : (N * TILE / 16 < 64 ? 64 : (N * TILE / 16 > 1024 ? 1024 : N * TILE / 16));
}

// Output of the row transforms: vector 0 is row r, vector 1 row mr of one scratch plane.
struct RowStore {
    float2 *plane;
    int nx, r, mr;
    OCS_D void operator()(int vec, int x, float2 v) const {
        if (vec == 1 && mr == r) return;
        plane[(size_t)(vec ? mr : r) * nx + x] = v;
    }
};

// Input of the column transforms: TILE consecutive columns of one scratch plane.
struct ColLoad {
    const float2 *plane;
    int nx, x0;
    OCS_D float2 operator()(int w, int y) const {
        const int x = x0 + w;
        return x < nx ? plane[(size_t)y * nx + x] : make_float2(0.f, 0.f);
    }
};

// Output of the column transforms: scale, additive terms, swell, two float32 fields.
struct ColStore {
    float *dA, *dB;
    const float2 *swell_exp;
    float2 swell_rot, smA, smB;
    float inv_n, addA, addB;
    int nx, x0;
    OCS_D void operator()(int w, int y, float2 z) const {
        const int x = x0 + w;
        if (x >= nx) return;
        float va = fadd(z.x * inv_n, addA);
        float vb = fadd(z.y * inv_n, addB);
        if (swell_exp) {
            const float2 s = c_mul(swell_exp[(size_t)y * nx + x], swell_rot);
            va = fadd(va, fsub(fmul(smA.x, s.x), fmul(smA.y, s.y)));
            vb = fadd(vb, fsub(fmul(smB.x, s.x), fmul(smB.y, s.y)));
        }
        dA[(size_t)y * nx + x] = va;
        if (dB) dB[(size_t)y * nx + x] = vb;
    }
};

// Compile-time field programs of the row pass.  Program 1 is the field set of sar_raw
// with the specular model (Dx Dy | Dz Diffx | Diffy Diffxx | Diffyy Diffxy), program 2
// the one without it (Dx Dy | Dz Diffx | Diffy -); any other list runs program 0, which
// evaluates the MultDesc recipes at run time.
constexpr int kNone = -2;       // no second field in the pair
constexpr int kRuntime = -1;    // recipe read from SurfaceArgs::mult

template <int CODE> __host__ __device__ constexpr bool needs_kinv() {
    return CODE == kRuntime || CODE == OCS_FIELD_DX || CODE == OCS_FIELD_DY || CODE == OCS_FIELD_VX ||
           CODE == OCS_FIELD_VY || CODE == OCS_FIELD_AX || CODE == OCS_FIELD_AY || CODE == OCS_FIELD_HMTF ||
           CODE >= OCS_FIELD_AUX_XX;
}

// Multiplier of a compile-time field code (kRuntime: the run-time recipe m).
template <int CODE>
OCS_D float2 mult_ct(const MultDesc &m, float kx, float ky, float k, float kinv, float om) {
    if constexpr (CODE == kRuntime) return field_mult(m, kx, ky, k, kinv, om);
    else if constexpr (CODE == OCS_FIELD_DZ) return make_float2(1.f, 0.f);
    else if constexpr (CODE == OCS_FIELD_DX) return make_float2(0.f, kx * kinv);
    else if constexpr (CODE == OCS_FIELD_DY) return make_float2(0.f, ky * kinv);
    else if constexpr (CODE == OCS_FIELD_DIFFX) return make_float2(0.f, kx);
    else if constexpr (CODE == OCS_FIELD_DIFFY) return make_float2(0.f, ky);
    else if constexpr (CODE == OCS_FIELD_DIFFXX) return make_float2(-(kx * kx), 0.f);
    else if constexpr (CODE == OCS_FIELD_DIFFYY) return make_float2(-(ky * ky), 0.f);
    else if constexpr (CODE == OCS_FIELD_DIFFXY) return make_float2(-(kx * ky), 0.f);
    else return field_mult(m, kx, ky, k, kinv, om);
}

// Packed spectra of transform p at the two mirror pairs of column x (pass 1):
// (r, x) <-> (mr, nx-x) and (r, nx-x) <-> (mr, x).
template <int CA, int CB>
OCS_D void build_packed(const SurfaceArgs &a, int p, int x, int nx, float kyr, float kymr, const float2 *cA,
                        const float2 *cB, const float *omA, const float *omB, float2 *rowA, float2 *rowB) {
    const MultDesc ma = a.mult[2 * p], mb = a.mult[2 * p + 1];
    const bool has_b = (CB == kRuntime) ? a.code[2 * p + 1] >= 0 : CB != kNone;
    constexpr bool need_k = needs_kinv<CA>() || needs_kinv<CB>();
    const int mx = (nx - x) % nx;
    const float kxx = a.kx[x], kxm = a.kx[mx];
#pragma unroll
    for (int pr = 0; pr < 2; ++pr) {
        const int xa = pr == 0 ? x : mx, xb = pr == 0 ? mx : x;   // columns of the pair
        const float kxa = pr == 0 ? kxx : kxm, kxb = pr == 0 ? kxm : kxx;
        const float2 c1 = cA[xa], c2 = cB[xb];
        const bool om_needed = (CA == kRuntime || CB == kRuntime) && a.needs_omega;
        const float o1 = om_needed ? omA[xa] : 0.f, o2 = om_needed ? omB[xb] : 0.f;
        float k1 = 0.f, k2 = 0.f, ki1 = 0.f, ki2 = 0.f;
        if constexpr (need_k) {
            // |k| and 1/|k| from one reciprocal square root (1/|k| is 0 where |k| does not
            // exceed min(kx_res, ky_res)/2, ocean.py:142-148)
            const float q1 = fadd(fmul(kxa, kxa), fmul(kyr, kyr));
            const float q2 = fadd(fmul(kxb, kxb), fmul(kymr, kymr));
            const float r1 = q1 > 0.f ? rsqrtf(q1) : 0.f, r2 = q2 > 0.f ? rsqrtf(q2) : 0.f;
            k1 = q1 * r1;
            k2 = q2 * r2;
            ki1 = k1 > a.kmin_half ? r1 : 0.f;
            ki2 = k2 > a.kmin_half ? r2 : 0.f;
        }
        const float2 xa1 = c_mul(mult_ct<CA>(ma, kxa, kyr, k1, ki1, o1), c1);
        const float2 xa2 = c_mul(mult_ct<CA>(ma, kxb, kymr, k2, ki2, o2), c2);
        float2 xb1 = make_float2(0.f, 0.f), xb2 = make_float2(0.f, 0.f);
        if (has_b) {
            xb1 = c_mul(mult_ct<CB>(mb, kxa, kyr, k1, ki1, o1), c1);
            xb2 = c_mul(mult_ct<CB>(mb, kxb, kymr, k2, ki2, o2), c2);
        }
        // Z(p) = (XA(p) + conj XA(-p)) / 2 + i (XB(p) + conj XB(-p)) / 2
        rowA[pad_idx(xa)] = make_float2(0.5f * (xa1.x + xa2.x) - 0.5f * (xb1.y - xb2.y),
                                        0.5f * (xa1.y - xa2.y) + 0.5f * (xb1.x + xb2.x));
        rowB[pad_idx(xb)] = make_float2(0.5f * (xa2.x + xa1.x) - 0.5f * (xb2.y - xb1.y),
                                        0.5f * (xa2.y - xa1.y) + 0.5f * (xb2.x + xb1.x));
    }
}

// One packed transform of the row pass: build, transform, store.
template <int N, int CA, int CB>
OCS_D void row_transform(const SurfaceArgs &a, int p, int nx, int ny, int r, int mr, float kyr, float kymr,
                         const float2 *cA, const float2 *cB, const float *omA, const float *omB,
                         float2 *rowA, float2 *rowB, const float2 *stw, int vstride) {
    const int nq = nx / 2 + 1;
    for (int x = threadIdx.x; x < nq; x += blockDim.x)
        build_packed<CA, CB>(a, p, x, nx, kyr, kymr, cA, cB, omA, omB, rowA, rowB);
    __syncthreads();
    if constexpr (N > 0) {
        // the last stage writes straight into the scratch plane
        const RowStore st{a.scratch + (size_t)p * ny * nx, nx, r, mr};
        ifft_pow2<N, 2, rows_threads<N>(), false, true>(rowA, vstride, stw, NoLoad(), st);
    } else {
        const float2 *res = ifft_generic(rowA, rowB + vstride, vstride, 2, a.px);
        float2 *outA = a.scratch + ((size_t)p * ny + r) * nx;
        float2 *outB = a.scratch + ((size_t)p * ny + mr) * nx;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            outA[x] = res[pad_idx(x)];
            if (mr != r) outB[x] = res[vstride + pad_idx(x)];
        }
    }
    __syncthreads();
}

// Pass 1, one item = the mirror row pair (r, ny - r).  Shared memory: c(t) of rows r and
// mr ([2][nx], unpadded), then the two padded FFT rows (and, for non-power-of-two lengths,
// two more for the ping-pong), then (power-of-two lengths) the stage-major twiddles, which
// are only (re)loaded when load_tw is set.
template <int N, int PROG>
OCS_D void rows_item(const SurfaceArgs &a, int r, float2 *sbuf, bool load_tw) {
    const int nx = (N > 0) ? N : a.nx;
    const int ny = a.ny;
    const int mr = (ny - r) % ny;
    const int vstride = (N > 0) ? pow2_vstride(nx, 2) : padded_len(nx);
    float2 *cA = sbuf, *cB = sbuf + nx;
    float2 *rowA = sbuf + 2 * nx, *rowB = rowA + vstride;
    float2 *stw = rowB + vstride;                 // power-of-two lengths: twiddles in smem
    if (N > 0 && load_tw)
        for (int i = threadIdx.x; i < nx; i += blockDim.x) stw[i] = a.stw_x[i];
    const float kyr = a.ky[r], kymr = a.ky[mr];
    const float *omA = a.omega + (size_t)r * nx, *omB = a.omega + (size_t)mr * nx;

    if constexpr (N > 0 && N % rows_threads<N>() == 0) {
        // all loads of the thread's columns first, then the phase rotations
        constexpr int T = rows_threads<N>(), J = N / T;
        float2 c0[J], c1[J];
        float o0[J], o1[J];
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int x = threadIdx.x + j * T;
            c0[j] = a.coefs[(size_t)r * nx + x];
            c1[j] = a.coefs[(size_t)mr * nx + x];
            o0[j] = a.omega[(size_t)r * nx + x];
            o1[j] = a.omega[(size_t)mr * nx + x];
        }
#pragma unroll
        for (int j = 0; j < J; ++j) {
            const int x = threadIdx.x + j * T;
            cA[x] = phased_v(c0[j], o0[j], a.t);
            cB[x] = phased_v(c1[j], o1[j], a.t);
        }
    } else {
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            cA[x] = phased(a, r, x);
            cB[x] = phased(a, mr, x);
        }
    }
    __syncthreads();

#define OCS_ROW_T(P, CA, CB) \
    row_transform<N, CA, CB>(a, P, nx, ny, r, mr, kyr, kymr, cA, cB, omA, omB, rowA, rowB, stw, vstride)
    if constexpr (PROG == 1) {
        OCS_ROW_T(0, OCS_FIELD_DX, OCS_FIELD_DY);
        OCS_ROW_T(1, OCS_FIELD_DZ, OCS_FIELD_DIFFX);
        OCS_ROW_T(2, OCS_FIELD_DIFFY, OCS_FIELD_DIFFXX);
        OCS_ROW_T(3, OCS_FIELD_DIFFYY, OCS_FIELD_DIFFXY);
    } else if constexpr (PROG == 2) {
        OCS_ROW_T(0, OCS_FIELD_DX, OCS_FIELD_DY);
        OCS_ROW_T(1, OCS_FIELD_DZ, OCS_FIELD_DIFFX);
        OCS_ROW_T(2, OCS_FIELD_DIFFY, kNone);
    } else {
        for (int p = 0; p < a.npair; ++p) OCS_ROW_T(p, kRuntime, kRuntime);
    }
#undef OCS_ROW_T
}

template <int N, int PROG>
__global__ void __launch_bounds__(rows_threads<N>(), rows_threads<N>() <= 512 ? 2 : 1)
surface_rows_kernel(const __grid_constant__ SurfaceArgs a) {
    extern __shared__ __align__(16) float2 sbuf[];
    rows_item<N, PROG>(a, blockIdx.x, sbuf, true);
}

// Pass 2, one item = (transform p, tile of TILE columns starting at x0).  Power-of-two
// lengths read the tile inside the first FFT stage and unpack the fields inside the last.
template <int N, int TILE>
OCS_D void cols_item(const SurfaceArgs &a, int p, int x0, float2 *sbuf, bool load_tw) {
    const int nx = a.nx;
    const int ny = (N > 0) ? N : a.ny;
    const int vstride = (N > 0) ? pow2_vstride(ny, TILE) : padded_len(ny);
    const float2 *src = a.scratch + (size_t)p * ny * nx;
    const ColStore st{a.dst[2 * p], a.dst[2 * p + 1], a.swell_exp, a.swell_rot, a.swm[2 * p],
                      a.swm[2 * p + 1], a.inv_n, a.add[2 * p], a.add[2 * p + 1], nx, x0};
    if constexpr (N > 0) {
        float2 *stw = sbuf + TILE * vstride;      // twiddles in smem (first used in stage 2)
        if (load_tw)
            for (int i = threadIdx.x; i < ny; i += blockDim.x) stw[i] = a.stw_y[i];
        ifft_pow2<N, TILE, cols_threads<N, TILE>(), true, true>(sbuf, vstride, stw, ColLoad{src, nx, x0}, st);
    } else {
        for (int i = threadIdx.x; i < ny * TILE; i += blockDim.x) {
            const int y = i / TILE, w = i - y * TILE;
            const int x = x0 + w;
            sbuf[w * vstride + pad_idx(y)] = (x < nx) ? src[(size_t)y * nx + x] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        const float2 *res = ifft_generic(sbuf, sbuf + TILE * vstride, vstride, TILE, a.py);
        for (int i = threadIdx.x; i < ny * TILE; i += blockDim.x) {
            const int y = i / TILE, w = i - y * TILE;
            st(w, y, res[w * vstride + pad_idx(y)]);
        }
    }
}

template <int N, int TILE>
__global__ void __launch_bounds__(cols_threads<N, TILE>(), cols_threads<N, TILE>() <= 512 ? 2 : 1)
surface_cols_kernel(const __grid_constant__ SurfaceArgs a) {
    extern __shared__ __align__(16) float2 sbuf[];
    cols_item<N, TILE>(a, blockIdx.y, blockIdx.x * TILE, sbuf, true);
}

// Choppy-wave slopes and curvatures from the auxiliary fields (ocean.py:451-456, 468-482).
struct ChoppyArgs {
    long long n;
    const float *ax, *ay, *axx, *ayy, *axxx, *ayyy, *axxy, *fxx, *fyy, *fxy;
    float *diffx, *diffy, *diffxx, *diffyy, *diffxy;
    const float2 *swell_exp;
    float2 swell_rot;
    float2 sw_dx, sw_dy, sw_dxx, sw_dyy, sw_dxy;
};

// One facet of the choppy step, with the swell rotation of the current time.
OCS_D void choppy_px(const ChoppyArgs &c, long long i, float2 swell_rot) {
    float2 s = make_float2(0.f, 0.f);
    if (c.swell_exp) s = c_mul(c.swell_exp[i], swell_rot);
    const float ax = c.ax[i], ay = c.ay[i], axx = c.axx[i], ayy = c.ayy[i];
    if (c.diffx) {
        c.diffx[i] = fadd(ax / (1.f + axx), fsub(fmul(c.sw_dx.x, s.x), fmul(c.sw_dx.y, s.y)));
        c.diffy[i] = fadd(ay / (1.f + ayy), fsub(fmul(c.sw_dy.x, s.x), fmul(c.sw_dy.y, s.y)));
    }
    if (c.diffxx) {
        const float px = 1.f + axx, py = 1.f + ayy;
        float vxx = (px * c.fxx[i] - c.axxx[i] * ax) / powf(px, 3.f);
        float vyy = (py * c.fyy[i] - c.ayyy[i] * ay) / powf(py, 3.f);
        float vxy = (px * c.fxy[i] - c.axxy[i] * ax) / (powf(px, 2.f) * py);
        c.diffxx[i] = fadd(vxx, fsub(fmul(c.sw_dxx.x, s.x), fmul(c.sw_dxx.y, s.y)));
        c.diffyy[i] = fadd(vyy, fsub(fmul(c.sw_dyy.x, s.x), fmul(c.sw_dyy.y, s.y)));
        c.diffxy[i] = fadd(vxy, fsub(fmul(c.sw_dxy.x, s.x), fmul(c.sw_dxy.y, s.y)));
    }
}

__global__ void surface_choppy_kernel(ChoppyArgs c) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < c.n;
         i += (long long)gridDim.x * blockDim.x)
        choppy_px(c, i, c.swell_rot);
}

// ---------------------------------------------------------------------------------------
// Host side.
static bool make_plan(int n, FftPlan &pl) {
    pl.n = n;
    pl.nstages = 0;
    int m = n;
    // radix 8 first, then a single 4 or 2 for the remaining power of two, then 3, 5, 7
    while (m % 8 == 0) { if (pl.nstages >= kMaxStages) return false; pl.radix[pl.nstages++] = 8; m /= 8; }
    while (m % 4 == 0) { if (pl.nstages >= kMaxStages) return false; pl.radix[pl.nstages++] = 4; m /= 4; }
    while (m % 2 == 0) { if (pl.nstages >= kMaxStages) return false; pl.radix[pl.nstages++] = 2; m /= 2; }
    const int others[3] = {3, 5, 7};
    for (int k = 0; k < 3; ++k)
        while (m % others[k] == 0) {
            if (pl.nstages >= kMaxStages) return false;
            pl.radix[pl.nstages++] = others[k];
            m /= others[k];
        }
    return m == 1;
}


// Stage-major twiddles of the power-of-two transform (radices of pow2_stage_radix): stage s with
// radix R after radices of product ns holds w^(r*j*n/(ns*R)) at [(r-1)*ns + j],
// 1 <= r < R, 0 <= j < ns, so that the lanes of a warp (consecutive j) read consecutive
// entries.  Total length < n.
__global__ void staged_twiddle_kernel(float2 *tw, int n) {
    int base = 0;
    for (int ns = 1; ns < n;) {
        const int rem = n / ns;
        const int R = pow2_stage_radix(n, ns);
        const int cnt = (R - 1) * ns;
        const int tstep = n / (ns * R);
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) {
            const int r = e / ns + 1, j = e % ns;
            double s, c;
            sincospi(2.0 * (double)(r * j * tstep) / (double)n, &s, &c);
            tw[base + e] = make_float2((float)c, (float)s);
        }
        base += cnt;
        ns *= R;
    }
}

__global__ void twiddle_kernel(float2 *tw, int n) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < n; m += gridDim.x * blockDim.x) {
        double s, c;
        sincospi(2.0 * (double)m / (double)n, &s, &c);
        tw[m] = make_float2((float)c, (float)s);
    }
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Workspace layout: [twiddles x (nx) | twiddles y (ny) | scratch planes npair*ny*nx].
static size_t ws_twx(int) { return 0; }
static size_t ws_twy(int nx) { return align256((size_t)nx * sizeof(float2)); }
static size_t ws_stx(int nx, int ny) { return ws_twy(nx) + align256((size_t)ny * sizeof(float2)); }
static size_t ws_sty(int nx, int ny) { return ws_stx(nx, ny) + align256((size_t)nx * sizeof(float2)); }
static size_t ws_scratch(int nx, int ny) { return ws_sty(nx, ny) + align256((size_t)ny * sizeof(float2)); }
static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Dynamic shared memory of a row item / column item.
static size_t rows_smem_bytes(int key, int nx) {
    return (key > 0) ? (3 * (size_t)nx + 2 * (size_t)pow2_vstride(nx, 2)) * sizeof(float2)
                     : (2 * (size_t)nx + 4 * (size_t)padded_len(nx)) * sizeof(float2);
}
static size_t cols_smem_bytes(int key, int tile, int ny) {
    return (key > 0) ? ((size_t)tile * pow2_vstride(ny, tile) + ny) * sizeof(float2)
                     : 2 * (size_t)tile * padded_len(ny) * sizeof(float2);
}
constexpr size_t kSmemLimit = 227 * 1024;
constexpr size_t kBatchStatic = 4096;     // static smem of the batch kernels (args + prefix)

template <int N, int PROG>
static cudaError_t launch_rows_prog(const SurfaceArgs &a, cudaStream_t st) {
    const size_t smem = rows_smem_bytes(N, a.nx);
    if (smem > kSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = ensure_smem((const void *)surface_rows_kernel<N, PROG>, smem);
    if (e != cudaSuccess) return e;
    surface_rows_kernel<N, PROG><<<a.ny / 2 + 1, rows_threads<N>(), smem, st>>>(a);
    return cudaGetLastError();
}

// Field program of a packed code list (see surface_rows_kernel).
static int field_program(const SurfaceArgs &a) {
    static const int std8[8] = {OCS_FIELD_DX, OCS_FIELD_DY, OCS_FIELD_DZ, OCS_FIELD_DIFFX,
                                OCS_FIELD_DIFFY, OCS_FIELD_DIFFXX, OCS_FIELD_DIFFYY, OCS_FIELD_DIFFXY};
    static const int std5[6] = {OCS_FIELD_DX, OCS_FIELD_DY, OCS_FIELD_DZ, OCS_FIELD_DIFFX, OCS_FIELD_DIFFY, -1};
    bool is8 = a.npair == 4, is5 = a.npair == 3;
    for (int i = 0; i < 8 && is8; ++i) is8 = a.code[i] == std8[i];
    for (int i = 0; i < 6 && is5; ++i) is5 = a.code[i] == std5[i];
    return is8 ? 1 : (is5 ? 2 : 0);
}

template <int N>
static cudaError_t launch_rows_n(const SurfaceArgs &a, cudaStream_t st) {
    switch (a.prog) {
        case 1: return launch_rows_prog<N, 1>(a, st);
        case 2: return launch_rows_prog<N, 2>(a, st);
        default: return launch_rows_prog<N, 0>(a, st);
    }
}

template <int N, int TILE>
static cudaError_t launch_cols_n(const SurfaceArgs &a, cudaStream_t st) {
    const size_t smem = cols_smem_bytes(N, TILE, a.ny);
    if (smem > kSmemLimit) return cudaErrorInvalidValue;
    cudaError_t e = ensure_smem((const void *)surface_cols_kernel<N, TILE>, smem);
    if (e != cudaSuccess) return e;
    dim3 grid((a.nx + TILE - 1) / TILE, a.npair);
    surface_cols_kernel<N, TILE><<<grid, cols_threads<N, TILE>(), smem, st>>>(a);
    return cudaGetLastError();
}

static cudaError_t launch_rows(const SurfaceArgs &a, cudaStream_t st) {
    switch (a.nx) {
        case 64: return launch_rows_n<64>(a, st);
        case 128: return launch_rows_n<128>(a, st);
        case 256: return launch_rows_n<256>(a, st);
        case 512: return launch_rows_n<512>(a, st);
        case 1024: return launch_rows_n<1024>(a, st);
        case 2048: return launch_rows_n<2048>(a, st);
        case 4096: return launch_rows_n<4096>(a, st);
        case 8192: return launch_rows_n<8192>(a, st);
        default: return launch_rows_n<0>(a, st);
    }
}

static cudaError_t launch_cols(const SurfaceArgs &a, cudaStream_t st) {
    switch (a.ny) {
        case 64: return launch_cols_n<64, 4>(a, st);
        case 128: return launch_cols_n<128, 4>(a, st);
        case 256: return launch_cols_n<256, 4>(a, st);
        case 512: return launch_cols_n<512, 8>(a, st);
        case 1024: return launch_cols_n<1024, 8>(a, st);
        case 2048: return launch_cols_n<2048, 8>(a, st);
        case 4096: return launch_cols_n<4096, 4>(a, st);
        case 8192: return launch_cols_n<8192, 2>(a, st);
        default: return launch_cols_n<0, 4>(a, st);
    }
}


// ---------------------------------------------------------------------------------------
// Scene batch (batch.cuh): one launch of the row (column) pass covers every live slot whose
// transform length is N.  The host sizes the grid for all slots in use; CTAs enumerate
// the live slots' items over the slot table and take one item each (a CTA that loops over
// several items makes the compiler keep the FFT's loop-invariant shared-memory addressing
// in registers across items, which spills).

// Copy a slot's SurfaceArgs into shared memory and set this pulse's time, additive terms
// and swell rotation from the slot's per-pulse tables.
OCS_D void load_slot_surface(const SlotState &g, SurfaceArgs &sa) {
    const int *src = static_cast<const int *>(g.sargs);
    int *dst = reinterpret_cast<int *>(&sa);
    for (int i = threadIdx.x; i < (int)(sizeof(SurfaceArgs) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int c = g.counter;
        sa.t = g.t_tab[c];
        for (int f = 0; f < g.nfields; ++f) sa.add[f] = g.add_tab[(size_t)c * g.nfields + f];
        if (g.swrot_tab) sa.swell_rot = g.swrot_tab[c];
    }
    __syncthreads();
}

OCS_D bool slot_surface_live(const SlotState &g) {
    return slot_live(g) && (g.flags_tab[g.counter] & kFlagSurface);
}

template <int N, int PROG>
__global__ void __launch_bounds__(rows_threads<N>(), rows_threads<N>() <= 512 ? 2 : 1)
batch_rows_kernel(const __grid_constant__ BatchRef b) {
    extern __shared__ __align__(16) float2 sbuf[];
    __shared__ SurfaceArgs sa;
    __shared__ int pref[kMaxSlots + 1];
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        return (g.rows_key == N && g.prog == PROG && slot_surface_live(g)) ? g.ny / 2 + 1 : 0;
    });
    const int item = blockIdx.x;
    if (item >= total) return;
    const int s = find_slot(pref, b.nslots, item);
    load_slot_surface(b.slots[s], sa);
    rows_item<N, PROG>(sa, item - pref[s], sbuf, true);
}

template <int N, int TILE>
__global__ void __launch_bounds__(cols_threads<N, TILE>(), cols_threads<N, TILE>() <= 512 ? 2 : 1)
batch_cols_kernel(const __grid_constant__ BatchRef b) {
    extern __shared__ __align__(16) float2 sbuf[];
    __shared__ SurfaceArgs sa;
    __shared__ int pref[kMaxSlots + 1];
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        return (g.cols_key == N && slot_surface_live(g)) ? g.npair * ((g.nx + TILE - 1) / TILE) : 0;
    });
    const int item = blockIdx.x;
    if (item >= total) return;
    const int s = find_slot(pref, b.nslots, item);
    load_slot_surface(b.slots[s], sa);
    const int j = item - pref[s];
    const int ntile = (sa.nx + TILE - 1) / TILE;
    const int p = j / ntile;
    cols_item<N, TILE>(sa, p, (j - p * ntile) * TILE, sbuf, true);
}

template <int N, int PROG>
static int batch_rows_prog(const BatchRef &b, int grid, size_t smem, cudaStream_t st) {
    auto k = batch_rows_kernel<N, PROG>;
    if (smem + kBatchStatic > kSmemLimit) return OCS_ERR_SIZE;
    if (ensure_smem((const void *)k, smem) != cudaSuccess) return OCS_ERR_CUDA;
    k<<<grid, rows_threads<N>(), smem, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <int N, int TILE>
static int batch_cols_n(const BatchRef &b, int grid, size_t smem, cudaStream_t st) {
    auto k = batch_cols_kernel<N, TILE>;
    if (smem + kBatchStatic > kSmemLimit) return OCS_ERR_SIZE;
    if (ensure_smem((const void *)k, smem) != cudaSuccess) return OCS_ERR_CUDA;
    k<<<grid, cols_threads<N, TILE>(), smem, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <int N>
static int batch_rows_n(const BatchRef &b, int prog, int grid, size_t smem, cudaStream_t st) {
    switch (prog) {
        case 1: return batch_rows_prog<N, 1>(b, grid, smem, st);
        case 2: return batch_rows_prog<N, 2>(b, grid, smem, st);
        default: return batch_rows_prog<N, 0>(b, grid, smem, st);
    }
}

size_t surface_args_bytes() { return sizeof(SurfaceArgs); }

int surface_key(int n) {
    switch (n) {
        case 64: case 128: case 256: case 512: case 1024: case 2048: case 4096: case 8192: return n;
        default: {
            FftPlan pl;
            return (n >= 2 && n <= 8192 && make_plan(n, pl)) ? 0 : -1;
        }
    }
}

// Column tile width per column length: wider tiles give longer contiguous row segments
// (loads of TILE complex64, stores of TILE float32 per row) where shared memory allows.
int surface_cols_tile(int key) {
    return key == 8192 ? 2 : ((key == 512 || key == 1024 || key == 2048) ? 8 : 4);
}

long long surface_rows_smem(int key, int nx) {
    const size_t b = rows_smem_bytes(key, nx);
    return b + kBatchStatic > kSmemLimit ? -1 : (long long)b;
}

long long surface_cols_smem(int key, int ny) {
    const size_t b = cols_smem_bytes(key, surface_cols_tile(key), ny);
    return b + kBatchStatic > kSmemLimit ? -1 : (long long)b;
}

int batch_launch_rows(const BatchRef &b, int key, int prog, int grid, size_t smem, cudaStream_t st) {
    if (grid < 1) return OCS_OK;
    switch (key) {
        case 64: return batch_rows_n<64>(b, prog, grid, smem, st);
        case 128: return batch_rows_n<128>(b, prog, grid, smem, st);
        case 256: return batch_rows_n<256>(b, prog, grid, smem, st);
        case 512: return batch_rows_n<512>(b, prog, grid, smem, st);
        case 1024: return batch_rows_n<1024>(b, prog, grid, smem, st);
        case 2048: return batch_rows_n<2048>(b, prog, grid, smem, st);
        case 4096: return batch_rows_n<4096>(b, prog, grid, smem, st);
        case 8192: return batch_rows_n<8192>(b, prog, grid, smem, st);
        case 0: return batch_rows_n<0>(b, prog, grid, smem, st);
        default: return OCS_ERR_ARG;
    }
}

int batch_launch_cols(const BatchRef &b, int key, int grid, size_t smem, cudaStream_t st) {
    if (grid < 1) return OCS_OK;
    switch (key) {
        case 64: return batch_cols_n<64, 4>(b, grid, smem, st);
        case 128: return batch_cols_n<128, 4>(b, grid, smem, st);
        case 256: return batch_cols_n<256, 4>(b, grid, smem, st);
        case 512: return batch_cols_n<512, 8>(b, grid, smem, st);
        case 1024: return batch_cols_n<1024, 8>(b, grid, smem, st);
        case 2048: return batch_cols_n<2048, 8>(b, grid, smem, st);
        case 4096: return batch_cols_n<4096, 4>(b, grid, smem, st);
        case 8192: return batch_cols_n<8192, 2>(b, grid, smem, st);
        case 0: return batch_cols_n<0, 4>(b, grid, smem, st);
        default: return OCS_ERR_ARG;
    }
}

// Choppy step of the batch: 256 facets of one live choppy slot per item.
__global__ void batch_choppy_kernel(const __grid_constant__ BatchRef b) {
    __shared__ int pref[kMaxSlots + 1];
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        if (!slot_live(g) || !g.cargs) return 0;
        return (int)((static_cast<const ChoppyArgs *>(g.cargs)->n + 255) / 256);
    });
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int s = find_slot(pref, b.nslots, item);
        const SlotState &g = b.slots[s];
        const ChoppyArgs &c = *static_cast<const ChoppyArgs *>(g.cargs);
        const long long i = (long long)(item - pref[s]) * 256 + threadIdx.x;
        const float2 rot = g.swrot_tab ? g.swrot_tab[g.counter] : make_float2(0.f, 0.f);
        if (i < c.n) choppy_px(c, i, rot);
    }
}

size_t choppy_args_bytes() { return sizeof(ChoppyArgs); }

int batch_launch_choppy(const BatchRef &b, cudaStream_t st) {
    int sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return OCS_ERR_CUDA;
    batch_choppy_kernel<<<sms * 16, 256, 0, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

}  // namespace ocs

using namespace ocs;

extern "C" int64_t ocs_surface_workspace_bytes(int32_t nx, int32_t ny, int32_t nfields) {
    if (nx < 2 || ny < 2 || nfields < 1 || nfields > 2 * kMaxPacked) return -1;
    int npair = (nfields + 1) / 2;
    return (int64_t)(ws_scratch(nx, ny) + (size_t)npair * nx * ny * sizeof(float2));
}

extern "C" int ocs_surface_prepare(int32_t nx, int32_t ny, void *workspace, void *stream) {
    if (!workspace || nx < 2 || ny < 2) return OCS_ERR_ARG;
    FftPlan px, py;
    if (!make_plan(nx, px) || !make_plan(ny, py)) return OCS_ERR_UNSUPPORTED;
    char *ws = (char *)workspace;
    cudaStream_t st = (cudaStream_t)stream;
    twiddle_kernel<<<(nx + 255) / 256, 256, 0, st>>>((float2 *)(ws + ws_twx(nx)), nx);
    twiddle_kernel<<<(ny + 255) / 256, 256, 0, st>>>((float2 *)(ws + ws_twy(nx)), ny);
    if (is_pow2(nx)) staged_twiddle_kernel<<<(nx + 255) / 256, 256, 0, st>>>((float2 *)(ws + ws_stx(nx, ny)), nx);
    if (is_pow2(ny)) staged_twiddle_kernel<<<(ny + 255) / 256, 256, 0, st>>>((float2 *)(ws + ws_sty(nx, ny)), ny);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// Launch arguments of a surface descriptor at time t (shared by the single-scene entry
// points and the scene batch).
int fill_surface_args(const ocs_surface_desc *d, float t, SurfaceArgs &a) {
    if (!d || !d->coefs_d || !d->omega_d || !d->kx_d || !d->ky_d || !d->workspace_d) return OCS_ERR_ARG;
    const int nx = d->nx, ny = d->ny;
    if (nx < 2 || ny < 2 || d->nfields < 1 || d->nfields > 2 * kMaxPacked) return OCS_ERR_ARG;
    if (nx > 8192 || ny > 8192) return OCS_ERR_SIZE;
    memset(&a, 0, sizeof(a));
    a.nx = nx;
    a.ny = ny;
    a.coefs = (const float2 *)d->coefs_d;
    a.omega = d->omega_d;
    a.kx = d->kx_d;
    a.ky = d->ky_d;
    a.kmin_half = d->kmin_half;
    a.t = t;
    a.inv_n = (float)(1.0 / ((double)nx * (double)ny));
    a.npair = (d->nfields + 1) / 2;
    for (int i = 0; i < 2 * a.npair; ++i) {
        if (i < d->nfields) {
            if (d->codes[i] < 0 || d->codes[i] >= OCS_FIELD_COUNT || !d->dst_d[i]) return OCS_ERR_ARG;
            a.code[i] = d->codes[i];
            a.mult[i] = mult_desc(d->codes[i]);
            if (a.mult[i].d > 0 || a.mult[i].hmtf) a.needs_omega = 1;
            a.dst[i] = d->dst_d[i];
            a.add[i] = d->add ? d->add[i] : 0.f;
            a.swm[i] = d->swell_mult ? make_float2(d->swell_mult[2 * i], d->swell_mult[2 * i + 1])
                                     : make_float2(0.f, 0.f);
        } else {
            a.code[i] = -1;
            a.dst[i] = nullptr;
        }
    }
    a.swell_exp = (const float2 *)d->swell_exp_d;
    a.swell_rot = make_float2(d->swell_rot_re, d->swell_rot_im);
    if (!make_plan(nx, a.px) || !make_plan(ny, a.py)) return OCS_ERR_UNSUPPORTED;
    char *ws = (char *)d->workspace_d;
    a.px.tw = (const float2 *)(ws + ws_twx(nx));
    a.py.tw = (const float2 *)(ws + ws_twy(nx));
    a.stw_x = (const float2 *)(ws + ws_stx(nx, ny));
    a.stw_y = (const float2 *)(ws + ws_sty(nx, ny));
    a.scratch = (float2 *)(ws + ws_scratch(nx, ny));
    a.prog = field_program(a);
    return OCS_OK;
}

namespace ocs {
int surface_args_fill(const ocs_surface_desc *d, void *out, int *prog) {
    SurfaceArgs a;
    const int st = fill_surface_args(d, 0.f, a);
    if (st == OCS_OK) {
        memcpy(out, &a, sizeof(a));
        *prog = a.prog;
    }
    return st;
}
}  // namespace ocs

extern "C" int ocs_surface_update_passes(const ocs_surface_desc *d, float t, int passes, void *stream) {
    if (passes < 1 || passes > 3) return OCS_ERR_ARG;
    SurfaceArgs a;
    const int fst = fill_surface_args(d, t, a);
    if (fst != OCS_OK) return fst;
    cudaStream_t st = (cudaStream_t)stream;

    cudaError_t e = (passes & 1) ? launch_rows(a, st) : cudaSuccess;
    if (e != cudaSuccess) return e == cudaErrorInvalidValue ? OCS_ERR_SIZE : OCS_ERR_CUDA;
    e = (passes & 2) ? launch_cols(a, st) : cudaSuccess;
    if (e != cudaSuccess) return e == cudaErrorInvalidValue ? OCS_ERR_SIZE : OCS_ERR_CUDA;
    return OCS_OK;
}

extern "C" int ocs_surface_update(const ocs_surface_desc *d, float t, void *stream) {
    return ocs_surface_update_passes(d, t, 3, stream);
}

int ocs::choppy_args_fill(const ocs_choppy_desc *d, void *out) {
    if (!d || d->n <= 0 || !d->ax_d || !d->ay_d || !d->axx_d || !d->ayy_d) return OCS_ERR_ARG;
    ChoppyArgs c;
    memset(&c, 0, sizeof(c));
    c.n = d->n;
    c.ax = d->ax_d; c.ay = d->ay_d; c.axx = d->axx_d; c.ayy = d->ayy_d;
    c.axxx = d->axxx_d; c.ayyy = d->ayyy_d; c.axxy = d->axxy_d;
    c.fxx = d->fxx_d; c.fyy = d->fyy_d; c.fxy = d->fxy_d;
    c.diffx = d->diffx_d; c.diffy = d->diffy_d;
    c.diffxx = d->diffxx_d; c.diffyy = d->diffyy_d; c.diffxy = d->diffxy_d;
    if ((c.diffx == nullptr) != (c.diffy == nullptr)) return OCS_ERR_ARG;
    if (c.diffxx && (!c.diffyy || !c.diffxy || !c.axxx || !c.ayyy || !c.axxy || !c.fxx || !c.fyy || !c.fxy))
        return OCS_ERR_ARG;
    c.swell_exp = (const float2 *)d->swell_exp_d;
    c.swell_rot = make_float2(d->swell_rot_re, d->swell_rot_im);
    const float *m = d->swell_mult;
    if (m) {
        c.sw_dx = make_float2(m[0], m[1]); c.sw_dy = make_float2(m[2], m[3]);
        c.sw_dxx = make_float2(m[4], m[5]); c.sw_dyy = make_float2(m[6], m[7]);
        c.sw_dxy = make_float2(m[8], m[9]);
    }
    memcpy(out, &c, sizeof(c));
    return OCS_OK;
}

extern "C" int ocs_surface_choppy(const ocs_choppy_desc *d, void *stream) {
    ChoppyArgs c;
    const int st = choppy_args_fill(d, &c);
    if (st != OCS_OK) return st;
    long long blocks = (d->n + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    surface_choppy_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(c);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------
// Surface update without allocation.
//
// Some callers cannot allocate device memory: hosts that drive this library through the
// bare C ABI with no device allocator of their own (for instance a ctypes binding in the
// reference code base, which has no CUDA runtime beside this library), and real-time loops
// that must never block on an allocation.  ocs_surface_update_noalloc serves them: its
// workspace (twiddle tables and the packed FFT scratch planes) lives in the file-scope
// device array below, so the caller passes only inputs and outputs.
//
// * Capacity: kNoAllocScratchBytes (32 MiB) per device, i.e. ocs_surface_workspace_bytes(
//   nx, ny, nfields) must not exceed it (for example 1024 x 1024 with up to 6 fields or
//   512 x 512 with up to 24); larger requests return OCS_ERR_SIZE.  The array is part of
//   the loaded module, so every GPU that loads the library holds it until exit.
// * Set-up: every call resolves the array's device address on the current device
//   (cudaGetSymbolAddress; cheap once the module is loaded, and never stale after a
//   context reset).  With lazy module loading the first call on a device also loads the
//   module and its 32 MiB array, so make one warm-up call before any latency-critical
//   loop or stream capture.
// * Errors: the descriptor is checked completely before anything is launched, so a bad
//   descriptor returns OCS_ERR_ARG / OCS_ERR_SIZE with the array untouched.
// * Sharing: every call on a device uses the same array, which keeps the last call's
//   contents.  Each call rewrites the twiddle tables and overwrites the scratch planes
//   completely before reading them, so nothing needs clearing, but calls that overlap on
//   the GPU (different streams, or different host threads) race on the array and must be
//   serialised by the caller.
// * No cudaMalloc / cudaFree or any allocating library routine is called.
constexpr size_t kNoAllocScratchBytes = 32u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

extern "C" int ocs_surface_update_noalloc(const ocs_surface_desc *d, float t, void *stream) {
    if (!d) return OCS_ERR_ARG;
    const int64_t need = ocs_surface_workspace_bytes(d->nx, d->ny, d->nfields);
    if (need < 0) return OCS_ERR_ARG;
    if ((size_t)need > kNoAllocScratchBytes) return OCS_ERR_SIZE;
    void *ws = nullptr;
    if (cudaGetSymbolAddress(&ws, g_noalloc_scratch) != cudaSuccess || !ws) return OCS_ERR_CUDA;
    ocs_surface_desc local = *d;
    local.workspace_d = ws;
    SurfaceArgs check;                     // full argument check before the array is touched
    const int fst = fill_surface_args(&local, t, check);
    if (fst != OCS_OK) return fst;
    const int st = ocs_surface_prepare(d->nx, d->ny, ws, stream);
    if (st != OCS_OK) return st;
    return ocs_surface_update(&local, t, stream);
}

// ---------------------------------------------------------------------------------------
// Time-interpolated surface (oceansar/surfaces/balancer.py:126-297): every field is the
// float32 blend w_l * F(t_l) + w_h * F(t_h) of the fields synthesised at the two ends of
// the ocean time step around t.
namespace ocs {
struct BlendArgs {
    long long n;
    int nfields;
    const float *a[2 * kMaxPacked];
    const float *b[2 * kMaxPacked];
    float *dst[2 * kMaxPacked];
    float w_l, w_h;
};

__global__ void surface_blend_kernel(const __grid_constant__ BlendArgs g) {
    const long long n4 = g.n / 4;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int f = 0; f < g.nfields; ++f) {
        const float4 *a = reinterpret_cast<const float4 *>(g.a[f]);
        const float4 *b = reinterpret_cast<const float4 *>(g.b[f]);
        float4 *d = reinterpret_cast<float4 *>(g.dst[f]);
        for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += stride) {
            const float4 x = a[i], y = b[i];
            d[i] = make_float4(fadd(fmul(g.w_l, x.x), fmul(g.w_h, y.x)), fadd(fmul(g.w_l, x.y), fmul(g.w_h, y.y)),
                               fadd(fmul(g.w_l, x.z), fmul(g.w_h, y.z)), fadd(fmul(g.w_l, x.w), fmul(g.w_h, y.w)));
        }
        for (long long i = 4 * n4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n; i += stride)
            g.dst[f][i] = fadd(fmul(g.w_l, g.a[f][i]), fmul(g.w_h, g.b[f][i]));
    }
}
}  // namespace ocs

extern "C" int ocs_surface_blend(int64_t n, int32_t nfields, const float *const *a_d, const float *const *b_d,
                                 float *const *dst_d, float w_l, float w_h, void *stream) {
    if (n < 0 || nfields < 0 || nfields > 2 * kMaxPacked) return OCS_ERR_ARG;
    if (n == 0 || nfields == 0) return OCS_OK;
    if (!a_d || !b_d || !dst_d) return OCS_ERR_ARG;
    BlendArgs g;
    memset(&g, 0, sizeof(g));
    g.n = n;
    g.nfields = nfields;
    for (int f = 0; f < nfields; ++f) {
        if (!a_d[f] || !b_d[f] || !dst_d[f]) return OCS_ERR_ARG;
        // the vector path needs 16-byte aligned planes
        if (((uintptr_t)a_d[f] | (uintptr_t)b_d[f] | (uintptr_t)dst_d[f]) & 15) return OCS_ERR_ARG;
        g.a[f] = a_d[f];
        g.b[f] = b_d[f];
        g.dst[f] = dst_d[f];
    }
    g.w_l = w_l;
    g.w_h = w_h;
    long long blocks = (n / 4 + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    surface_blend_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(g);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}
