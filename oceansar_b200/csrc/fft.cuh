// Shared-memory mixed-radix (2, 3, 4, 5, 7, 8, 16) inverse FFT used by the surface kernels.
//
// A CTA transforms `nvec` vectors of length n held in shared memory with the
// self-sorting Stockham formulation: at a stage of radix R after radices of product Ns,
// butterfly j reads x[j + r*n/R] (r < R), multiplies by w^(r*(j mod Ns)*n/(Ns*R)),
// takes an R-point DFT and writes x[(j/Ns)*Ns*R + j mod Ns + r*Ns].  Power-of-two lengths
// are compiled per length (radix 16 while it divides, then 8, then one 4 or 2;
// pow2_stage_radix): each thread keeps its butterflies in
// registers between a read phase and a write phase separated by a barrier, so one buffer
// suffices.  Other lengths (primes 3, 5, 7) run a runtime plan out of place between two
// buffers.  Element i of a vector lives at smem index
// i + (i >> 3) (one pad slot per 8) to break the power-of-two strides of the first stage.
// Twiddles w^m = exp(+2*pi*i*m/n) come from a float64-accurate table in global memory.
#pragma once
#include "common.cuh"

namespace ocs {

constexpr int kMaxStages = 16;

struct FftPlan {
    int n;
    int nstages;
    int radix[kMaxStages];
    const float2 *tw;       // [n] twiddles exp(+2 pi i m / n)
};

OCS_HD int pad_idx(int i) { return i + (i >> 3); }
// Vector stride in shared memory: the padded length rounded up to 4 (mod 16) float2 slots,
// so that the column tiles' transposed stores (4 vectors x 4 consecutive elements per
// half-warp) fall on 16 different 8-byte banks.
OCS_HD int padded_len(int n) {
    int v = n + (n >> 3) + 1;
    return v + ((4 - (v & 15)) & 15);
}

OCS_D float2 c_mul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
OCS_D float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
OCS_D float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
OCS_D float2 c_ipos(float2 a) { return make_float2(-a.y, a.x); }     // +i * a

// In-place R-point inverse DFT (positive exponent) of v[0..R).
template <int R> OCS_D void dft_inv(float2 *v);

template <> OCS_D void dft_inv<2>(float2 *v) {
    float2 a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}
template <> OCS_D void dft_inv<4>(float2 *v) {
    float2 a0 = c_add(v[0], v[2]), a1 = c_sub(v[0], v[2]);
    float2 b0 = c_add(v[1], v[3]), b1 = c_ipos(c_sub(v[1], v[3]));
    v[0] = c_add(a0, b0);
    v[2] = c_sub(a0, b0);
    v[1] = c_add(a1, b1);
    v[3] = c_sub(a1, b1);
}
template <> OCS_D void dft_inv<8>(float2 *v) {
    const float h = 0.70710678118654752f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft_inv<4>(e);
    dft_inv<4>(o);
    // o[k] *= exp(+2 pi i k / 8)
    o[1] = make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y));
    o[2] = c_ipos(o[2]);
    o[3] = make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = c_add(e[k], o[k]);
        v[k + 4] = c_sub(e[k], o[k]);
    }
}
template <> OCS_D void dft_inv<3>(float2 *v) {
    const float c1 = -0.5f, s1 = 0.86602540378443865f;
    float2 a = v[0], b = v[1], c = v[2];
    float2 t = c_add(b, c);
    float2 d = c_sub(b, c);
    float2 m = make_float2(a.x + c1 * t.x, a.y + c1 * t.y);
    v[0] = c_add(a, t);
    v[1] = make_float2(m.x - s1 * d.y, m.y + s1 * d.x);
    v[2] = make_float2(m.x + s1 * d.y, m.y - s1 * d.x);
}
template <> OCS_D void dft_inv<5>(float2 *v) {
    const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
    const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;
    float2 a = v[0];
    float2 t1 = c_add(v[1], v[4]), d1 = c_sub(v[1], v[4]);
    float2 t2 = c_add(v[2], v[3]), d2 = c_sub(v[2], v[3]);
    v[0] = c_add(a, c_add(t1, t2));
    float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
    float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
    float2 n1 = make_float2(s1 * d1.x + s2 * d2.x, s1 * d1.y + s2 * d2.y);
    float2 n2 = make_float2(s2 * d1.x - s1 * d2.x, s2 * d1.y - s1 * d2.y);
    v[1] = make_float2(m1.x - n1.y, m1.y + n1.x);
    v[4] = make_float2(m1.x + n1.y, m1.y - n1.x);
    v[2] = make_float2(m2.x - n2.y, m2.y + n2.x);
    v[3] = make_float2(m2.x + n2.y, m2.y - n2.x);
}
template <> OCS_D void dft_inv<7>(float2 *v) {
    // X[j] = a + sum_k (t_k cos(2 pi jk/7) + i d_k sin(2 pi jk/7)), k = 1..3, with
    // t_k = v[k] + v[7-k] and d_k = v[k] - v[7-k]; X[7-j] takes the conjugate sine part.
    const float C7[7] = {1.f, 0.62348980185873353f, -0.22252093395631440f, -0.90096886790241913f,
                         -0.90096886790241913f, -0.22252093395631440f, 0.62348980185873353f};
    const float S7[7] = {0.f, 0.78183148246802981f, 0.97492791218182361f, 0.43388373911755812f,
                         -0.43388373911755812f, -0.97492791218182361f, -0.78183148246802981f};
    float2 a = v[0];
    float2 t[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { t[k] = c_add(v[k + 1], v[6 - k]); d[k] = c_sub(v[k + 1], v[6 - k]); }
    v[0] = c_add(a, c_add(t[0], c_add(t[1], t[2])));
#pragma unroll
    for (int j = 1; j <= 3; ++j) {
        float2 m = a, n = make_float2(0.f, 0.f);
#pragma unroll
        for (int k = 1; k <= 3; ++k) {
            const int idx = (j * k) % 7;
            m.x += C7[idx] * t[k - 1].x; m.y += C7[idx] * t[k - 1].y;
            n.x += S7[idx] * d[k - 1].x; n.y += S7[idx] * d[k - 1].y;
        }
        v[j] = make_float2(m.x - n.y, m.y + n.x);
        v[7 - j] = make_float2(m.x + n.y, m.y - n.x);
    }
}

// Radix-16 inverse DFT as 4 x 4: A[n2][k1] = DFT4 over n1 of v[4 n1 + n2], then
// X[k1 + 4 k2] = DFT4 over n2 of w16^(n2 k1) A[n2][k1], w16 = exp(+2 pi i / 16).
template <> OCS_D void dft_inv<16>(float2 *v) {
    const float c1 = 0.92387953251128674f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
    float2 a[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        float2 t[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
        dft_inv<4>(t);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
    }
    // twiddles w16^(n2 k1): m = 0, 1, 2, 3 (n2 = 1), 0, 2, 4, 6 (n2 = 2), 0, 3, 6, 9 (n2 = 3)
    const float2 w1 = make_float2(c1, s1), w2 = make_float2(h, h), w3 = make_float2(s1, c1);
    const float2 w6 = make_float2(-h, h), w9 = make_float2(-c1, -s1);
    a[1][1] = c_mul(a[1][1], w1);
    a[1][2] = c_mul(a[1][2], w2);
    a[1][3] = c_mul(a[1][3], w3);
    a[2][1] = c_mul(a[2][1], w2);
    a[2][2] = c_ipos(a[2][2]);
    a[2][3] = c_mul(a[2][3], w6);
    a[3][1] = c_mul(a[3][1], w3);
    a[3][2] = c_mul(a[3][2], w6);
    a[3][3] = c_mul(a[3][3], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
        dft_inv<4>(t);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
    }
}

// Radix of the stage of a power-of-two transform of length n that follows radices of
// product ns: 16 while 16 divides the rest (for n a multiple of 128, so that every stage
// has a multiple of 8 butterflies per vector), then 8, then the remaining 4 or 2.  The
// stage-major twiddle table is built with the same sequence.
OCS_HD constexpr int pow2_stage_radix(int n, int ns) {
    return ((n / ns) % 16 == 0 && n % 128 == 0) ? 16 : (((n / ns) % 8 == 0) ? 8 : n / ns);
}

// Power-of-two lengths: NVEC vectors of compile-time length N, T threads.  Butterfly b
// of a stage maps to vector b % NVEC and index b / NVEC (vector fastest), and vectors sit
// pow2_vstride(N, NVEC) slots apart, so that the 16 lanes of a half-warp always hit 16
// different 8-byte banks.  The first stage may read its inputs from a loader functor
// (ld(vec, i) -> float2) instead of shared memory and the last stage may hand its outputs
// to a storer functor (st(vec, i, value)) instead of writing them back: each saves one
// pass over shared memory and a barrier.  Middle stages work in place: every thread loads
// and transforms up to IT butterflies into registers, then, after a barrier, stores them.
// tw: the stage-major twiddle table, w^(r*j*N/(NS*R)) of a stage at [(r-1)*NS + j].
OCS_HD int pow2_vstride(int n, int nvec) {
    int v = n + (n >> 3) + 1;
    const int want = nvec >= 16 ? 0 : 16 / nvec;
    return v + ((want - (v & 15)) & 15);
}

struct NoLoad {
    OCS_D float2 operator()(int, int) const { return make_float2(0.f, 0.f); }
};
struct NoStore {
    OCS_D void operator()(int, int, float2) const {}
};

template <int R, int IT, int N, int NS, int NVEC, bool FIRST, bool LAST, class Ld, class St>
OCS_D void fft_stage_pow2(float2 *buf, int vstride, const float2 *tw, const Ld &ld, const St &st) {
    constexpr int nb = N / R;
    static_assert(nb % 8 == 0, "power-of-two stages need N/R to be a multiple of 8");
    constexpr int in_step = nb + nb / 8;                       // padded stride of the reads
    // padded offset of output r from output 0: the writes go to d + r*NS; with NS a multiple
    // of 8 that is r*(NS + NS/8) slots, with NS == 1 (d a multiple of 8) it is pad_idx(r)
    auto out_off = [](int r) { return (NS % 8 == 0) ? r * (NS + NS / 8) : r + (r >> 3); };
    static_assert(NS == 1 || NS % 8 == 0, "stage spans must be 1 or multiples of 8");
    if constexpr (FIRST && !LAST && NS == 1) {
        // first stage from a loader: every load of the thread's butterflies is issued
        // before the first transform (NS == 1: no twiddles)
        float2 v[IT][R];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int b = threadIdx.x + it * blockDim.x;
            if (b < nb * NVEC) {
                const int vec = b % NVEC, j = b / NVEC;
#pragma unroll
                for (int r = 0; r < R; ++r) v[it][r] = ld(vec, j + r * nb);
            }
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int b = threadIdx.x + it * blockDim.x;
            if (b < nb * NVEC) {
                const int vec = b % NVEC, j = b / NVEC;
                dft_inv<R>(v[it]);
                float2 *y = buf + vec * vstride + pad_idx(j * R);
#pragma unroll
                for (int r = 0; r < R; ++r) y[out_off(r)] = v[it][r];
            }
        }
        __syncthreads();
    } else if constexpr (FIRST || LAST) {
        // independent butterflies: nothing else in shared memory is read (FIRST) or
        // written (LAST) in this stage, so each result is written out immediately
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int b = threadIdx.x + it * blockDim.x;
            if (b < nb * NVEC) {
                const int vec = b % NVEC, j = b / NVEC;
                const int jm = j % NS;
                float2 v[R];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 a;
                    if constexpr (FIRST) a = ld(vec, j + r * nb);
                    else a = buf[vec * vstride + pad_idx(j) + r * in_step];
                    if (r > 0 && jm > 0) a = c_mul(a, tw[(r - 1) * NS + jm]);
                    v[r] = a;
                }
                dft_inv<R>(v);
                const int d = (j - jm) * R + jm;
                if constexpr (LAST) {
#pragma unroll
                    for (int r = 0; r < R; ++r) st(vec, d + r * NS, v[r]);
                } else {
                    float2 *y = buf + vec * vstride + pad_idx(d);
#pragma unroll
                    for (int r = 0; r < R; ++r) y[out_off(r)] = v[r];
                }
            }
        }
        if constexpr (!LAST) __syncthreads();
    } else {
        float2 v[IT][R];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int b = threadIdx.x + it * blockDim.x;
            if (b < nb * NVEC) {
                const int vec = b % NVEC, j = b / NVEC;
                const float2 *x = buf + vec * vstride + pad_idx(j);
                const int jm = j % NS;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 a = x[r * in_step];
                    if (r > 0 && jm > 0) a = c_mul(a, tw[(r - 1) * NS + jm]);
                    v[it][r] = a;
                }
                dft_inv<R>(v[it]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int b = threadIdx.x + it * blockDim.x;
            if (b < nb * NVEC) {
                const int vec = b % NVEC, j = b / NVEC;
                const int jm = j % NS;
                float2 *y = buf + vec * vstride + pad_idx((j - jm) * R + jm);
#pragma unroll
                for (int r = 0; r < R; ++r) y[out_off(r)] = v[it][r];
            }
        }
        __syncthreads();
    }
}

// The whole transform: the stages of pow2_stage_radix.  Without a loader
// the inputs are read from buf (and must be complete before the call); without a storer
// the results are left in buf (complete when the call returns).
template <int N, int NVEC, int T, bool HAS_LD, bool HAS_ST, int NS = 1, class Ld = NoLoad, class St = NoStore>
OCS_D void ifft_pow2(float2 *buf, int vstride, const float2 *tw, const Ld &ld = Ld(), const St &st = St()) {
    if constexpr (NS < N) {
        constexpr int REM = N / NS;
        constexpr int R = pow2_stage_radix(N, NS);
        constexpr int IT = ((N / R) * NVEC + T - 1) / T;
        constexpr bool first = HAS_LD && NS == 1;
        constexpr bool last = HAS_ST && NS * R == N;
        fft_stage_pow2<R, IT, N, NS, NVEC, first, last>(buf, vstride, tw, ld, st);
        ifft_pow2<N, NVEC, T, HAS_LD, HAS_ST, NS * R>(buf, vstride, tw + (R - 1) * NS, ld, st);
    }
}

// One out-of-place Stockham stage (any length, runtime radix R <= 8): src -> dst.
template <int R>
OCS_D void fft_stage_pp(const float2 *src, float2 *dst, int vstride, int nvec, int n, int ns,
                        const float2 *tw) {
    const int nb = n / R;
    const int tstep = n / (ns * R);
    for (int b = threadIdx.x; b < nb * nvec; b += blockDim.x) {
        const int vec = b / nb, j = b - vec * nb;
        const float2 *x = src + vec * vstride;
        float2 *y = dst + vec * vstride;
        const int jm = j % ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 a = x[pad_idx(j + r * nb)];
            if (r > 0 && jm > 0) a = c_mul(a, __ldg(&tw[r * jm * tstep]));
            v[r] = a;
        }
        dft_inv<R>(v);
        const int d = (j - jm) * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) y[pad_idx(d + r * ns)] = v[r];
    }
}

// Mixed-radix inverse FFT with a runtime plan, ping-ponging between a and b.  Returns the
// buffer that holds the result.
OCS_D float2 *ifft_generic(float2 *a, float2 *b, int vstride, int nvec, const FftPlan &plan) {
    int ns = 1;
    float2 *src = a, *dst = b;
    for (int s = 0; s < plan.nstages; ++s) {
        const int R = plan.radix[s];
        switch (R) {
            case 8: fft_stage_pp<8>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
            case 4: fft_stage_pp<4>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
            case 2: fft_stage_pp<2>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
            case 3: fft_stage_pp<3>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
            case 5: fft_stage_pp<5>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
            default: fft_stage_pp<7>(src, dst, vstride, nvec, plan.n, ns, plan.tw); break;
        }
        __syncthreads();
        float2 *t = src; src = dst; dst = t;
        ns *= R;
    }
    return src;
}

}  // namespace ocs
