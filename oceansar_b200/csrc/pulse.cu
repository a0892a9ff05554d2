// One radar pulse of the raw-data generator on sm_100a: the body of the azimuth loop of
// sar_raw (oceansar/radarsim/sar_raw_nompi.py:349-535) after the surface update, fused
// into one kernel per pulse so that no per-facet intermediate ever reaches HBM:
//
//   slant range of every facet (:366-369), Kodis specular field (:392-400),
//   Romeiser Bragg RCS refreshed every ocean_dt (:431-458, stored as sqrt(RCS) between
//   refreshes), Bragg phases + random sub-grid scatterers (:470-480), antenna pattern and
//   per-channel ATI / XTI phases (:485-495), and the range-profile accumulation
//   (range_profile.py:83-116) through the register-window engine of accum.cuh.
//
// Layout: a CTA owns BX consecutive ground-range columns (one per thread) and a strip of
// rows; each thread walks its column down the strip, so a warp reads 32 consecutive
// float32 of every field (coalesced) and its range bins drift slowly, keeping the
// register windows warm.  Per-row quantities (azimuth, antenna pattern, ATI phase) are
// computed once per CTA into shared memory.
//
// Scatterometer mode (MODE = kModeSca, the DopSCA generator, oceansar/dopscasim/dopsca_raw.py:
// 343-520): the columns are N_repeat_x range blocks side by side, each reading the same
// surface (field column = column mod field_nx) with its rows rolled by the integer azimuth
// shift (field row = (row + roll) mod ny); the scene is scaled by (sr0 / (sr0 + r))^2, the
// Bragg RCS is evaluated on every launch, the Bragg phase advances with the sub-pulse time
// cap_t, the range bins see the sub-pulse delay sr_bin_off, and the NRCS sums are kept per
// range block.
//
// SKIM mode (MODE & kModeSkim, the SKIM generator, oceansar/radarsim/skim_raw.py:465-689):
// sin_az = az / sr per facet (absolute slant range of the column), the two-way antenna
// pattern evaluated per facet, 10-tap pulse, and the facets of every ny_integ rows
// accumulated into their own output row (the two-scale Doppler's range-only profiles
// summed over ny_integ rows; ny_integ = ny gives the single-row form).
//
// Precision forms (template T):
//   double -- the drop-in: every operation in float64 in the reference's order; slant
//             range and the bin / LUT indices bit-identical to numpy.
//   float  -- mixed: slant range, bin / LUT indices and the 2 k0 r phase reduction in
//             float64, everything else (NRCS, scene, accumulation) in float32.
#include <cudaTypedefs.h>
#include <string.h>

#include <mutex>

#include "accum.cuh"
#include "batch.cuh"
#include "physics.cuh"

namespace ocs {

constexpr int kPulseCols = 128;     // columns (threads) per CTA
constexpr int kPulseRows = 64;      // rows per tile (single-scene launches)
constexpr int kPulseRowsMax = 128;  // largest rows per tile (shared row tables)
constexpr int kMaxCh = 8;
constexpr int kPulseNbw = 160;      // CTA shared bin window

// Kernel modes (bits): Kirchhoff specular, scatterometer (DopSCA), SKIM; SKIM combines with
// the Kirchhoff specular term (kModeSkim | kModeKa).
enum { kModeStd = 0, kModeKa = 1, kModeSca = 2, kModeSkim = 4 };
constexpr int kSkimTaps = 10;       // n_sinc_samples of the SKIM generator (skim_raw.py:164)
template <int MODE> __host__ __device__ constexpr int mode_taps() { return (MODE & kModeSkim) ? kSkimTaps : kSincTaps; }

struct PulseArgs {
    int nx, ny, npol, nch;
    int out0, nout;                         // outputs [out0, out0+nout) of npol*nch, o = pol*nch + ch
    const float *dx_f, *dy_f, *dz_f, *diffx, *diffy, *diffxx, *diffyy, *diffxy, *hmtf;
    const float *y;                         // [ny] float32 azimuth coordinates
    const double *sr_col, *sin_inc, *cos_inc, *tan_inc, *inc, *c_b;   // [nx]
    double inc_angle, sr0, gr0, k0, az_now, min_sr, binsize, inv_binsize, t_step;
    int any_xti;
    int az_step;
    long long tind;                         // int(t_now * prf)
    double ltx_over_l, lrx_over_l;          // antenna length / wavelength
    double b_ati[kMaxCh], b_xti[kMaxCh];
    int do_kodis, do_bragg, refresh, use_hmtf;
    KodisParams kodis;
    RomeiserParams rom;
    void *scat;                             // [npol][2][ny][nx] sqrt(RCS) (T)
    const double *s_m, *s_p;                // complex128 random-scatterer series
    const float *s_m32, *s_p32;             // complex64 copies (mixed form), or null
    int n_m, n_p;
    int tmod_m, tmod_p;                     // int(t_now * prf) mod n_m, n_p
    const int *ind0_m, *ind0_p;             // [ny][nx]
    const float *sinc;                      // [8*20 + 1]
    double *rowtab;                         // per-pulse row table, see pulse_rows_kernel
    void *raw;                              // [npol*nch][az_steps][rg_samp] complex T
    long long raw_out_stride, raw_row;      // elements between outputs, offset of this pulse row
    int nbins;
    double *nrcs_spec;                      // [az_steps]  sum |E_spec|^2
    double *nrcs_bragg;                     // [npol][az_steps] sum RCS (refresh pulses)
    int az_steps;
    int tile_rows;                          // rows per tile of a single-scene launch
    int spec_mode;                          // 0 Kodis, 1 Kirchhoff facet approach, 2 stationary phase
    const float *x_f;                       // [nx] facet x positions (Kirchhoff)
    KaParams ka;
    const void *lut;                        // Romeiser LUT [npol][2][naz][ndy][ndx] (T), or null
    int lut_naz, lut_ndy, lut_ndx;
    double lut_az0, lut_daz, lut_dy0, lut_ddy, lut_dx0, lut_ddx;
    int sca;                                // scatterometer mode (see the file comment)
    int fnx, roll;                          // field columns, azimuth roll of the field rows
    double sr_bin_off, cap_t;               // sub-pulse range delay, Bragg phase time
    int nblk, nrcs_row, nrcs_rows;          // range blocks; NRCS row of this call, rows in all
    int az_f32;                             // azimuth y - az_now rounded to float32 (see pulse_row)
    int skim, ny_integ, s_int;              // SKIM mode: output row per ny_integ facet rows
    int skim_az2, skim_rcm;                 // SKIM: az/2 sin_az in the phase range / in the bins only
    double atx, arx;                        // SKIM: antenna lengths / wavelength (tx, rx)
    int pt_mode, pt_x, pt_y;                // SKIM calibration target: 0 none, 1 floating, 2 fixed
    double pt_amp;
    long long lut_block;                    // scatterometer LUT: elements between block tables
};

// Kirchhoff specular term of one facet and polarisation code pc (0 = hh, 1 = vv),
// sar_raw_nompi.py:402-426: exp(-1j (2 k0 r)) (4 pi)^1.5 RCSKA.field(1, 1, ...).  Only the
// Kirchhoff instantiations of the pulse kernel (MODE = kModeKa) contain it.
OCS_D c128 ka_specular(const KaParams &kp, int pc, double srs, double x, double y, double st,
                                         double ct, double tt, double sp, double cp, float dz, float dx, float dy,
                                         float dxx, float dyy, float dxy) {
    const c128 e = ka_facet(kp, pc, pc, x, y, st, ct, tt, sp, cp, dz, dx, dy, dxx, dyy, dxy);
    const c128 ph = cexpi(-dmul(2.0 * kp.k0, srs));
    const double s15 = 44.54662397465366;                // (4 pi)^1.5
    return cmul128(cmulr(ph, s15), e);
}

// LUT mode of the Romeiser model (romeiser97.py:109-134): RCS of both Bragg lines of
// polarisation p at (azimuth index of the row, clamped slope indices of the facet).
// Indices round half to even from float64 differences and divisions, as numpy does.
template <typename T>
OCS_D void romeiser_lut(const PulseArgs &a, int az_ind, float diffx, float diffy, int p, T (&r)[2],
                        long long table = 0) {
    int iy = (int)rint(ddiv(dsub((double)diffy, a.lut_dy0), a.lut_ddy));
    int ix = (int)rint(ddiv(dsub((double)diffx, a.lut_dx0), a.lut_ddx));
    iy = iy > 0 ? (iy < a.lut_ndy ? iy : a.lut_ndy - 1) : 0;
    ix = ix > 0 ? (ix < a.lut_ndx ? ix : a.lut_ndx - 1) : 0;
    const T *lut = static_cast<const T *>(a.lut) + table;
    const long long plane = (long long)a.lut_naz * a.lut_ndy * a.lut_ndx;
    const long long off = ((long long)az_ind * a.lut_ndy + iy) * a.lut_ndx + ix;
    r[0] = lut[(2LL * p) * plane + off];
    r[1] = lut[(2LL * p + 1) * plane + off];
}

// Azimuth index of a row's ground-projected azimuth angle (negative: from the end, as numpy
// indexing takes it; out-of-table rows are rejected by the host before launch, and are
// clamped here so that no access leaves the table).
OCS_D int lut_az_index(const PulseArgs &a, double azp) {
    int i = (int)rint(ddiv(dsub(azp, a.lut_az0), a.lut_daz));
    if (i < 0) i += a.lut_naz;
    return i < 0 ? 0 : (i >= a.lut_naz ? a.lut_naz - 1 : i);
}

// Asynchronous global -> shared copies (cp.async): each thread copies the words it will
// read itself, so a cp.async.wait_group by that thread is all the ordering needed.
OCS_D void cp_async(void *dst, const void *src, int bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if (bytes == 4) asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
OCS_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> OCS_D void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Staging of the per-facet inputs in shared memory: stage_rows rows of every input array
// ([8] float32 fields, [4] sqrt(RCS) of type T, [2] int32 scatterer offsets, kPulseCols
// columns each) in a ring of stage_rows slots, and two slots of the
// gathered scatterer-series values (complex128 of both Bragg lines), filled one row ahead.
// Ring slots: the mixed form keeps two rows in flight while it processes one (four
// slots); the float64 form, limited to two CTAs per SM by its registers, one (three slots,
// measured faster there).
template <typename T> OCS_HD constexpr int stage_rows() { return sizeof(T) == 4 ? 4 : 3; }
template <typename T> OCS_HD constexpr size_t stage_slot_bytes() {
    return (8 * 4 + 4 * sizeof(T) + 2 * 4) * (size_t)kPulseCols;
}
template <typename T> OCS_HD constexpr size_t stage_bytes() {
    return stage_rows<T>() * stage_slot_bytes<T>() + 2 * 2 * 16 * (size_t)kPulseCols + 16;
}

template <typename T> struct Stage {
    unsigned char *base;          // 16-byte aligned
    OCS_D float *f(int slot, int k) const {
        return reinterpret_cast<float *>(base + slot * stage_slot_bytes<T>()) + k * kPulseCols + threadIdx.x;
    }
    OCS_D T *scat(int slot, int k) const {
        return reinterpret_cast<T *>(base + slot * stage_slot_bytes<T>() + 32 * kPulseCols) + k * kPulseCols +
               threadIdx.x;
    }
    OCS_D int *ind(int slot, int k) const {
        return reinterpret_cast<int *>(base + slot * stage_slot_bytes<T>() + (32 + 4 * sizeof(T)) * kPulseCols) +
               k * kPulseCols + threadIdx.x;
    }
    OCS_D double2 *gather(int g, int k) const {
        return reinterpret_cast<double2 *>(base + stage_rows<T>() * stage_slot_bytes<T>()) + (2 * g + k) * kPulseCols +
               threadIdx.x;
    }
};

// Inputs of one facet.
template <typename T> struct FacetIn {
    float dx, dy, dz, diffx, diffy, diffxx, diffyy, diffxy;
    T scat[2][2];
    // start the copies of facet idx's inputs into stage slot `slot`
    // (fidx: index into the surface fields; idx: into the per-facet scatterer arrays)
    template <typename A>
    static OCS_D void issue(const A &a, const Stage<T> &st, int slot, long long idx, long long npix,
                            const T *scat_buf, bool load_scat, long long fidx) {
        cp_async(st.f(slot, 0), a.dx_f + fidx, 4);
        cp_async(st.f(slot, 1), a.dy_f + fidx, 4);
        cp_async(st.f(slot, 2), a.dz_f + fidx, 4);
        if (a.diffx) {
            cp_async(st.f(slot, 3), a.diffx + fidx, 4);
            cp_async(st.f(slot, 4), a.diffy + fidx, 4);
        }
        if (a.do_kodis) {
            cp_async(st.f(slot, 5), a.diffxx + fidx, 4);
            cp_async(st.f(slot, 6), a.diffyy + fidx, 4);
            cp_async(st.f(slot, 7), a.diffxy + fidx, 4);
        }
        if (a.do_bragg) {
            cp_async(st.ind(slot, 0), a.ind0_m + idx, 4);
            cp_async(st.ind(slot, 1), a.ind0_p + idx, 4);
        }
        if (load_scat) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < 2 * a.npol) cp_async(st.scat(slot, k), scat_buf + k * npix + idx, sizeof(T));
        }
    }
    // start the gathers of the scatterer-series values of the facet staged in `slot`
    template <typename A>
    static OCS_D void issue_gather(const A &a, const Stage<T> &st, int slot, int g) {
        int i0 = *st.ind(slot, 0) + a.tmod_m;
        i0 = i0 >= a.n_m ? i0 - a.n_m : i0;
        int i1 = *st.ind(slot, 1) + a.tmod_p;
        i1 = i1 >= a.n_p ? i1 - a.n_p : i1;
        if (sizeof(T) == 4 && a.s_m32) {
            cp_async(st.gather(g, 0), a.s_m32 + 2 * (long long)i0, 8);
            cp_async(st.gather(g, 1), a.s_p32 + 2 * (long long)i1, 8);
        } else {
            cp_async(st.gather(g, 0), a.s_m + 2 * (long long)i0, 16);
            cp_async(st.gather(g, 1), a.s_p + 2 * (long long)i1, 16);
        }
    }
    template <typename A>
    OCS_D void read(const A &a, const Stage<T> &st, int slot, bool load_scat) {
        dx = *st.f(slot, 0);
        dy = *st.f(slot, 1);
        dz = *st.f(slot, 2);
        if (a.diffx) { diffx = *st.f(slot, 3); diffy = *st.f(slot, 4); }
        if (a.do_kodis) { diffxx = *st.f(slot, 5); diffyy = *st.f(slot, 6); diffxy = *st.f(slot, 7); }
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            if (load_scat && p < a.npol) {
                scat[p][0] = *st.scat(slot, 2 * p);
                scat[p][1] = *st.scat(slot, 2 * p + 1);
            } else {
                scat[p][0] = (T)0;
                scat[p][1] = (T)0;
            }
        }
    }
};

template <typename T> OCS_D cplx<T> cexp_phase(double ph);
template <> OCS_D cplx<double> cexp_phase<double>(double ph) { return cexpi(ph); }
template <> OCS_D cplx<float> cexp_phase<float>(double ph) {
    float s, c;
    __sincosf((float)reduce_2pi(ph), &s, &c);
    return {c, s};
}

// Block-wide sum of a double; thread 0 adds it to *dst.
OCS_D void block_atomic_sum(double v, double *dst, double *sred) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sred[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += sred[i];
        if (s != 0.0) atomicAdd(dst, s);
    }
}

// Per-pulse row table (sar_raw_nompi.py:353-363, 485-493): for every facet row y,
// rowtab[q*ny + y] holds az, sin_az = az/sr0, the ground-projected azimuth angle and its
// cos / sin (q = 0..4), then rowtab[5*ny + 2*(y*nch + c)] the complex antenna-pattern x
// ATI-phase factor of channel c.  float64, computed once per pulse for all tiles.
OCS_D void pulse_row(const PulseArgs &a, double az_now, int y) {
    // the scatterometer's azimuth residual is float32 when the reference computes it from
    // a float32 grid step (numpy promotion), and then y - residual is a float32 difference
    const double az = a.az_f32 ? (double)__fsub_rn(a.y[y], (float)az_now) : dsub((double)a.y[y], az_now);
    const double sin_az = ddiv(az, a.sr0);
    const double azp = asin(az / a.gr0);
    a.rowtab[y] = az;
    a.rowtab[(long long)a.ny + y] = sin_az;
    a.rowtab[2LL * a.ny + y] = azp;
    a.rowtab[3LL * a.ny + y] = cos(azp);
    a.rowtab[4LL * a.ny + y] = sin(azp);
    const double bp = np_sinc(a.ltx_over_l * sin_az) * np_sinc(a.lrx_over_l * sin_az);
    double *fac = a.rowtab + 5LL * a.ny + 2LL * y * a.nch;
    for (int c = 0; c < a.nch; ++c) {
        const c128 ati = cexpi((-a.k0 * a.b_ati[c]) * sin_az);
        fac[2 * c] = bp * ati.re;
        fac[2 * c + 1] = bp * ati.im;
    }
}

__global__ void pulse_rows_kernel(const __grid_constant__ PulseArgs a) {
    for (int y = blockIdx.x * blockDim.x + threadIdx.x; y < a.ny; y += gridDim.x * blockDim.x)
        pulse_row(a, a.az_now, y);
}

// Shared memory of the pulse kernel: pre-shifted weight table, CTA bin window, the tile's
// rows of the per-pulse row table ([5][RCAP] float64 + [RCAP][nch] complex, RCAP = the
// largest tile height of the launch), and the block-reduction scratch.
template <typename T> struct PulseSmem {
    T *wtab, *bins;
    double *r_az;
    cplx<T> *r_fac;
    double *sred;
    Stage<T> stage;
};

template <typename T, int NOUT, int S, int RCAP>
OCS_HD constexpr size_t pulse_smem_bytes(int nch) {
    return (size_t)wtab_len<T, S>(kSincTaps, kSincOvs) * sizeof(T) + (size_t)NOUT * kPulseNbw * 2 * sizeof(T) +
           5 * RCAP * sizeof(double) + (size_t)RCAP * nch * sizeof(cplx<T>) + 32 * sizeof(double) +
           stage_bytes<T>();
}

template <typename T, int NOUT, int S, int RCAP>
OCS_D PulseSmem<T> pulse_smem(unsigned char *smem, int nch) {
    PulseSmem<T> sm;
    sm.wtab = reinterpret_cast<T *>(smem);
    sm.bins = sm.wtab + wtab_len<T, S>(kSincTaps, kSincOvs);             // [NOUT][nbw][2]
    sm.r_az = reinterpret_cast<double *>(sm.bins + NOUT * kPulseNbw * 2);
    sm.r_fac = reinterpret_cast<cplx<T> *>(sm.r_az + 5 * RCAP);            // [rows][nch]
    sm.sred = reinterpret_cast<double *>(sm.r_fac + RCAP * nch);
    const size_t st = reinterpret_cast<size_t>(sm.sred + 32);
    sm.stage.base = reinterpret_cast<unsigned char *>((st + 15) & ~(size_t)15);
    return sm;
}

// One tile of kPulseCols columns x tile_rows rows: NRCS, scene and accumulation of every
// facet into this pulse's raw rows; the tile's NRCS sums are added to spec_sum and
// bragg_sum.
template <typename T, int NOUT, int S, int RCAP, int MODE = kModeStd>
OCS_D void pulse_tile(const PulseArgs &a, int tile, int tile_rows, const PulseSmem<T> &sm, double &spec_sum,
                      double (&bragg_sum)[2]) {
    const int tiles_x = (a.nx + kPulseCols - 1) / kPulseCols;
    const int x = (tile % tiles_x) * kPulseCols + threadIdx.x;
    const int y0 = (tile / tiles_x) * tile_rows;
    const int nrows = min(tile_rows, a.ny - y0);
    __syncthreads();                    // previous tile's bins and row tables are consumed
    // this tile's rows of the per-pulse row table (pulse_rows_kernel)
    for (int i = threadIdx.x; i < nrows * 5; i += blockDim.x) {
        const int q = i / nrows, k = i - q * nrows;
        sm.r_az[q * RCAP + k] = a.rowtab[(long long)q * a.ny + y0 + k];
    }
    {
        const double *fac = a.rowtab + 5LL * a.ny + 2LL * y0 * a.nch;
        for (int i = threadIdx.x; i < nrows * a.nch; i += blockDim.x)
            sm.r_fac[i] = {(T)fac[2 * i], (T)fac[2 * i + 1]};
    }

    CtaBins<T, NOUT> cb;
    cb.acc = sm.bins;
    cb.nbw = kPulseNbw;
    cb.nout = a.nout;
    cb.nbins = a.nbins;
    cb.out = reinterpret_cast<T *>(a.raw) + 2 * ((long long)a.out0 * a.raw_out_stride + a.raw_row);
    if constexpr ((MODE & kModeSkim) != 0) cb.out += 2 * (long long)(y0 / a.ny_integ) * a.nbins;
    cb.out_stride = a.raw_out_stride;
    {
        // window base: bin of this CTA's first column at its first row, undisplaced
        const int xc = min((tile % tiles_x) * kPulseCols, a.nx - 1);
        const double az = (double)a.y[y0] - a.az_now;
        const double srg = a.sr_col[xc] + az * 0.5 * (az / a.sr0) + a.sr_bin_off;
        cb.cta_base = (int)floor((srg - a.min_sr) / a.binsize) - 24;
    }
    cb.zero();
    __syncthreads();

    BinWindow<T, S, NOUT> win;
    win.reset();
    if (x < a.nx) {
        const double sr_c = a.sr_col[x], sin_i = a.sin_inc[x], cos_i = a.cos_inc[x];
        const double inc_c = a.inc[x];
        const double dinc0 = inc_c - a.inc_angle;
        const double tan_i = a.do_kodis ? a.tan_inc[x] : 0.0;
        double cap = 0.0;
        if (a.do_bragg) {
            if constexpr ((MODE & kModeSca)) cap = dmul(dmul(2.0 * a.k0, a.c_b[x]), a.cap_t);
            else cap = ((2.0 * a.k0) * a.t_step) * a.c_b[x] * (double)(a.az_step + 1);
        }
        const float cap_r = (float)reduce_2pi(cap);
        const double two_k0 = 2.0 * a.k0;
        const long long npix = (long long)a.nx * a.ny;
        T *scat = reinterpret_cast<T *>(a.scat);
        const bool load_scat = a.do_bragg && !a.refresh;
        // software pipeline through shared memory: the inputs of the next rows and
        // the scatterer-series gathers of row i + 1 are in flight while row i is processed
        const Stage<T> &st = sm.stage;
        const long long idx0 = (long long)y0 * a.nx + x;
        // outputs of this pass, 5 bits each: channel (bits 0-2), polarisation (bit 3) and
        // whether the channel has an XTI phase (bit 4)
        unsigned outs = 0;
#pragma unroll
        for (int k = 0; k < NOUT; ++k) {
            const int o = a.out0 + k;
            const int p = o / a.nch, c = o - p * a.nch;
            const bool xti = k < a.nout && a.b_xti[c] != 0.0;
            outs |= (unsigned)(c | (p << 3) | (xti ? 16 : 0)) << (5 * k);
        }
        // indices of tile row r: per-facet arrays (ridx) and surface fields (fidx); the
        // scatterometer mode reads the fields of the rolled row and the column mod fnx
        int fx = x;
        if constexpr ((MODE & kModeSca)) fx = x % a.fnx;
        auto row_index = [&](int r, long long &ridx, long long &fidx) {
            if constexpr ((MODE & kModeSca)) {
                int fr = y0 + r + a.roll;
                fr = fr >= a.ny ? fr - a.ny : fr;
                ridx = (long long)fr * a.nx + x;
                fidx = (long long)fr * a.fnx + fx;
            } else {
                ridx = idx0 + (long long)r * a.nx;
                fidx = ridx;
            }
        };
        auto issue_row = [&](int r, int slot) {
            if (r < nrows) {
                long long ridx, fidx;
                row_index(r, ridx, fidx);
                FacetIn<T>::issue(a, st, slot, ridx, npix, scat, load_scat, fidx);
            }
            cp_async_commit();
        };
        FacetIn<T> cur;
        if constexpr (stage_rows<T>() == 4) {
            // Commit order: rows 0, 1; gathers of row 0; row 2; then per row i the gathers of
            // row i + 1 and row i + 3.  Waiting for all groups but the newest at the top of
            // row i completes rows <= i + 1 and the gathers of row i and leaves row i + 2 in
            // flight, so two rows of inputs are on their way while a row is processed.
            issue_row(0, 0);
            issue_row(1, 1);
            cp_async_wait<1>();
            if (a.do_bragg) FacetIn<T>::issue_gather(a, st, 0, 0);
            cp_async_commit();
            issue_row(2, 2);
        } else {
            // rows 0, 1, then gathers of row 0; per row i: row i + 2, gathers of row i + 1
            issue_row(0, 0);
            issue_row(1, 1);
            cp_async_wait<1>();
            if (a.do_bragg) FacetIn<T>::issue_gather(a, st, 0, 0);
            cp_async_commit();
        }
        int slot_i = 0;
        for (int i = 0; i < nrows; ++i) {
            const long long idx = idx0 + (long long)i * a.nx;
            int slot_n;
            if constexpr (stage_rows<T>() == 4) {
                slot_n = (i + 1) & 3;
                cp_async_wait<1>();             // rows <= i + 1 and the gathers of row i have landed
                if (a.do_bragg && i + 1 < nrows) FacetIn<T>::issue_gather(a, st, slot_n, (i + 1) & 1);
                cp_async_commit();
                issue_row(i + 3, (i + 3) & 3);  // into the slot of row i - 1
            } else {
                slot_n = slot_i == 2 ? 0 : slot_i + 1;
                issue_row(i + 2, slot_i == 0 ? 2 : slot_i - 1);
                cp_async_wait<1>();             // rows <= i + 1 and the gathers of row i have landed
                if (a.do_bragg && i + 1 < nrows) FacetIn<T>::issue_gather(a, st, slot_n, (i + 1) & 1);
                cp_async_commit();
            }
            cur.read(a, st, slot_i, load_scat);
            slot_i = slot_n;
            // SKIM calibration target: a fixed one sits at zero displacement (skim_raw.py:490-493)
            const bool pt_here = (MODE & kModeSkim) && a.pt_mode != 0 && y0 + i == a.pt_y && x == a.pt_x;
            if (pt_here && a.pt_mode == 2) {
                cur.dx = 0.f;
                cur.dy = 0.f;
                cur.dz = 0.f;
            }
            const double az = sm.r_az[i];
            // SKIM: sin_az = az / sr of this facet's column (skim_raw.py:486)
            const double sin_az = (MODE & kModeSkim) ? ddiv(az, sr_c) : sm.r_az[RCAP + i];
            // slant range: sr - cos_inc*Dz + az/2*sin_az + Dx*sin_inc + Dy*sin_az, float64,
            // left to right, no fused multiply-adds (bit-identical with numpy); the SKIM
            // two-scale form leaves az/2*sin_az out of the phase range (skim_raw.py:494-505)
            double srs = dsub(sr_c, dmul(cos_i, (double)cur.dz));
            if (!(MODE & kModeSkim) || a.skim_az2) srs = dadd(srs, dmul(az * 0.5, sin_az));
            srs = dadd(srs, dmul((double)cur.dx, sin_i));
            srs = dadd(srs, dmul((double)cur.dy, sin_az));
            int bin_d, lut;
            {
                // the scatterometer's sub-pulses arrive later by sr_bin_off; the SKIM
                // two-scale form with rcm adds az/2*sin_az to the bins only
                double srb = ((MODE & kModeSca)) ? dadd(srs, a.sr_bin_off) : srs;
                if ((MODE & kModeSkim) && a.skim_rcm) srb = dadd(srs, dmul(az * 0.5, sin_az));
                if (sizeof(T) == 8) bin_and_lut(srb, a.min_sr, a.binsize, kSincOvs, bin_d, lut);
                else bin_and_lut_fast(srb, a.min_sr, a.inv_binsize, kSincOvs, bin_d, lut);
            }
            // two-way spreading of the scatterometer scene, (sr0 / (sr0 + r))^2
            T rscale = (T)1;
            if constexpr ((MODE & kModeSca)) {
                const double q = ddiv(a.sr0, dadd(a.sr0, srs));
                rscale = (T)dmul(q, q);
            }

            cplx<T> scene[2] = {{(T)0, (T)0}, {(T)0, (T)0}};      // per polarisation
            if constexpr ((MODE & kModeKa) != 0) {
                c128 last = {0.0, 0.0};
                for (int p = 0; p < a.npol; ++p) {
                    const int pc = a.rom.pol == POL_DP ? p : (a.rom.pol == POL_HH ? 0 : 1);
                    last = ka_specular(a.ka, pc, srs, (double)a.x_f[fx], (double)a.y[y0 + i], sin_i, cos_i, tan_i,
                                       sm.r_az[4 * RCAP + i], sm.r_az[3 * RCAP + i], cur.dz, cur.diffx, cur.diffy,
                                       cur.diffxx, cur.diffyy, cur.diffxy);
                    scene[p] = {(T)last.re, (T)last.im};
                    // the scatterometer scales the field by the two-way spreading
                    if constexpr ((MODE & kModeSca) != 0) scene[p] = {scene[p].re * rscale, scene[p].im * rscale};
                }
                spec_sum += last.re * last.re + last.im * last.im;
            } else if (a.do_kodis) {
                const cplx<T> e = kodis_facet<T>(a.kodis, srs, sin_i, cos_i, tan_i, sm.r_az[3 * RCAP + i], sm.r_az[4 * RCAP + i],
                                                 cur.diffx, cur.diffy, cur.diffxx, cur.diffyy, cur.diffxy);
                const T s4 = (T)3.5449077018110318;                 // sqrt(4 pi)
                const cplx<T> es = {e.re * s4, e.im * s4};
                spec_sum += (double)es.re * es.re + (double)es.im * es.im;
                if constexpr ((MODE & kModeSca)) {
                    scene[0] = {es.re * rscale, es.im * rscale};
                    scene[1] = scene[0];
                } else {
                    scene[0] = es;
                    scene[1] = es;
                }
            }
            if (a.do_bragg) {
                T sc[2][2];                                            // [pol][line]
                if (a.refresh) {
                    T hh[2], vv[2];
                    if (a.lut) {
                        // the table holds the model's output polarisation(s) in output order
                        const int ai = lut_az_index(a, sm.r_az[2 * RCAP + i]);
                        // the scatterometer's range blocks each have their own table
                        const long long tb = ((MODE & kModeSca)) ? (long long)(x / a.fnx) * a.lut_block : 0;
                        T r0[2], r1[2];
                        romeiser_lut<T>(a, ai, cur.diffx, cur.diffy, 0, r0, tb);
                        if (a.npol == 2) romeiser_lut<T>(a, ai, cur.diffx, cur.diffy, 1, r1, tb);
                        else { r1[0] = r0[0]; r1[1] = r0[1]; }
                        const bool vv_first = a.rom.pol == POL_VV;
                        hh[0] = vv_first ? r1[0] : r0[0]; hh[1] = vv_first ? r1[1] : r0[1];
                        vv[0] = vv_first ? r0[0] : r1[0]; vv[1] = vv_first ? r0[1] : r1[1];
                    } else {
                        romeiser_facet<T>(a.rom, (T)inc_c, (T)sm.r_az[2 * RCAP + i], (T)sm.r_az[3 * RCAP + i],
                                          (T)sm.r_az[4 * RCAP + i], (T)cur.diffx, (T)cur.diffy, hh, vv);
                    }
                    if (a.use_hmtf) {
                        float hm;
                        if constexpr ((MODE & kModeSca)) {
                            // the scatterometer generator weights by 1 + hMTF of the rolled
                            // row, unclipped (its clipping writes land in the unrolled surface,
                            // dopsca_raw.py:463-472)
                            long long ridx_h, fidx_h;
                            row_index(i, ridx_h, fidx_h);
                            hm = a.hmtf[fidx_h];
                        } else {
                            hm = a.hmtf[idx];
                            hm = hm < -1.f ? -1.f : hm;
                        }
                        const T f = (T)(1.f + hm);
                        hh[0] *= f; hh[1] *= f; vv[0] *= f; vv[1] *= f;
                    }
#pragma unroll
                    for (int p = 0; p < 2; ++p) {
                        if (p < a.npol) {
                            const bool use_vv = a.rom.pol == POL_VV || (a.rom.pol == POL_DP && p == 1);
                            const T r0 = use_vv ? vv[0] : hh[0], r1 = use_vv ? vv[1] : hh[1];
                            bragg_sum[p] += (double)r0 + (double)r1;
                            sc[p][0] = tsqrt(r0);
                            sc[p][1] = tsqrt(r1);
                            if (!(MODE & kModeSca) && a.out0 == 0) {   // one output group stores the RCS
                                scat[(2 * p) * npix + idx] = sc[p][0];
                                scat[(2 * p + 1) * npix + idx] = sc[p][1];
                            }
                        }
                    }
                } else {
#pragma unroll
                    for (int p = 0; p < 2; ++p) { sc[p][0] = cur.scat[p][0]; sc[p][1] = cur.scat[p][1]; }
                }
                // Bragg phases: -2 k0 r -/+ 2 k0 t_step c_b (az_step + 1)
                cplx<T> e0, e1;
                if (sizeof(T) == 8) {
                    const double surf = (-two_k0) * srs;
                    e0 = cexp_phase<T>(surf - cap);
                    e1 = cexp_phase<T>(surf + cap);
                } else {
                    const float rs = (float)reduce_2pi((-two_k0) * srs);
                    float s0, c0, s1, c1;
                    __sincosf(rs - cap_r, &s0, &c0);
                    __sincosf(rs + cap_r, &s1, &c1);
                    e0 = {(T)c0, (T)s0};
                    e1 = {(T)c1, (T)s1};
                }
                cplx<T> sm, sp;
                if (sizeof(T) == 4 && a.s_m32) {
                    const float2 smf = *reinterpret_cast<const float2 *>(st.gather(i & 1, 0));
                    const float2 spf = *reinterpret_cast<const float2 *>(st.gather(i & 1, 1));
                    sm = {(T)smf.x, (T)smf.y};
                    sp = {(T)spf.x, (T)spf.y};
                } else {
                    const double2 smd = *st.gather(i & 1, 0);
                    const double2 spd = *st.gather(i & 1, 1);
                    sm = {(T)smd.x, (T)smd.y};
                    sp = {(T)spd.x, (T)spd.y};
                }
#pragma unroll
                for (int p = 0; p < 2; ++p) {
                    if (p < a.npol) {
                        const cplx<T> l0 = cmul(cplx<T>{sc[p][0] * e0.re, sc[p][0] * e0.im}, sm);
                        const cplx<T> l1 = cmul(cplx<T>{sc[p][1] * e1.re, sc[p][1] * e1.im}, sp);
                        cplx<T> lb = cadd(l0, l1);
                        if constexpr ((MODE & kModeSca)) lb = {lb.re * rscale, lb.im * rscale};
                        scene[p] = cadd(scene[p], lb);
                    }
                }
            }
            if (pt_here) {
                // the target replaces the facet's scene value: pt_amp exp(-2 i k0 r)
                // (skim_raw.py:608-615), float64 like the reference's complex128 scene
                double ps, pc;
                sincos((-two_k0) * srs, &ps, &pc);
                for (int p = 0; p < a.npol; ++p) scene[p] = {(T)(a.pt_amp * pc), (T)(a.pt_amp * ps)};
            }
            // channels of this pass: antenna pattern x ATI phase (per row) x XTI phase
            cplx<T> coef[NOUT];
            double wave_dinc = 0.0;
            if (a.any_xti) wave_dinc = ((double)cur.dz * sin_i + (double)cur.dx * sin_i) / a.sr0;
            T bp_f = (T)1;
            if constexpr ((MODE & kModeSkim) != 0) {
                // two-way antenna pattern of this facet, power units for both the transmit
                // and the receive pattern (antenna.py:28-42 passes its field flag to the
                // positional catch-all of sinc_bp)
                T tx, rx;
                if constexpr (sizeof(T) == 8) {
                    tx = np_sinc(a.atx * sin_az);
                    rx = np_sinc(a.arx * sin_az);
                } else {
                    tx = np_sinc((float)(a.atx * sin_az));
                    rx = np_sinc((float)(a.arx * sin_az));
                }
                bp_f = (tx * tx) * (rx * rx);
            }
#pragma unroll
            for (int k = 0; k < NOUT; ++k) {
                if (k < a.nout) {
                    const unsigned ok = outs >> (5 * k);
                    const int c = ok & 7;
                    cplx<T> v;
                    if constexpr ((MODE & kModeSkim) != 0) {
                        const cplx<T> sc = (ok & 8) ? scene[1] : scene[0];
                        v = {sc.re * bp_f, sc.im * bp_f};
                    } else {
                        v = cmul((ok & 8) ? scene[1] : scene[0], sm.r_fac[i * a.nch + c]);
                    }
                    if (ok & 16) {
                        const double ph = (-a.k0 * a.b_xti[c]) * (dinc0 + wave_dinc);
                        v = cmul(v, cexp_phase<T>(ph));
                    }
                    coef[k] = v;
                } else {
                    coef[k] = {(T)0, (T)0};
                }
            }
            if (bin_d > -(1 << 29))
                win.add(bin_d - mode_taps<MODE>() / 2, lut, coef, sm.wtab, a.sinc, mode_taps<MODE>(), kSincOvs, cb);
        }
        cp_async_wait<0>();
    }
    if constexpr ((MODE & kModeSca)) {
        // the scatterometer's NRCS sums are kept per range block: each column adds its
        // tile's sums to its block
        if (x < a.nx) {
            const long long blk = x / a.fnx;
            if (a.do_kodis && spec_sum != 0.0) atomicAdd(&a.nrcs_spec[(long long)a.nrcs_row * a.nblk + blk], spec_sum);
            if (a.do_bragg)
                for (int p = 0; p < a.npol; ++p)
                    if (bragg_sum[p] != 0.0)
                        atomicAdd(&a.nrcs_bragg[((long long)p * a.nrcs_rows + a.nrcs_row) * a.nblk + blk], bragg_sum[p]);
        }
        spec_sum = 0.0;
        bragg_sum[0] = bragg_sum[1] = 0.0;
    }
    win.flush(cb);
    __syncthreads();
    cb.flush_to_global();
}

// NRCS bookkeeping of a CTA (only the first output group accumulates it).
template <typename T>
OCS_D void pulse_nrcs(const PulseArgs &a, const PulseSmem<T> &sm, double spec_sum, const double (&bragg_sum)[2]) {
    if (a.out0 == 0) {
        if (a.do_kodis) block_atomic_sum(spec_sum, &a.nrcs_spec[a.az_step], sm.sred);
        if (a.do_bragg && a.refresh)
            for (int p = 0; p < a.npol; ++p)
                block_atomic_sum(bragg_sum[p], &a.nrcs_bragg[(long long)p * a.az_steps + a.az_step], sm.sred);
    }
}

template <typename T, int NOUT, int S, int MODE>
__global__ void __launch_bounds__(kPulseCols, (sizeof(T) == 4 && NOUT < 4) ? 4 : 2)
pulse_kernel(const __grid_constant__ PulseArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const PulseSmem<T> sm = pulse_smem<T, NOUT, S, kPulseRows>(smem, a.nch);
    build_wtab<T, S>(sm.wtab, a.sinc, mode_taps<MODE>(), kSincOvs);
    const int tiles = ((a.nx + kPulseCols - 1) / kPulseCols) * ((a.ny + a.tile_rows - 1) / a.tile_rows);
    double spec_sum = 0.0, bragg_sum[2] = {0.0, 0.0};
    // persistent CTAs: each walks tiles of kPulseCols columns x tile_rows rows
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x)
        pulse_tile<T, NOUT, S, kPulseRows, MODE>(a, tile, a.tile_rows, sm, spec_sum, bragg_sum);
    pulse_nrcs<T>(a, sm, spec_sum, bragg_sum);
}

}  // namespace ocs

#include "pulse_mixed.cuh"

namespace ocs {

// ---------------------------------------------------------------------------------------
// Scene batch (batch.cuh).  Output groups: a slot's npol*nch outputs are taken G at a time
// (G = 4 in the mixed form, 2 in FP64); a group of w outputs runs in the kernel of width
// class 1 (w = 1), 2 (w = 2) or 4 (w = 3, 4).  On refresh pulses every group evaluates the
// Romeiser model and only the first group stores sqrt(RCS), so groups need no ordering.
OCS_HD constexpr int width_class(int w) { return w <= 1 ? 1 : (w == 2 ? 2 : 4); }

// Number of groups of width class K among nout outputs; out0 / width of the j-th one.
OCS_D int groups_of_class(int nout, int G, int K, int j, int &out0, int &width) {
    int n = 0;
    for (int o = 0; o < nout; o += G) {
        const int w = nout - o < G ? nout - o : G;
        if (width_class(w) == K) {
            if (n == j) { out0 = o; width = w; }
            ++n;
        }
    }
    return n;
}

OCS_D int slot_pulse_tiles(const SlotState &g) {
    return ((g.nx + kPulseCols - 1) / kPulseCols) * ((g.ny + g.tile_rows - 1) / g.tile_rows);
}

template <bool MIXED>
__global__ void batch_pulse_rows_kernel(const __grid_constant__ BatchRef b) {
    __shared__ int pref[kMaxSlots + 1];
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        return slot_live(g) ? (g.ny + (int)blockDim.x - 1) / (int)blockDim.x : 0;
    });
    for (int item = blockIdx.x; item < total; item += gridDim.x) {
        const int s = find_slot(pref, b.nslots, item);
        const SlotState &g = b.slots[s];
        const PulseArgs &a = *static_cast<const PulseArgs *>(g.pargs);
        const int y = (item - pref[s]) * blockDim.x + threadIdx.x;
        if (y < a.ny) {
            // Kirchhoff slots run the float64-range kernel, which reads the float64 table only
            if (MIXED && g.kind == kSlotStd) mix_row(a, g.aznow_tab[g.counter], y);
            else pulse_row(a, g.aznow_tab[g.counter], y);
        }
    }
}

// One launch covers every live slot's groups of width class NOUT among the slots of its
// pulse-kernel class (MODE = kModeStd: Kodis / Bragg slots, kModeKa: Kirchhoff slots); the
// host sizes the grid for all slots in use and each CTA takes one (slot, group, tile) item.
template <typename T, int NOUT, int S, int MODE = kModeStd>
__global__ void __launch_bounds__(kPulseCols, (sizeof(T) == 4 && NOUT < 4) ? 4 : 2)
batch_pulse_kernel(const __grid_constant__ BatchRef b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ PulseArgs pa;
    __shared__ int pref[kMaxSlots + 1];
    constexpr int G = sizeof(T) == 4 ? 4 : 2;
    constexpr int kind = (MODE & kModeKa) ? kSlotKa : kSlotStd;
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        int o, w;
        return (slot_live(g) && g.kind == kind) ? groups_of_class(g.nout, G, NOUT, -1, o, w) * slot_pulse_tiles(g) : 0;
    });
    const int item = blockIdx.x;
    if (item >= total) return;
    const int s = find_slot(pref, b.nslots, item);
    const SlotState &g = b.slots[s];
    const int tiles = slot_pulse_tiles(g);
    const int j = item - pref[s];
    const int grp = j / tiles, tile = j - grp * tiles;
    {
        const int *src = static_cast<const int *>(g.pargs);
        int *dst = reinterpret_cast<int *>(&pa);
        for (int i = threadIdx.x; i < (int)(sizeof(PulseArgs) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int c = g.counter;
        int o = 0, w = 0;
        groups_of_class(g.nout, G, NOUT, grp, o, w);
        pa.out0 = o;
        pa.nout = w;
        pa.az_step = c;
        pa.az_now = g.aznow_tab[c];
        pa.refresh = (g.flags_tab[c] & kFlagRefresh) ? 1 : 0;
        pa.tmod_m = g.tmod_tab[2 * c];
        pa.tmod_p = g.tmod_tab[2 * c + 1];
        pa.raw_row = (long long)c * pa.nbins;
    }
    __syncthreads();
    const PulseSmem<T> sm = pulse_smem<T, NOUT, S, kPulseRowsMax>(smem, kMaxCh);
    build_wtab<T, S>(sm.wtab, pa.sinc, kSincTaps, kSincOvs);
    double spec_sum = 0.0, bragg_sum[2] = {0.0, 0.0};
    pulse_tile<T, NOUT, S, kPulseRowsMax, MODE>(pa, tile, g.tile_rows, sm, spec_sum, bragg_sum);
    pulse_nrcs<T>(pa, sm, spec_sum, bragg_sum);
}

// The mixed form of the batch: every slot's scene passes pulse_split_ok (checked when the
// slot is set) and its tile runs the split-range kernel's tile (mix_tile); the raw rows
// take the CTA's compensated bins through plain float32 atomics (no compensation row).
template <int NOUT>
__global__ void __launch_bounds__(kMixCols, NOUT < 4 ? 3 : 2)
batch_pulse_mixed_kernel(const __grid_constant__ BatchRef b) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ PulseArgs pa;
    __shared__ int pref[kMaxSlots + 1];
    constexpr int G = 4;
    const int total = scan_slots(b, pref, [](const SlotState &g) {
        int o, w;
        return (slot_live(g) && g.kind == kSlotStd) ? groups_of_class(g.nout, G, NOUT, -1, o, w) * slot_pulse_tiles(g)
                                                    : 0;
    });
    const int item = blockIdx.x;
    if (item >= total) return;
    const int s = find_slot(pref, b.nslots, item);
    const SlotState &g = b.slots[s];
    const int tiles = slot_pulse_tiles(g);
    const int j = item - pref[s];
    const int grp = j / tiles, tile = j - grp * tiles;
    {
        const int *src = static_cast<const int *>(g.pargs);
        int *dst = reinterpret_cast<int *>(&pa);
        for (int i = threadIdx.x; i < (int)(sizeof(PulseArgs) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int c = g.counter;
        int o = 0, w = 0;
        groups_of_class(g.nout, G, NOUT, grp, o, w);
        pa.out0 = o;
        pa.nout = w;
        pa.az_step = c;
        pa.az_now = g.aznow_tab[c];
        pa.refresh = (g.flags_tab[c] & kFlagRefresh) ? 1 : 0;
        pa.tmod_m = g.tmod_tab[2 * c];
        pa.tmod_p = g.tmod_tab[2 * c + 1];
        pa.raw_row = (long long)c * pa.nbins;
        pa.tile_rows = g.tile_rows;
    }
    const MixSmem<NOUT> sm = mix_smem<NOUT>(smem, kMaxCh, kPulseRowsMax);
    build_wtab<float, kMixS>(sm.wtab, pa.sinc, kSincTaps, kSincOvs);
    mix_init<NOUT>(sm);
    double spec_sum = 0.0, bragg_sum[2] = {0.0, 0.0};
    unsigned rseq = 0;
    bool bad = false;
    // the fast configurations of the single-scene kernel, chosen per CTA from its slot
    const bool fast = pa.do_kodis && pa.do_bragg && pa.npol == 1 && pa.nout == NOUT && !pa.lut && !pa.use_hmtf;
    if (fast && !pa.any_xti)
        mix_tile<NOUT, true, false, 2, 1>(pa, nullptr, nullptr, tile, g.tile_rows, sm, rseq, bad, spec_sum, bragg_sum);
    else if (fast)
        mix_tile<NOUT, true, false, 2, 2>(pa, nullptr, nullptr, tile, g.tile_rows, sm, rseq, bad, spec_sum, bragg_sum);
    else
        mix_tile<NOUT, true, false>(pa, nullptr, nullptr, tile, g.tile_rows, sm, rseq, bad, spec_sum, bragg_sum);
    if (pa.out0 == 0) {
        if (pa.do_kodis) block_atomic_sum(spec_sum, &pa.nrcs_spec[pa.az_step], sm.sred);
        if (pa.do_bragg && pa.refresh)
            for (int p = 0; p < pa.npol; ++p)
                block_atomic_sum(bragg_sum[p], &pa.nrcs_bragg[(long long)p * pa.az_steps + pa.az_step], sm.sred);
    }
}

template <typename T, int NOUT, int S>
static int launch_pulse(PulseArgs a, cudaStream_t st) {
    const size_t smem = pulse_smem_bytes<T, NOUT, S, kPulseRows>(a.nch);
    auto k = a.sca ? (a.spec_mode != 0 ? pulse_kernel<T, NOUT, S, kModeSca | kModeKa>
                                       : pulse_kernel<T, NOUT, S, kModeSca>)
           : a.skim ? (a.spec_mode != 0 ? pulse_kernel<T, NOUT, S, kModeSkim | kModeKa>
                                        : pulse_kernel<T, NOUT, S, kModeSkim>)
                    : (a.spec_mode != 0 ? pulse_kernel<T, NOUT, S, kModeKa> : pulse_kernel<T, NOUT, S, kModeStd>);
    if (ensure_smem((const void *)k, smem) != cudaSuccess)
        return OCS_ERR_CUDA;
    const int resident = resident_ctas((const void *)k, kPulseCols, smem);
    if (resident <= 0) return OCS_ERR_CUDA;
    // Tile height: the tallest (<= kPulseRows) that still gives every resident CTA slot a
    // tile in the last wave, so that no SM runs one tile more than the others.
    const int tiles_x = (a.nx + kPulseCols - 1) / kPulseCols;
    const long long want = (long long)resident * (((long long)tiles_x * ((a.ny + kPulseRows - 1) / kPulseRows) +
                                                   resident - 1) / resident);
    long long per_col = want / tiles_x;
    if (per_col < 1) per_col = 1;
    int rows = (int)((a.ny + per_col - 1) / per_col);
    a.tile_rows = rows < 16 ? (a.ny < 16 ? a.ny : 16) : (rows > kPulseRows ? kPulseRows : rows);
    // SKIM: a tile must not straddle two output rows (ny_integ is a power of two or ny)
    if (a.skim && a.ny_integ < a.ny) {
        a.tile_rows = a.ny_integ;
        while (a.tile_rows > kPulseRows) {
            if (a.tile_rows % 2) return OCS_ERR_ARG;
            a.tile_rows /= 2;
        }
    }
    const long long tiles = (long long)tiles_x * ((a.ny + a.tile_rows - 1) / a.tile_rows);
    const long long grid = tiles < resident ? tiles : resident;
    k<<<(unsigned)grid, kPulseCols, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// Tile height for a persistent launch: the tallest (<= kPulseRows) that still gives every
// resident CTA slot a tile in the last wave.
static int tile_rows_for(int nx, int ny, int cols, int resident) {
    const int tiles_x = (nx + cols - 1) / cols;
    const long long want = (long long)resident * (((long long)tiles_x * ((ny + kPulseRows - 1) / kPulseRows) +
                                                   resident - 1) / resident);
    long long per_col = want / tiles_x;
    if (per_col < 1) per_col = 1;
    const int rows = (int)((ny + per_col - 1) / per_col);
    return rows < 16 ? (ny < 16 ? ny : 16) : (rows > kPulseRows ? kPulseRows : rows);
}

template <int NOUT, bool KODIS>
static int launch_pulse_mixed(PulseArgs a, const MixMaps &maps, float *lo_row, cudaStream_t st) {
    const size_t smem = mix_smem_bytes<NOUT>(a.nch, kPulseRows);
    // the common configurations (one polarisation, every output in this pass, Kodis and
    // direct Romeiser Bragg, no hMTF; without (1) or with (2) XTI channels) run
    // instantiations with those fixed
    const bool fast = KODIS && a.do_kodis && a.do_bragg && a.npol == 1 && a.nout == NOUT && !a.lut && !a.use_hmtf;
    constexpr int F1 = KODIS ? 1 : 0, F2 = KODIS ? 2 : 0;
    auto k = !fast ? (a.refresh ? pulse_mixed_kernel<NOUT, KODIS, 1> : pulse_mixed_kernel<NOUT, KODIS, 0>)
             : !a.any_xti ? (a.refresh ? pulse_mixed_kernel<NOUT, KODIS, 1, F1> : pulse_mixed_kernel<NOUT, KODIS, 0, F1>)
                          : (a.refresh ? pulse_mixed_kernel<NOUT, KODIS, 1, F2> : pulse_mixed_kernel<NOUT, KODIS, 0, F2>);
    if (ensure_smem((const void *)k, smem) != cudaSuccess) return OCS_ERR_CUDA;
    const int resident = resident_ctas((const void *)k, kMixCols, smem);
    if (resident <= 0) return OCS_ERR_CUDA;
    a.tile_rows = tile_rows_for(a.nx, a.ny, kMixCols, resident);
    const long long tiles = (long long)((a.nx + kMixCols - 1) / kMixCols) * ((a.ny + a.tile_rows - 1) / a.tile_rows);
    const long long grid = tiles < resident ? tiles : resident;
    k<<<(unsigned)grid, kMixCols, smem, st>>>(a, maps, lo_row);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <bool KODIS>
static int launch_pulse_mixed_n(const PulseArgs &a, const MixMaps &maps, float *lo_row, cudaStream_t st) {
    if (a.nout == 1) return launch_pulse_mixed<1, KODIS>(a, maps, lo_row, st);
    if (a.nout == 2) return launch_pulse_mixed<2, KODIS>(a, maps, lo_row, st);
    return launch_pulse_mixed<4, KODIS>(a, maps, lo_row, st);
}

// Tensor-map encoder of the driver, resolved once through the runtime (no link to libcuda).
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// One map of a [depth][ny][nx] tensor of 4-byte elements with planes `plane` bytes apart
// and boxes of one row of kMixCols columns times `depth` planes (depth 1: two-dimensional).
static bool encode_rows_map(CUtensorMap &m, const void *base, CUtensorMapDataType type, int nx, int ny, int depth,
                            unsigned long long plane) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint32_t rank = depth > 1 ? 3 : 2;
    const cuuint64_t dims[3] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)depth};
    const cuuint64_t strides[2] = {(cuuint64_t)nx * 4, (cuuint64_t)plane};
    const cuuint32_t box[3] = {(cuuint32_t)kMixCols, 1, (cuuint32_t)depth};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(&m, type, rank, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of a pulse descriptor for the split-range kernel; false when its inputs do not
// allow them (fields not equally spaced in one allocation, misaligned bases, or nx not a
// multiple of 4).
static bool fill_mix_maps(const ocs_pulse_desc *d, MixMaps &m) {
    memset(&m, 0, sizeof(m));
    if (d->nx % 4 != 0 || d->nx < 4) return false;
    const int nf = d->do_kodis ? 8 : 5;
    const char *f[8] = {(const char *)d->dx_d, (const char *)d->dy_d, (const char *)d->dz_d,
                        (const char *)d->diffx_d, (const char *)d->diffy_d, (const char *)d->diffxx_d,
                        (const char *)d->diffyy_d, (const char *)d->diffxy_d};
    const long long plane = (long long)(f[1] - f[0]);
    const long long need = (long long)d->nx * d->ny * 4;
    if (plane < need || plane % 16 != 0 || ((uintptr_t)f[0] & 15)) return false;
    for (int k = 1; k < nf; ++k)
        if (!f[k] || f[k] - f[0] != k * plane) return false;
    m.nf = nf;
    if (!encode_rows_map(m.fields, f[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d->nx, d->ny, nf, (unsigned long long)plane))
        return false;
    if (d->do_bragg) {
        if ((((uintptr_t)d->ind0_m_d) | ((uintptr_t)d->ind0_p_d) | ((uintptr_t)d->scat_d)) & 15) return false;
        if (!encode_rows_map(m.indm, d->ind0_m_d, CU_TENSOR_MAP_DATA_TYPE_INT32, d->nx, d->ny, 1, 0) ||
            !encode_rows_map(m.indp, d->ind0_p_d, CU_TENSOR_MAP_DATA_TYPE_INT32, d->nx, d->ny, 1, 0) ||
            !encode_rows_map(m.scat, d->scat_d, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, d->nx, d->ny, 2 * d->npol,
                             (unsigned long long)need))
            return false;
    }
    return true;
}

}  // namespace ocs

using namespace ocs;

static int fill_pulse_args(const ocs_pulse_desc *d, PulseArgs &a) {
    memset(&a, 0, sizeof(a));
    if (!d || d->nx < 1 || d->ny < 1 || d->npol < 1 || d->npol > 2 || d->nch < 1 || d->nch > kMaxCh)
        return OCS_ERR_ARG;
    if (!d->dx_d || !d->dy_d || !d->dz_d || !d->y_d || !d->sr_col_d || !d->sin_inc_d || !d->cos_inc_d ||
        !d->inc_d || !d->sinc_d || !d->raw_d)
        return OCS_ERR_ARG;
    if (d->do_kodis && (!d->diffx_d || !d->diffy_d || !d->diffxx_d || !d->diffyy_d || !d->diffxy_d ||
                        !d->tan_inc_d || !d->nrcs_spec_d))
        return OCS_ERR_ARG;
    if (d->do_bragg && (!d->diffx_d || !d->diffy_d || !d->c_b_d || (!d->scat_d && !d->sca) || !d->s_m_d || !d->s_p_d ||
                        !d->ind0_m_d || !d->ind0_p_d || d->n_m < 1 || d->n_p < 1 || !d->spec_k_d ||
                        !d->spec_s_d || d->spec_n < 2 || !d->nrcs_bragg_d))
        return OCS_ERR_ARG;
    if (d->do_bragg && d->use_hmtf && !d->hmtf_d) return OCS_ERR_ARG;
    if (d->az_step < 0 || d->az_step >= d->az_steps || d->nbins < 1 || !d->rowtab_d) return OCS_ERR_ARG;
    if ((d->npol == 2) != (d->pol == POL_DP)) return OCS_ERR_ARG;
    a.nx = d->nx; a.ny = d->ny; a.npol = d->npol; a.nch = d->nch;
    a.dx_f = d->dx_d; a.dy_f = d->dy_d; a.dz_f = d->dz_d;
    a.diffx = d->diffx_d; a.diffy = d->diffy_d;
    a.diffxx = d->diffxx_d; a.diffyy = d->diffyy_d; a.diffxy = d->diffxy_d; a.hmtf = d->hmtf_d;
    a.y = d->y_d;
    a.sr_col = d->sr_col_d; a.sin_inc = d->sin_inc_d; a.cos_inc = d->cos_inc_d; a.tan_inc = d->tan_inc_d;
    a.inc = d->inc_d; a.c_b = d->c_b_d;
    a.inc_angle = d->inc_angle; a.sr0 = d->sr0; a.gr0 = d->gr0; a.k0 = d->k0; a.az_now = d->az_now;
    a.min_sr = d->min_sr; a.binsize = d->binsize; a.inv_binsize = 1.0 / d->binsize;
    a.t_step = d->t_step; a.az_step = d->az_step;
    a.tind = d->tind;
    a.ltx_over_l = d->ant_l_tx * d->f0 / 2.99792458e8;
    a.lrx_over_l = d->ant_l_rx * d->f0 / 2.99792458e8;
    for (int c = 0; c < d->nch; ++c) {
        a.b_ati[c] = d->b_ati[c];
        a.b_xti[c] = d->b_xti[c];
        if (d->b_xti[c] != 0.0) a.any_xti = 1;
    }
    a.do_kodis = d->do_kodis; a.do_bragg = d->do_bragg; a.refresh = d->refresh; a.use_hmtf = d->use_hmtf;
    a.kodis.k0 = d->k0;
    a.kodis.R_re = d->kodis_R_re; a.kodis.R_im = d->kodis_R_im;
    a.kodis.hdx = (double)d->facet_dx * 0.5; a.kodis.hdy = (double)d->facet_dy * 0.5;
    RomeiserParams &r = a.rom;
    r.k0 = d->k0; r.d = d->bragg_d; r.dx = (double)d->facet_dx; r.dy = (double)d->facet_dy;
    r.wind_dir = d->wind_dir; r.wind_U = d->wind_U; r.pol = d->pol; r.spread = d->spread;
    r.ck_p = d->spread_ck_p; r.ck_m = d->spread_ck_m; r.a0 = d->spread_a0; r.ap = d->spread_ap;
    r.am = d->spread_am;
    r.tab_k = d->spec_k_d; r.tab_s = d->spec_s_d; r.tab_n = d->spec_n;
    r.eps_re = 73.0; r.eps_im = 18.0;
    r.seps_re = d->sqrt_eps_re; r.seps_im = d->sqrt_eps_im;
    r.eps2_re = 73.0 * 73.0 - 18.0 * 18.0; r.eps2_im = 2.0 * 73.0 * 18.0;
    a.scat = d->scat_d; a.s_m = d->s_m_d; a.s_p = d->s_p_d;
    if (d->s_m32_d && d->s_p32_d) { a.s_m32 = d->s_m32_d; a.s_p32 = d->s_p32_d; }
    if (d->do_bragg) {
        if (d->n_m > (1LL << 30) || d->n_p > (1LL << 30) || d->tind < 0) return OCS_ERR_SIZE;
        a.n_m = (int)d->n_m; a.n_p = (int)d->n_p;
        a.tmod_m = (int)(d->tind % d->n_m); a.tmod_p = (int)(d->tind % d->n_p);
    }
    a.ind0_m = d->ind0_m_d; a.ind0_p = d->ind0_p_d;
    a.sinc = d->sinc_d;
    a.raw = d->raw_d;
    a.rowtab = (double *)d->rowtab_d;
    a.nbins = d->nbins;
    a.raw_out_stride = (long long)d->az_steps * d->nbins;
    a.raw_row = (long long)d->az_step * d->nbins;
    a.nrcs_spec = d->nrcs_spec_d; a.nrcs_bragg = d->nrcs_bragg_d; a.az_steps = d->az_steps;
    a.spec_mode = d->do_kodis ? d->spec_mode : 0;
    if (a.spec_mode < 0 || a.spec_mode > 2) return OCS_ERR_ARG;
    if (a.spec_mode != 0 && !d->x_d) return OCS_ERR_ARG;
    a.x_f = d->x_d;
    a.ka.k0 = d->k0; a.ka.dx = d->ka_dx; a.ka.dy = d->ka_dy; a.ka.K_re = d->ka_K_re; a.ka.K_im = d->ka_K_im;
    a.ka.mode = a.spec_mode == 2 ? 1 : 0;
    if (d->skim) {
        // SKIM mode: one channel; the facets of every skim_ny_integ rows go to their
        // own output row: raw_d holds [npol][az_steps][ny / skim_ny_integ][nbins]
        if (d->sca || d->nch != 1 || d->skim_ny_integ < 1 || d->ny % d->skim_ny_integ != 0) return OCS_ERR_ARG;
        if (d->skim_ny_integ > kPulseRows && d->skim_ny_integ < d->ny) {
            for (int n = d->skim_ny_integ; n > kPulseRows; n /= 2)
                if (n % 2) return OCS_ERR_ARG;
        }
        a.skim = 1;
        a.ny_integ = d->skim_ny_integ;
        a.s_int = d->ny / d->skim_ny_integ;
        a.skim_az2 = d->skim_az2 != 0;
        a.skim_rcm = d->skim_rcm != 0;
        if (d->pt_mode < 0 || d->pt_mode > 2) return OCS_ERR_ARG;
        a.pt_mode = d->pt_mode;
        a.pt_x = d->pt_x;
        a.pt_y = d->pt_y;
        a.pt_amp = d->pt_amp;
        a.atx = a.ltx_over_l;
        a.arx = a.lrx_over_l;
        a.raw_out_stride = (long long)d->az_steps * a.s_int * d->nbins;
        a.raw_row = (long long)d->az_step * a.s_int * d->nbins;
    }
    if (d->sca) {
        // scatterometer mode: one channel, Kodis or Kirchhoff specular (the field scaled by
        // the two-way spreading like the Kodis field), Bragg model (hMTF, when on,
        // read at the rolled row of the [ny][field_nx] surface, unclipped); the columns are
        // whole range blocks of field_nx columns; the Bragg RCS is evaluated on every launch
        // and not stored
        if (d->nch != 1 || d->field_nx < 1 || d->nx % d->field_nx != 0 || d->roll < 0 || d->roll >= d->ny ||
            d->lut_block < 0)
            return OCS_ERR_ARG;
        a.lut_block = d->lut_d ? d->lut_block : 0;
        if (!(d->sr_bin_offset >= 0.0) || !(d->cap_t >= 0.0)) return OCS_ERR_ARG;
        if (d->nrcs_rows < 1 || d->nrcs_row < 0 || d->nrcs_row >= d->nrcs_rows) return OCS_ERR_ARG;
        a.sca = 1;
        a.az_f32 = d->az_f32 != 0;
        a.nblk = d->nx / d->field_nx;
        a.nrcs_row = d->nrcs_row;
        a.nrcs_rows = d->nrcs_rows;
        a.fnx = d->field_nx;
        a.roll = d->roll;
        a.sr_bin_off = d->sr_bin_offset;
        a.cap_t = d->cap_t;
        a.refresh = 1;
        a.scat = nullptr;
    } else {
        a.fnx = d->nx;
    }
    a.lut = d->lut_d;
    if (a.lut) {
        if (d->lut_naz < 1 || d->lut_ndy < 1 || d->lut_ndx < 1 || !(d->lut_daz != 0.0) || !(d->lut_ddy != 0.0) ||
            !(d->lut_ddx != 0.0))
            return OCS_ERR_ARG;
        a.lut_naz = d->lut_naz; a.lut_ndy = d->lut_ndy; a.lut_ndx = d->lut_ndx;
        a.lut_az0 = d->lut_az0; a.lut_daz = d->lut_daz; a.lut_dy0 = d->lut_dy0; a.lut_ddy = d->lut_ddy;
        a.lut_dx0 = d->lut_dx0; a.lut_ddx = d->lut_ddx;
    }
    return OCS_OK;
}

namespace ocs {

size_t pulse_args_bytes() { return sizeof(PulseArgs); }

int pulse_args_fill(const ocs_pulse_desc *d, void *out) {
    if (d && (d->sca || d->skim)) return OCS_ERR_ARG;   // the scene batch runs SAR scenes only
    PulseArgs a;
    const int st = fill_pulse_args(d, a);
    if (st == OCS_OK) memcpy(out, &a, sizeof(a));
    return st;
}

int batch_launch_pulse_rows(const BatchRef &b, int precision, cudaStream_t st) {
    int sms = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return OCS_ERR_CUDA;
    if (precision == OCS_PREC_MIXED) batch_pulse_rows_kernel<true><<<sms * 4, 128, 0, st>>>(b);
    else batch_pulse_rows_kernel<false><<<sms * 4, 128, 0, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <int NOUT>
static int batch_pulse_mixed_n(const BatchRef &b, int grid, cudaStream_t st) {
    const size_t smem = mix_smem_bytes<NOUT>(kMaxCh, kPulseRowsMax);
    auto k = batch_pulse_mixed_kernel<NOUT>;
    if (ensure_smem((const void *)k, smem) != cudaSuccess) return OCS_ERR_CUDA;
    k<<<grid, kMixCols, smem, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

template <typename T, int NOUT, int S, int MODE = kModeStd>
static int batch_pulse_n(const BatchRef &b, int grid, cudaStream_t st) {
    const size_t smem = pulse_smem_bytes<T, NOUT, S, kPulseRowsMax>(kMaxCh);
    auto k = batch_pulse_kernel<T, NOUT, S, MODE>;
    if (ensure_smem((const void *)k, smem) != cudaSuccess) return OCS_ERR_CUDA;
    k<<<grid, kPulseCols, smem, st>>>(b);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

int batch_pulse_items(int nx, int ny, int tile_rows, int nout, int precision, int width) {
    const int G = precision == OCS_PREC_F64 ? 2 : 4;
    int groups = 0;
    for (int o = 0; o < nout; o += G) groups += width_class(nout - o < G ? nout - o : G) == width;
    return groups * ((nx + kPulseCols - 1) / kPulseCols) * ((ny + tile_rows - 1) / tile_rows);
}

int pulse_kind(const ocs_pulse_desc *d) { return (d->do_kodis && d->spec_mode != 0) ? kSlotKa : kSlotStd; }

int batch_launch_pulse(const BatchRef &b, int precision, int kind, int width, int grid, cudaStream_t st) {
    if (grid < 1) return OCS_OK;
    if (kind == kSlotKa) {
        // Kirchhoff scenes: float64 ranges and phases in both precisions, as their single-scene
        // pulses run (float32 for the rest in the mixed form)
        if (precision == OCS_PREC_F64) {
            if (width == 1) return batch_pulse_n<double, 1, 12, kModeKa>(b, grid, st);
            if (width == 2) return batch_pulse_n<double, 2, 12, kModeKa>(b, grid, st);
            return OCS_ERR_ARG;
        }
        if (precision == OCS_PREC_MIXED) {
            if (width == 1) return batch_pulse_n<float, 1, 12, kModeKa>(b, grid, st);
            if (width == 2) return batch_pulse_n<float, 2, 12, kModeKa>(b, grid, st);
            if (width == 4) return batch_pulse_n<float, 4, 12, kModeKa>(b, grid, st);
            return OCS_ERR_ARG;
        }
        return OCS_ERR_ARG;
    }
    if (precision == OCS_PREC_F64) {
        if (width == 1) return batch_pulse_n<double, 1, 12>(b, grid, st);
        if (width == 2) return batch_pulse_n<double, 2, 12>(b, grid, st);
        return OCS_ERR_ARG;
    }
    if (precision == OCS_PREC_MIXED) {
        if (width == 1) return batch_pulse_mixed_n<1>(b, grid, st);
        if (width == 2) return batch_pulse_mixed_n<2>(b, grid, st);
        if (width == 4) return batch_pulse_mixed_n<4>(b, grid, st);
        return OCS_ERR_ARG;
    }
    return OCS_ERR_ARG;
}

}  // namespace ocs

extern "C" int64_t ocs_pulse_workspace_bytes(int32_t ny, int32_t nch) {
    if (ny < 1 || nch < 1 || nch > kMaxCh) return -1;
    return (int64_t)(mix_hdr_offset(ny, nch) + kMixHdrBytes);
}

// Whether the split-range mixed kernel takes this pulse: SAR mode with Kodis and / or
// direct / LUT Bragg scattering, the float32 scatterer series, column counts and base
// pointers that allow 16-byte bulk copies of every input row.
static bool mixed_split_ok(const ocs_pulse_desc *d);
namespace ocs {
bool pulse_split_ok(const ocs_pulse_desc *d) { return mixed_split_ok(d); }
}  // namespace ocs
static bool mixed_split_ok(const ocs_pulse_desc *d) {
    if (d->sca || d->skim || (d->do_kodis && d->spec_mode != 0) || !(d->do_kodis || d->do_bragg)) return false;
    if (d->do_bragg && (!d->s_m32_d || !d->s_p32_d)) return false;
    if (!d->diffx_d || !d->diffy_d || ((uintptr_t)d->rowtab_d & 15)) return false;
    MixMaps m;
    return fill_mix_maps(d, m);
}

// Compensation row of the mixed kernel (complex64 [npol*nch][nbins]) and the workspace
// header: reset before a scene (pending row -1, error flag 0, row zeroed).
extern "C" int ocs_pulse_reset(const ocs_pulse_desc *d, void *stream) {
    if (!d || !d->rowtab_d || d->ny < 1 || d->nch < 1 || d->nch > kMaxCh) return OCS_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *hdr = (unsigned char *)d->rowtab_d + mix_hdr_offset(d->ny, d->nch);
    if (cudaMemsetAsync(hdr, 0xff, 4, s) != cudaSuccess) return OCS_ERR_CUDA;
    if (cudaMemsetAsync(hdr + 4, 0, kMixHdrBytes - 4, s) != cudaSuccess) return OCS_ERR_CUDA;
    if (d->raw_lo_d) {
        const size_t n = (size_t)d->npol * d->nch * d->nbins * 2 * sizeof(float);
        if (cudaMemsetAsync(d->raw_lo_d, 0, n, s) != cudaSuccess) return OCS_ERR_CUDA;
    }
    return OCS_OK;
}

// Fold the last pulse's compensation row into its raw row (the scene's final step, or
// before the raw cube is read); no-op when nothing is pending.
extern "C" int ocs_pulse_flush(const ocs_pulse_desc *d, void *stream) {
    PulseArgs a;
    int st = fill_pulse_args(d, a);
    if (st != OCS_OK) return st;
    if (!d->raw_lo_d) return OCS_OK;
    const int nout = d->npol * d->nch;
    const long long n = (long long)nout * d->nbins;
    long long blocks = (n + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    pulse_flush_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a, (float *)d->raw_lo_d, nout);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// Status of the mixed kernel's bounded waits since the last reset (synchronises with the
// device): OCS_OK, or OCS_ERR_TIMEOUT if a wait gave up.
extern "C" int ocs_pulse_error(const ocs_pulse_desc *d) {
    if (!d || !d->rowtab_d || d->ny < 1 || d->nch < 1 || d->nch > kMaxCh) return OCS_ERR_ARG;
    int flag = 0;
    const unsigned char *hdr = (const unsigned char *)d->rowtab_d + mix_hdr_offset(d->ny, d->nch);
    if (cudaMemcpy(&flag, hdr + 4, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return OCS_ERR_CUDA;
    return flag ? OCS_ERR_TIMEOUT : OCS_OK;
}

extern "C" int ocs_pulse(const ocs_pulse_desc *d, int precision, void *stream) {
    PulseArgs a;
    int st = fill_pulse_args(d, a);
    if (st != OCS_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int nout = d->npol * d->nch;
    if (!(precision == OCS_PREC_MIXED && mixed_split_ok(d))) {
        pulse_rows_kernel<<<(d->ny + 127) / 128, 128, 0, s>>>(a);
        if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
    }
    if (precision == OCS_PREC_F64) {
        for (int o = 0; o < nout; o += 2) {
            a.out0 = o;
            a.nout = nout - o < 2 ? nout - o : 2;
            st = (a.nout == 1) ? launch_pulse<double, 1, 12>(a, s) : launch_pulse<double, 2, 12>(a, s);
            if (st != OCS_OK) return st;
            a.refresh = 0;                  // later groups read the refreshed RCS
        }
        return OCS_OK;
    }
    if (precision == OCS_PREC_MIXED && mixed_split_ok(d)) {
        MixMaps maps;
        if (!fill_mix_maps(d, maps)) return OCS_ERR_CUDA;
        float *lo_row = (float *)d->raw_lo_d;
        const int rows = d->ny > nout * d->nbins ? d->ny : nout * d->nbins;
        long long blocks = (rows + 127) / 128;
        if (blocks > 4096) blocks = 4096;
        pulse_rows_mixed_kernel<<<(unsigned)blocks, 128, 0, s>>>(a, lo_row, nout);
        if (cudaGetLastError() != cudaSuccess) return OCS_ERR_CUDA;
        for (int o = 0; o < nout; o += 4) {
            a.out0 = o;
            a.nout = nout - o < 4 ? nout - o : 4;
            st = d->do_kodis ? launch_pulse_mixed_n<true>(a, maps, lo_row, s)
                             : launch_pulse_mixed_n<false>(a, maps, lo_row, s);
            if (st != OCS_OK) return st;
            a.refresh = 0;
        }
        return OCS_OK;
    }
    if (precision == OCS_PREC_MIXED) {
        for (int o = 0; o < nout; o += 4) {
            a.out0 = o;
            a.nout = nout - o < 4 ? nout - o : 4;
            if (a.nout == 1) st = launch_pulse<float, 1, 12>(a, s);
            else if (a.nout == 2) st = launch_pulse<float, 2, 12>(a, s);
            else st = launch_pulse<float, 4, 12>(a, s);
            if (st != OCS_OK) return st;
            a.refresh = 0;
        }
        return OCS_OK;
    }
    return OCS_ERR_ARG;
}
