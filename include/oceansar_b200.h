/*
 * oceansar_b200 -- C ABI of the B200 (sm_100a) raw-data-generation path.
 *
 * Plain pointers and sizes only.  Every pointer argument named *_d is a DEVICE pointer
 * (cudaMalloc / torch CUDA tensor storage) on the current device; `stream` is a
 * cudaStream_t (NULL = legacy default stream).  Every call is asynchronous on `stream`
 * and returns an ocs_status; a kernel launch error is reported as OCS_ERR_CUDA.
 * Complex arrays are interleaved (re, im) pairs: complex128 = 2 doubles, complex64 =
 * 2 floats.  2-D arrays are C-contiguous [rows][cols].
 *
 * Each entry point names the reference (pakodekker/oceansar) interface it replaces.
 */
#ifndef OCEANSAR_B200_H
#define OCEANSAR_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    OCS_OK = 0,
    OCS_ERR_ARG = -1,          /* null pointer, negative size, inconsistent arguments   */
    OCS_ERR_CUDA = -2,         /* a CUDA launch / runtime call failed                    */
    OCS_ERR_SIZE = -3,         /* sizes beyond what the kernels support                 */
    OCS_ERR_UNSUPPORTED = -4,  /* a valid option this build does not implement          */
    OCS_ERR_TIMEOUT = -5       /* a bounded device-side wait gave up                    */
} ocs_status;

/* Library version, "major.minor.patch". */
const char *ocs_version(void);

/* ------------------------------------------------------------------------------------
 * Facet-to-range-bin accumulation.
 *
 * Replaces chan_profile_numba (oceansar/radarsim/range_profile.py:83-116), i.e. the
 * bin / LUT prologue (:103-108) followed by profile_integrator (:22-49):
 *   bin_f = (srg - min_sr) / binsize; bin_d = floor(bin_f);
 *   lut = round_half_even(sinc_ovs * (1 - (bin_f - bin_d)));
 *   output[bin_d - n/2 + j] += sinc_vec[lut + j*sinc_ovs] * scene,  0 <= j < n,
 * dropping taps outside [0, nbins).  `output` is accumulated in place (never cleared).
 * srg_d: float64 [npts]; scene_d: complex128 [npts]; sinc_vec_d: float32
 * [n*sinc_ovs + 1] (calc_sinc_vec, range_profile.py:15-19); output_d: complex128 [nbins].
 * n_sinc_samples <= 16.
 */
int ocs_chan_profile_f64(const double *srg_d, const double *scene_d, int64_t npts,
                         double binsize, double min_sr, const float *sinc_vec_d,
                         int n_sinc_samples, int sinc_ovs, double *output_d, int64_t nbins,
                         void *stream);

/* Row-wise form (rg_only=True): replaces profile_integrator_1d (range_profile.py:52-80).
 * srg_d [naz][npts], scene_d complex128 [naz][npts], output_d complex128 [naz][nbins]. */
int ocs_chan_profile_rows_f64(const double *srg_d, const double *scene_d, int64_t naz,
                              int64_t npts, double binsize, double min_sr,
                              const float *sinc_vec_d, int n_sinc_samples, int sinc_ovs,
                              double *output_d, int64_t nbins, void *stream);

/* Single-precision accumulation of a complex64 scene into a complex64 output (same
 * float64 bin / LUT prologue).  No reference counterpart: the mixed-precision form. */
int ocs_chan_profile_c64(const double *srg_d, const float *scene_d, int64_t npts,
                         double binsize, double min_sr, const float *sinc_vec_d,
                         int n_sinc_samples, int sinc_ovs, float *output_d, int64_t nbins,
                         void *stream);

/* ocs_chan_profile_f64 for facets laid out as a [ny][nx] surface (azimuth rows, ground-
 * range columns; the order sar_raw flattens them in, sar_raw_nompi.py:535): the same sum
 * into output[nbins], computed column-wise so that each thread's range bin barely moves.
 * Replaces chan_profile_numba (range_profile.py:83-116) when the caller keeps the 2-D
 * shape; the result equals ocs_chan_profile_f64 on the flattened arrays up to summation
 * order.  _c64: the single-precision scene / output form (no reference counterpart). */
int ocs_chan_profile_2d_f64(const double *srg_d, const double *scene_d, int64_t ny, int64_t nx,
                            double binsize, double min_sr, const float *sinc_vec_d,
                            int n_sinc_samples, int sinc_ovs, double *output_d, int64_t nbins,
                            void *stream);
int ocs_chan_profile_2d_c64(const double *srg_d, const float *scene_d, int64_t ny, int64_t nx,
                            double binsize, double min_sr, const float *sinc_vec_d,
                            int n_sinc_samples, int sinc_ovs, float *output_d, int64_t nbins,
                            void *stream);


/* ------------------------------------------------------------------------------------
 * Per-pulse surface synthesis.
 *
 * Replaces the OceanSurface.t setter (oceansar/surfaces/ocean.py:418-526): propagation
 * c(t) = wave_coefs * exp(-i omega t) (:424-427) and one inverse 2-D FFT per field, here
 * two real fields per complex transform.  Field codes name the reference's attributes;
 * the OCS_FIELD_AUX_* codes are the intermediate choppy-wave transforms (:452-482).
 */
enum {
    OCS_FIELD_DZ = 0, OCS_FIELD_DX = 1, OCS_FIELD_DY = 2,
    OCS_FIELD_DIFFX = 3, OCS_FIELD_DIFFY = 4,
    OCS_FIELD_DIFFXX = 5, OCS_FIELD_DIFFYY = 6, OCS_FIELD_DIFFXY = 7,
    OCS_FIELD_VX = 8, OCS_FIELD_VY = 9, OCS_FIELD_VZ = 10,
    OCS_FIELD_AX = 11, OCS_FIELD_AY = 12, OCS_FIELD_AZ = 13,
    OCS_FIELD_HMTF = 14,
    OCS_FIELD_AUX_XX = 15, OCS_FIELD_AUX_YY = 16,
    OCS_FIELD_AUX_XXX = 17, OCS_FIELD_AUX_YYY = 18, OCS_FIELD_AUX_XXY = 19,
    OCS_FIELD_COUNT = 20
};

typedef struct {
    int32_t nx, ny;            /* grid (Nx, Ny); every prime factor in {2, 3, 5, 7}      */
    const void *coefs_d;       /* complex64 [ny][nx] wave_coefs (ocean.py:236)          */
    const float *omega_d;      /* float32 [ny][nx] dispersion relation (ocean.py:155-158) */
    const float *kx_d;         /* float32 [nx] 2*pi*fftfreq(nx, dx) (ocean.py:131)      */
    const float *ky_d;         /* float32 [ny] 2*pi*fftfreq(ny, dy) (ocean.py:133)      */
    float kmin_half;           /* min(kx_res, ky_res)/2, the |k| cut of kxn/kyn/kinv (:142) */
    int32_t nfields;           /* 1 .. 24                                               */
    const int32_t *codes;      /* host [nfields] OCS_FIELD_* codes                      */
    float *const *dst_d;       /* host [nfields] device pointers, float32 [ny][nx]      */
    const float *add;          /* host [nfields] constant term (current*t, current) or NULL */
    const float *swell_mult;   /* host [2*nfields] complex factor of the swell term or NULL */
    const void *swell_exp_d;   /* complex64 [ny][nx] monochromatic swell (:231-233) or NULL */
    float swell_rot_re;        /* exp(-i swell_omega t), complex64                      */
    float swell_rot_im;
    void *workspace_d;         /* ocs_surface_workspace_bytes() bytes, ocs_surface_prepare()d */
} ocs_surface_desc;

/* Workspace for a grid and field count: twiddle tables + packed scratch planes; < 0 on
 * invalid sizes. */
int64_t ocs_surface_workspace_bytes(int32_t nx, int32_t ny, int32_t nfields);

/* Fill the twiddle tables of a workspace (once per grid). */
int ocs_surface_prepare(int32_t nx, int32_t ny, void *workspace_d, void *stream);

/* Synthesize the requested fields at time t (float32, as ocean.py:424 casts it). */
int ocs_surface_update(const ocs_surface_desc *desc, float t, void *stream);

/* One or both passes of ocs_surface_update: passes = 1 runs the row pass (phase evolution,
 * spectral multipliers, row transforms into the workspace), 2 the column pass (column
 * transforms, field store), 3 both (= ocs_surface_update).  Pass 2 reads what pass 1 of
 * the same descriptor and t left in the workspace.  Lets a caller time or schedule the two
 * kernels separately; same reference interface as ocs_surface_update. */
int ocs_surface_update_passes(const ocs_surface_desc *desc, float t, int passes, void *stream);

typedef struct {
    int64_t n;                                       /* ny*nx                               */
    const float *ax_d, *ay_d, *axx_d, *ayy_d;        /* Re ifft2 of i kx c, i ky c, -kx^2/k c, -ky^2/k c */
    const float *axxx_d, *ayyy_d, *axxy_d;           /* -i kx^3/k c, -i ky^3/k c, -i kx^2 ky/k c (Diff2 only) */
    const float *fxx_d, *fyy_d, *fxy_d;              /* -kx^2 c, -ky^2 c, -kx ky c (Diff2 only) */
    float *diffx_d, *diffy_d;                        /* outputs (NULL: skip the slopes)    */
    float *diffxx_d, *diffyy_d, *diffxy_d;           /* outputs (NULL: skip the curvatures) */
    const void *swell_exp_d;                         /* complex64 swell or NULL            */
    float swell_rot_re, swell_rot_im;
    const float *swell_mult;                         /* host [10]: Diffx, Diffy, Diffxx, Diffyy, Diffxy */
} ocs_choppy_desc;

/* Choppy-wave slopes / curvatures from the auxiliary fields (ocean.py:451-456, 468-482). */
int ocs_surface_choppy(const ocs_choppy_desc *desc, void *stream);

/* Time-interpolated fields (OceanSurfaceBalancer.t, oceansar/surfaces/balancer.py:126-297):
 * dst[f][i] = w_l * a[f][i] + w_h * b[f][i] in float32 for nfields float32 planes of n
 * elements (16-byte aligned); a / b hold the fields synthesised at the ends of the ocean
 * time step.  a_d, b_d, dst_d are host arrays of device pointers. */
int ocs_surface_blend(int64_t n, int32_t nfields, const float *const *a_d, const float *const *b_d,
                      float *const *dst_d, float w_l, float w_h, void *stream);

/* ocs_surface_update for callers that cannot allocate device memory (no counterpart in the
 * reference).  desc->workspace_d is ignored: the workspace is a 32 MiB device array
 * compiled into the library, so ocs_surface_workspace_bytes(nx, ny, nfields) must be at
 * most 32 MiB (else OCS_ERR_SIZE).  The descriptor is checked before anything is
 * launched.  Every call resolves the array's address on the current device; with lazy
 * module loading the first call on a device also loads the module, so make one warm-up
 * call before any latency-critical loop or stream capture.  All calls on a device share
 * the array, so calls that overlap on the GPU race and must be serialised by the caller.
 * Allocates nothing. */
int ocs_surface_update_noalloc(const ocs_surface_desc *desc, float t, void *stream);

/* ------------------------------------------------------------------------------------
 * One radar pulse of the raw-data generator.
 *
 * Replaces the body of the azimuth loop of sar_raw (oceansar/radarsim/sar_raw_nompi.py:
 * 351-535) once the surface fields of the pulse exist: slant range (:366-369), Kodis
 * specular field (:392-400, nrcs/kodis.py:38-73), Romeiser Bragg RCS refreshed when
 * `refresh` is set (:431-458, nrcs/romeiser97.py:252-393), Bragg phases and random
 * sub-grid scatterers (:470-480, closure/random_scatterers.py:28-31), antenna pattern and
 * ATI / XTI channel phases (:485-495, radarsim/antenna.py:5-25), accumulated into range
 * bins (chan_profile_numba).  All device arrays stay resident between pulses.
 */
enum { OCS_PREC_F64 = 0, OCS_PREC_MIXED = 1 };
enum { OCS_POL_VV = 0, OCS_POL_HH = 1, OCS_POL_DP = 2 };
enum { OCS_SPREAD_ELFOUHAILY = 0, OCS_SPREAD_COS2S = 1 };

typedef struct {
    int32_t nx, ny;                      /* facet grid                                       */
    int32_t npol;                        /* 1, or 2 for pol == OCS_POL_DP (hh then vv)       */
    int32_t pol;                         /* OCS_POL_*                                       */
    int32_t nch;                         /* channels, <= 8                                  */
    /* float32 [ny][nx] surface fields of this pulse */
    const float *dx_d, *dy_d, *dz_d, *diffx_d, *diffy_d, *diffxx_d, *diffyy_d, *diffxy_d, *hmtf_d;
    const float *y_d;                    /* float32 [ny] azimuth coordinate of each row      */
    /* float64 [nx] per ground-range column: slant range minus its minimum, sin / cos / tan
     * of the incidence angle, incidence angle, Bragg phase speed sin(inc) sqrt(g/kb + ...) */
    const double *sr_col_d, *sin_inc_d, *cos_inc_d, *tan_inc_d, *inc_d, *c_b_d;
    double inc_angle;                    /* nominal incidence [rad]                          */
    double sr0, gr0;                     /* slant / ground range of the scene centre         */
    double k0, f0;                       /* radar wavenumber, carrier frequency              */
    double az_now;                       /* (t_now - t_span/2) * v_ground                    */
    double min_sr, binsize;              /* range window start, range bin size               */
    double t_step;                       /* 1 / prf                                          */
    int32_t az_step, az_steps;           /* this pulse, pulses in the raw cube               */
    int64_t tind;                        /* int(t_now * prf) of the scatterer series         */
    double ant_l_tx, ant_l_rx;           /* antenna lengths                                  */
    const double *b_ati, *b_xti;         /* host [nch] along- / cross-track baselines        */
    int32_t do_kodis, do_bragg, refresh, use_hmtf;
    double kodis_R_re, kodis_R_im;       /* (eps - sqrt eps)/(eps + sqrt eps), eps = 73+18j  */
    float facet_dx, facet_dy;            /* surface dx, dy (float32)                         */
    double bragg_d;                      /* Bragg filter threshold d                         */
    double wind_dir, wind_U;             /* effective wind for the Bragg spectrum            */
    int32_t spread;                      /* OCS_SPREAD_*                                     */
    double spread_ck_p, spread_ck_m, spread_a0, spread_ap, spread_am;  /* Elfouhaily Delta(k) */
    const double *spec_k_d, *spec_s_d;   /* float64 [spec_n] omni-directional spectrum table */
    int32_t spec_n;
    double sqrt_eps_re, sqrt_eps_im;     /* sqrt(73+18j)                                     */
    void *scat_d;                        /* [npol][2][ny][nx] sqrt(RCS): float64 (F64) or float32 (MIXED) */
    const double *s_m_d, *s_p_d;         /* complex128 scatterer series (rndscat_m, rndscat_p) */
    int64_t n_m, n_p;
    const int32_t *ind0_m_d, *ind0_p_d;  /* int32 [ny][nx] start indices                     */
    const float *sinc_d;                 /* float32 [161] calc_sinc_vec(8, 20, over_fs)      */
    void *raw_d;                         /* [npol*nch][az_steps][nbins] complex128 (F64) / complex64 (MIXED) */
    int32_t nbins;                       /* rg_samp                                          */
    double *nrcs_spec_d;                 /* float64 [az_steps]: += sum |E_spec|^2            */
    double *nrcs_bragg_d;                /* float64 [npol][az_steps]: += sum RCS at refresh  */
    void *rowtab_d;                      /* ocs_pulse_workspace_bytes(ny, nch) bytes         */
    /* Romeiser LUT mode (romeiser97.py:71-134): on refresh pulses the Bragg RCS is looked up
     * at (round((az - lut_az0)/lut_daz), clamp(round((Diffy - lut_dy0)/lut_ddy)),
     * clamp(round((Diffx - lut_dx0)/lut_ddx))) instead of evaluated.  lut_d: [npol][2][naz]
     * [ndy][ndx] float64 (F64) / float32 (MIXED); NULL: direct model.  Negative azimuth
     * indices count from the end, as numpy indexing does; larger ones are the caller's error
     * (checked on the host). */
    const void *lut_d;
    int32_t lut_naz, lut_ndy, lut_ndx;
    double lut_az0, lut_daz, lut_dy0, lut_ddy, lut_dx0, lut_ddx;
    /* Specular model when do_kodis is set: 0 Kodis (kodis.py), 1 Kirchhoff facet approach,
     * 2 Kirchhoff stationary phase (ka.py; sar_raw_nompi.py:402-426, per polarisation
     * exp(-2j k0 r) (4 pi)^1.5 RCSKA.field).  x_d: float32 [nx] facet x positions (Kirchhoff
     * only); ka_dx / ka_dy: facet sizes; ka_K: RCSKA's constant for R_i = R_s = 1. */
    int32_t spec_mode;
    const float *x_d;
    double ka_dx, ka_dy, ka_K_re, ka_K_im;
    /* Optional complex64 copies of s_m_d / s_p_d: the mixed form gathers these (half the
     * bytes) when both are set; NULL: it reads the complex128 series. */
    const float *s_m32_d, *s_p32_d;
    /* Scatterometer mode (sca = 1; the DopSCA generator, dopscasim/dopsca_raw.py:343-520):
     * nx = N_repeat_x * field_nx columns (range blocks, each with its own geometry
     * columns) read the surface fields at column x mod field_nx and row (y + roll) mod ny
     * (the azimuth shift by whole rows); the per-facet scatterer indices ind0_m/p_d are
     * [ny][nx] and read at the rolled row too.  The scene is scaled by (sr0/(sr0 + r))^2,
     * the range bins see r + sr_bin_offset (the sub-pulse delay), the Bragg phase uses
     * 2 k0 c_b cap_t, and the Bragg RCS is evaluated on every call (scat_d unused).
     * The NRCS sums are kept per range block: nrcs_spec_d[nrcs_row][nblk] and
     * nrcs_bragg_d[npol][nrcs_rows][nblk] (float64, +=), nblk = nx / field_nx.
     * az_f32 = 1: the azimuth residual az_now is a float32 value and the row azimuth is the
     * float32 difference y - az_now (the reference's numpy promotion when the grid step is
     * float32 and the residual is not a float64 scalar).
     * Requires nch = 1; Kodis or Kirchhoff specular (spec_mode 0 / 1 / 2, the Kirchhoff
     * field at the field column's x, scaled like the Kodis one); the LUT mode reads the table of the column's
     * range block (lut_block); hMTF (use_hmtf) is read at the rolled
     * row of the [ny][field_nx] surface and not clipped (the DopSCA generator's weighting,
     * dopsca_raw.py:461-472).  The scene batch rejects it. */
    int32_t sca;
    int32_t field_nx, roll;
    double sr_bin_offset, cap_t;
    int32_t nrcs_row, nrcs_rows;
    int32_t az_f32;
    /* SKIM mode (skim = 1; the SKIM generator, radarsim/skim_raw.py:465-689): sin_az =
     * az / sr per facet (sr_col_d holds absolute slant ranges), the two-way antenna pattern
     * per facet (ant_l_tx / ant_l_rx: transmit / receive lengths, power units), a 10-tap
     * pulse (sinc_d: calc_sinc_vec(10, 20, Fs)), and the facets of every skim_ny_integ rows
     * accumulated into their own row: raw_d is [npol][az_steps][ny / skim_ny_integ][nbins]
     * (skim_ny_integ = ny: one row per pulse).  skim_az2: az/2 sin_az is part of the phase
     * range (the single-scale form); skim_rcm: it is added to the range bins only.
     * skim_ny_integ must divide ny and, when below ny, be a power of two above 64.  Requires
     * nch = 1; Kodis or Kirchhoff specular; direct or LUT Bragg model.  The scene batch
     * rejects it. */
    int32_t skim, skim_ny_integ, skim_az2, skim_rcm;
    /* Mixed form only, optional: complex64 [npol*nch][nbins] compensation row.  The
     * rounding errors of the compensated adds into the raw row collect here and are folded
     * into the raw row by the next pulse's launch or by ocs_pulse_flush.  NULL: the raw row
     * is accumulated with plain float32 atomics. */
    void *raw_lo_d;
    /* SKIM calibration target (oceansar/radarsim/skim_raw.py:151-164, 490-493, 608-615):
     * pt_mode 0 none, 1 floating, 2 fixed.  The scene value of facet (pt_y, pt_x) becomes
     * pt_amp exp(-2 i k0 r) of its phase range r (before the antenna pattern); a fixed
     * target also takes that facet's displacements Dx, Dy, Dz as zero.  SKIM mode only. */
    int32_t pt_mode, pt_x, pt_y;
    double pt_amp;
    /* Scatterometer mode with the Romeiser LUT: elements between the tables of consecutive
     * range blocks in lut_d (the DopSCA generator builds one table per block at the block's
     * mean incidence, dopsca_raw.py:329-356); 0: one table for every block. */
    int64_t lut_block;
} ocs_pulse_desc;

/* Workspace of ocs_pulse (per-pulse float64 and float32 tables of the row quantities and
 * a 16-byte header); < 0 on invalid sizes.  Reset it with ocs_pulse_reset before the
 * first pulse of a scene. */
int64_t ocs_pulse_workspace_bytes(int32_t ny, int32_t nch);

/* Accumulate one pulse into raw_d.
 * OCS_PREC_F64: the float64 drop-in (every facet's slant range, bins and phase in float64
 * in the reference's order).
 * OCS_PREC_MIXED: for SAR scenes with Kodis specular and / or Bragg scattering, nx a
 * multiple of 4 and 16-byte aligned inputs, the split-range form: float64 only for each
 * pulse row's and each column's reference range (reduced 2 k0 R mod 2 pi and the range-bin
 * position, split into float32 hi + lo); each facet's range offset, bin, phase, NRCS and
 * scene in float32, with the float64 decision only for facets within the float32 error
 * bound of a rounding boundary (so bins, LUT indices and specular facet selection equal the
 * float64 form's); compensated float32 accumulation (see raw_lo_d).  Other mixed-precision
 * pulses (Kirchhoff specular, DopSCA, SKIM) keep the facet's slant range, bins and phase
 * reduction in float64. */
int ocs_pulse(const ocs_pulse_desc *desc, int precision, void *stream);

/* Reset the workspace header (pending compensation row, error flag) and zero raw_lo_d;
 * enqueued on `stream`. */
int ocs_pulse_reset(const ocs_pulse_desc *desc, void *stream);

/* Fold the compensation row of the last mixed-precision pulse into its raw row; call
 * after a scene's last pulse (or before reading raw_d).  Enqueued on `stream`. */
int ocs_pulse_flush(const ocs_pulse_desc *desc, void *stream);

/* OCS_ERR_TIMEOUT if a bounded device-side wait of the mixed kernel gave up since the last
 * reset, else OCS_OK.  Synchronises with the device. */
int ocs_pulse_error(const ocs_pulse_desc *desc);

/* SKIM two-scale Doppler (upsample_and_dopplerize, oceansar/radarsim/skim_raw.py:51-81):
 * the step profiles x_d (complex128 [N][G][R]: N simulated steps, G row groups, R range
 * bins) up-sampled by n_up as the reference's zero-padded spectrum does (band-limited
 * interpolation with the period-M Dirichlet kernel, M = N n_up) and modulated by each
 * group's Doppler dop_d (float64 [G][R]) at t = m / prf, summed over the groups into y_d
 * (complex128 [M][R]).  D_d: complex128 [M] scratch.  Float64 throughout. */
int ocs_skim_upsample(const double *x_d, const double *dop_d, double *y_d, double *D_d, int32_t N, int32_t G,
                      int32_t R, int32_t n_up, double prf, void *stream);

/* Complex128 power-of-two FFTs of the SAR processor (the transforms of sar_focus,
 * oceansar/radarsim/sar_processor.py:170, 176, 217, whose sizes optimize_fftsize pads to
 * powers of two).  ocs_fft64_rows: in-place transform of nrows contiguous rows of length
 * n, forward (inverse = 0, exp(-2 pi i k m / n)) or inverse (inverse = 1, exp(+...) and
 * 1/n), as numpy.fft; n <= 8192 needs no scratch, longer rows (four-step) need
 * ocs_fft64_workspace_bytes(nrows, n) bytes of scratch (-1: n not a power of two).
 * ocs_transpose_c128: dst[b][c][r] = src[b][r][c] for batch rows x cols matrices (the
 * azimuth transforms of a [pol][az][rg] cube run as row transforms of its transpose). */
int64_t ocs_fft64_workspace_bytes(int64_t nrows, int64_t n);
int ocs_fft64_rows(double *data, int64_t nrows, int64_t n, int32_t inverse, double *scratch, void *stream);
int ocs_transpose_c128(const double *src, double *dst, int64_t batch, int64_t rows, int64_t cols, void *stream);

/* Arithmetic-rate probe (no reference counterpart; a diagnostic of the device the two
 * precision forms run on): `blocks` x `threads` threads each run iters x 8 independent
 * FMAs in float64 (kind 0), float32 (kind 1) or packed float32x2 (kind 2, two FMAs per
 * instruction).  sink: >= blocks floats, not written in practice.  The caller times the
 * launch on `stream`. */
int ocs_fma_rate(int32_t kind, int32_t blocks, int32_t threads, int32_t iters, float *sink, void *stream);

/* ------------------------------------------------------------------------------------
 * Standalone NRCS models (float64).
 *
 * ocs_rcs_romeiser replaces RCSRomeiser97.rcs / rcs_numba (oceansar/nrcs/romeiser97.py:
 * 95-107, 252-393) on a [ny][nx] grid: out_*_d[l][y][x] is the RCS of Bragg line l.
 * Azimuth and incidence angles are read at az_d[y*az_row_stride + x*az_col_stride] (and
 * likewise inc_d), so a [ny] column vector uses strides (1, 0) and a [nx] row (0, 1).
 */
typedef struct {
    int32_t nx, ny;
    const double *az_d;  int64_t az_row_stride, az_col_stride;
    const double *inc_d; int64_t inc_row_stride, inc_col_stride;
    const double *diffx_d, *diffy_d;     /* float64 [ny][nx] slopes                          */
    double k0, d, dx, dy, wind_dir, wind_U;
    int32_t pol, spread;                 /* OCS_POL_*, OCS_SPREAD_*                          */
    double spread_ck_p, spread_ck_m, spread_a0, spread_ap, spread_am;
    const double *spec_k_d, *spec_s_d;   /* omni-directional spectrum table                  */
    int32_t spec_n;
    double sqrt_eps_re, sqrt_eps_im;
    double *out_hh_d, *out_vv_d;         /* float64 [2][ny][nx] each, or NULL                */
} ocs_rcs_desc;

int ocs_rcs_romeiser(const ocs_rcs_desc *desc, void *stream);

/* ocs_field_kodis replaces RCSKodis.field (oceansar/nrcs/kodis.py:38-73): complex128
 * [ny][nx] specular field for float32 slopes / curvatures and float64 slant range. */
typedef struct {
    int32_t nx, ny;
    const double *az_d; int64_t az_row_stride, az_col_stride;
    const double *sin_inc_d, *cos_inc_d, *tan_inc_d;   /* float64 [nx]                       */
    const double *sr_d;                                /* float64 [ny][nx]                   */
    const float *diffx_d, *diffy_d, *diffxx_d, *diffyy_d, *diffxy_d;
    double k0, R_re, R_im;
    double dx, dy;                                     /* facet sizes (stationary-point window) */
    double *out_d;                                     /* complex128 [ny][nx]                */
} ocs_kodis_desc;

int ocs_field_kodis(const ocs_kodis_desc *desc, void *stream);

/* ocs_field_ka replaces RCSKA.field (oceansar/nrcs/ka.py:110-284), monostatic: complex128
 * [ny][nx] Kirchhoff-approximation field by the facet approach (mode 0) or the stationary-
 * phase approximation (mode 1) for incident / scattered polarisations pol_i, pol_s (0 = h,
 * 1 = v).  theta / phi are broadcast to the grid through their strides (elements). */
typedef struct {
    int32_t nx, ny;
    const double *x_d, *y_d;                           /* float64 [nx], [ny] facet positions   */
    const double *theta_d; int64_t theta_row_stride, theta_col_stride;   /* incidence [rad]  */
    const double *phi_d; int64_t phi_row_stride, phi_col_stride;         /* azimuth [rad]    */
    const float *dz_d, *diffx_d, *diffy_d;             /* float32 [ny][nx]                     */
    const float *diffxx_d, *diffyy_d, *diffxy_d;       /* float32 [ny][nx] (mode 1 only)       */
    double k0, dx, dy;
    double K_re, K_im;                                 /* -1j k0 exp(-1j k0 (R_i+R_s)) / ((4 pi)^2 R_i R_s) */
    int32_t mode, pol_i, pol_s;
    double *out_d;                                     /* complex128 [ny][nx]                  */
} ocs_ka_desc;

int ocs_field_ka(const ocs_ka_desc *desc, void *stream);

/* Range-Doppler focusing (sar_focus, oceansar/radarsim/sar_processor.py:30-274): the phase
 * multiplications between its FFTs, on complex128 data [npol][naz][nrg] in place.
 * ocs_rd_rcmc: range-cell-migration correction in the 2-D frequency domain, data *=
 * exp(1j (4 pi rcmc[a] / c) fr[r]) (:170-176).  ocs_rd_azfilter: azimuth compression
 * filter, data *= h[a] with h = exp(1j ph_ac) weighting (:213-217; h complex128 [naz]). */
int ocs_rd_rcmc(double *data_d, int64_t npol, int32_t naz, int32_t nrg, const double *rcmc_d,
                const double *fr_d, double c, void *stream);
int ocs_rd_azfilter(double *data_d, int64_t npol, int32_t naz, int32_t nrg, const double *h_d, void *stream);

/* ---- Scene batch ----------------------------------------------------------------------
 * Many independent scenes (any mix of grid sizes, geometries and channel counts) advanced
 * together, one pulse of every scene per step, by persistent kernels that find their work
 * in a device-resident slot table.  Each step is a fixed launch sequence needing no host
 * arguments, so it can be recorded once into a CUDA graph and replayed while scenes enter
 * and leave the slots (as long as the set of grid sizes and output widths in use stays
 * the same).  No counterpart in the reference: its sar_raw
 * (oceansar/radarsim/sar_raw_nompi.py:32-641) runs the same per-pulse body for one scene
 * per call; a slot runs exactly that body (ocs_surface_update + ocs_pulse) at each pulse.
 * SAR scenes with Kodis or Kirchhoff specular (spec_mode 0 / 1 / 2) and Bragg scattering,
 * linear or choppy surfaces; Kirchhoff scenes form launch classes of their own, choppy
 * scenes add one launch per step; DopSCA and SKIM pulses are rejected. */
typedef struct {
    const ocs_surface_desc *surface;   /* as for ocs_surface_update; t, add and swell_rot are
                                          taken per pulse from the tables below           */
    const ocs_pulse_desc *pulse;       /* as for ocs_pulse (az_step = 0); az_step, az_now,
                                          tind and refresh are taken from the tables below */
    int32_t tile_rows;                 /* facet rows per pulse-kernel tile, 1..128 (0: 64) */
    const float *t_d;                  /* [az_steps] float32 surface time of each pulse     */
    const float *add_d;                /* [az_steps][surface->nfields] additive terms       */
    const float *swell_rot_d;          /* [az_steps][2] exp(-i w_s t), or NULL              */
    const double *az_now_d;            /* [az_steps] platform azimuth position              */
    const int32_t *flags_d;            /* [az_steps] 1: synthesise the surface, 2: refresh
                                          the Bragg RCS at this pulse                       */
    const int32_t *tmod_d;             /* [az_steps][2] int(t prf) mod N_m, mod N_p         */
    const ocs_choppy_desc *choppy;     /* choppy surfaces: the slope / curvature step run
                                          after the column pass (ocs_surface_choppy; its
                                          swell_rot is taken per pulse from swell_rot_d);
                                          NULL for linear surfaces                          */
} ocs_scene_desc;

typedef struct ocs_batch ocs_batch;    /* opaque engine handle                              */

/* Engine with max_slots (1..256) scene slots for one precision (OCS_PREC_*). */
int ocs_batch_create(int32_t max_slots, int32_t precision, ocs_batch **out);
int ocs_batch_destroy(ocs_batch *batch);
/* Put a scene in a slot with its pulse counter at 0 (the caller zeroes its raw cube and
 * NRCS accumulators).  Ordered on the stream (steps enqueued after it see the scene);
 * returns without waiting for the stream. */
int ocs_batch_set(ocs_batch *batch, int32_t slot, const ocs_scene_desc *scene, void *stream);
/* Take the scene out of a slot.  Ordered on the stream; returns without waiting for it. */
int ocs_batch_clear(ocs_batch *batch, int32_t slot, void *stream);
/* Enqueue `pulses` steps: every slot whose counter is below its az_steps runs one pulse per
 * step; finished and empty slots cost nothing. */
int ocs_batch_step(ocs_batch *batch, int32_t pulses, void *stream);
/* Kernel launches one step enqueues for the slots in use. */
int ocs_batch_launches_per_step(const ocs_batch *batch);
/* Pulse counter of every slot (-1 for empty slots) into out[max_slots]; synchronous. */
int ocs_batch_counters(const ocs_batch *batch, int32_t *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* OCEANSAR_B200_H */
