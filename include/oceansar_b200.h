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

#ifdef __cplusplus
}
#endif

#endif /* OCEANSAR_B200_H */
