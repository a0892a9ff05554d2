/*
 * Oracle (test infrastructure only): CPU restatement of the OCEANSAR facet-to-range-bin
 * accumulation.  Used by the tests, smoke() and bench.py's CPU-baseline leg as the
 * checker; never linked into the product library.
 *
 * Follows oceansar/radarsim/range_profile.py:
 *   - chan_profile_numba prologue (:103-108): bin_f = (srg - min_sr) / binsize;
 *     bin_d = int32(floor(bin_f)); lut = int32(round_half_even(ovs * (1 - (bin_f - bin_d))))
 *   - profile_integrator (:22-49): for each facet i and tap j < n_samp,
 *     out[bin_d - n_samp/2 + j] += pulse[lut + j*ovs] * scene[i], taps outside
 *     [0, nbins) dropped.  Facets are visited in order, so the sums are bit-identical to
 *     the serial numba loop.  The real weight multiplies the complex scene as the complex
 *     product (w + 0i)(sr + i si), as numba evaluates it, so non-finite scene values
 *     propagate the same way.
 * Complex values are interleaved (re, im) doubles; the sinc table is float32.
 */
#include <math.h>
#include <stdint.h>

/* nearbyint() follows the current rounding mode (round-to-nearest-even by default),
 * which is numpy's np.round rule. */
static inline int32_t lut_index(double bin_f, int32_t bin_d, int ovs)
{
    double frac = bin_f - (double)bin_d;
    double v = (double)ovs * (1.0 - frac);
    return (int32_t)nearbyint(v);
}

void oracle_chan_profile(const double *srg, const double *scene, int64_t n,
                         double binsize, double min_sr,
                         const float *pulse, int n_samp, int ovs,
                         double *out, int64_t nbins)
{
    const int64_t rnbins = nbins - n_samp - 1;
    const int half = n_samp / 2;
    for (int64_t i = 0; i < n; ++i) {
        double bin_f = (srg[i] - min_sr) / binsize;
        int32_t bin_d = (int32_t)floor(bin_f);
        int32_t sbin = lut_index(bin_f, bin_d, ovs);
        int64_t bin_now = (int64_t)bin_d - half;
        const double sr = scene[2 * i], si = scene[2 * i + 1];
        if (bin_now < 0 || bin_now > rnbins) {
            for (int j = 0; j < n_samp; ++j) {
                if (bin_now >= 0 && bin_now < nbins) {
                    double w = (double)pulse[sbin + j * ovs];
                    out[2 * bin_now] += w * sr - 0.0 * si;
                    out[2 * bin_now + 1] += w * si + 0.0 * sr;
                }
                ++bin_now;
            }
        } else {
            for (int j = 0; j < n_samp; ++j) {
                double w = (double)pulse[sbin + j * ovs];
                out[2 * bin_now] += w * sr - 0.0 * si;
                out[2 * bin_now + 1] += w * si + 0.0 * sr;
                ++bin_now;
            }
        }
    }
}

/* Row-wise variant (profile_integrator_1d, range_profile.py:52-80): row a of
 * srg/scene [naz, npts] accumulates into row a of out [naz, nbins]. */
void oracle_chan_profile_rows(const double *srg, const double *scene, int64_t naz, int64_t npts,
                              double binsize, double min_sr,
                              const float *pulse, int n_samp, int ovs,
                              double *out, int64_t nbins)
{
    for (int64_t a = 0; a < naz; ++a)
        oracle_chan_profile(srg + a * npts, scene + 2 * a * npts, npts, binsize, min_sr,
                            pulse, n_samp, ovs, out + 2 * a * nbins, nbins);
}
