// Standalone NRCS kernels: the drop-ins for RCSRomeiser97.rcs (oceansar/nrcs/romeiser97.py:
// 95-107 -> rcs_numba :324-393) and RCSKodis.field (oceansar/nrcs/kodis.py:38-73) when they
// are called directly rather than from inside the fused pulse kernel.  Both evaluate the
// per-facet physics of physics.cuh in float64 over a [ny][nx] grid whose azimuth and
// incidence angles broadcast along rows / columns through explicit strides.
#include <string.h>

#include "physics.cuh"

namespace ocs {

struct RcsArgs {
    int nx, ny;
    const double *az;
    long long az_rs, az_cs;
    const double *inc;
    long long inc_rs, inc_cs;
    const double *diffx, *diffy;
    RomeiserParams rom;
    double *out_hh, *out_vv;        // [2][ny][nx] or null
};

__global__ void rcs_kernel(const __grid_constant__ RcsArgs a) {
    const long long n = (long long)a.nx * a.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / a.nx, c = i - r * a.nx;
        const double az = a.az[r * a.az_rs + c * a.az_cs];
        const double inc = a.inc[r * a.inc_rs + c * a.inc_cs];
        double hh[2], vv[2];
        romeiser_facet<double>(a.rom, inc, az, cos(az), sin(az), a.diffx[i], a.diffy[i], hh, vv);
        if (a.out_hh) { a.out_hh[i] = hh[0]; a.out_hh[n + i] = hh[1]; }
        if (a.out_vv) { a.out_vv[i] = vv[0]; a.out_vv[n + i] = vv[1]; }
    }
}

struct KodisArgs {
    int nx, ny;
    const double *az;
    long long az_rs, az_cs;
    const double *sin_inc, *cos_inc, *tan_inc;     // [nx]
    const double *sr;                              // [ny][nx]
    const float *diffx, *diffy, *diffxx, *diffyy, *diffxy;
    KodisParams kp;
    double *out;                                   // complex128 [ny][nx]
};

__global__ void kodis_kernel(const __grid_constant__ KodisArgs a) {
    const long long n = (long long)a.nx * a.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / a.nx, c = i - r * a.nx;
        const double az = a.az[r * a.az_rs + c * a.az_cs];
        const c128 e = kodis_facet<double>(a.kp, a.sr[i], a.sin_inc[c], a.cos_inc[c], a.tan_inc[c], cos(az),
                                           sin(az), a.diffx[i], a.diffy[i], a.diffxx[i], a.diffyy[i],
                                           a.diffxy[i]);
        a.out[2 * i] = e.re;
        a.out[2 * i + 1] = e.im;
    }
}

}  // namespace ocs

using namespace ocs;

extern "C" int ocs_rcs_romeiser(const ocs_rcs_desc *d, void *stream) {
    if (!d || d->nx < 1 || d->ny < 1 || !d->az_d || !d->inc_d || !d->diffx_d || !d->diffy_d) return OCS_ERR_ARG;
    if (!d->out_hh_d && !d->out_vv_d) return OCS_ERR_ARG;
    if (!d->spec_k_d || !d->spec_s_d || d->spec_n < 2) return OCS_ERR_ARG;
    RcsArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = d->nx; a.ny = d->ny;
    a.az = d->az_d; a.az_rs = d->az_row_stride; a.az_cs = d->az_col_stride;
    a.inc = d->inc_d; a.inc_rs = d->inc_row_stride; a.inc_cs = d->inc_col_stride;
    a.diffx = d->diffx_d; a.diffy = d->diffy_d;
    RomeiserParams &r = a.rom;
    r.k0 = d->k0; r.d = d->d; r.dx = d->dx; r.dy = d->dy; r.wind_dir = d->wind_dir; r.wind_U = d->wind_U;
    r.pol = d->pol; r.spread = d->spread;
    r.ck_p = d->spread_ck_p; r.ck_m = d->spread_ck_m; r.a0 = d->spread_a0; r.ap = d->spread_ap;
    r.am = d->spread_am;
    r.tab_k = d->spec_k_d; r.tab_s = d->spec_s_d; r.tab_n = d->spec_n;
    r.eps_re = 73.0; r.eps_im = 18.0; r.seps_re = d->sqrt_eps_re; r.seps_im = d->sqrt_eps_im;
    r.eps2_re = 73.0 * 73.0 - 18.0 * 18.0; r.eps2_im = 2.0 * 73.0 * 18.0;
    a.out_hh = d->out_hh_d; a.out_vv = d->out_vv_d;
    long long n = (long long)d->nx * d->ny;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    rcs_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

extern "C" int ocs_field_kodis(const ocs_kodis_desc *d, void *stream) {
    if (!d || d->nx < 1 || d->ny < 1 || !d->az_d || !d->sr_d || !d->sin_inc_d || !d->cos_inc_d ||
        !d->tan_inc_d || !d->diffx_d || !d->diffy_d || !d->diffxx_d || !d->diffyy_d || !d->diffxy_d ||
        !d->out_d)
        return OCS_ERR_ARG;
    KodisArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = d->nx; a.ny = d->ny;
    a.az = d->az_d; a.az_rs = d->az_row_stride; a.az_cs = d->az_col_stride;
    a.sin_inc = d->sin_inc_d; a.cos_inc = d->cos_inc_d; a.tan_inc = d->tan_inc_d;
    a.sr = d->sr_d;
    a.diffx = d->diffx_d; a.diffy = d->diffy_d; a.diffxx = d->diffxx_d; a.diffyy = d->diffyy_d;
    a.diffxy = d->diffxy_d;
    a.kp.k0 = d->k0; a.kp.R_re = d->R_re; a.kp.R_im = d->R_im;
    a.kp.hdx = d->dx * 0.5; a.kp.hdy = d->dy * 0.5;
    a.out = d->out_d;
    long long n = (long long)d->nx * d->ny;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    kodis_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------
// Kirchhoff-approximation specular field (RCSKA.field, oceansar/nrcs/ka.py:110-284).
namespace ocs {
struct KaArgs {
    int nx, ny;
    const double *x, *y;
    const double *theta;
    long long th_rs, th_cs;
    const double *phi;
    long long ph_rs, ph_cs;
    const float *dz, *diffx, *diffy, *diffxx, *diffyy, *diffxy;
    KaParams kp;
    int pol_i, pol_s;
    double *out;
};

__global__ void ka_kernel(const __grid_constant__ KaArgs a) {
    const long long n = (long long)a.nx * a.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / a.nx), c = (int)(i - (long long)r * a.nx);
        const double th = a.theta[r * a.th_rs + c * a.th_cs];
        const double ph = a.phi[r * a.ph_rs + c * a.ph_cs];
        double st, ct, sp, cp;
        sincos(th, &st, &ct);
        sincos(ph, &sp, &cp);
        const c128 e = ka_facet(a.kp, a.pol_i, a.pol_s, a.x[c], a.y[r], st, ct, tan(th), sp, cp, a.dz[i], a.diffx[i],
                                a.diffy[i], a.diffxx[i], a.diffyy[i], a.diffxy[i]);
        a.out[2 * i] = e.re;
        a.out[2 * i + 1] = e.im;
    }
}
}  // namespace ocs

extern "C" int ocs_field_ka(const ocs_ka_desc *d, void *stream) {
    if (!d || d->nx < 1 || d->ny < 1 || !d->x_d || !d->y_d || !d->theta_d || !d->phi_d || !d->dz_d ||
        !d->diffx_d || !d->diffy_d || !d->out_d)
        return OCS_ERR_ARG;
    if (d->mode != 0 && d->mode != 1) return OCS_ERR_ARG;
    if (d->mode == 1 && (!d->diffxx_d || !d->diffyy_d || !d->diffxy_d)) return OCS_ERR_ARG;
    if ((d->pol_i != 0 && d->pol_i != 1) || (d->pol_s != 0 && d->pol_s != 1)) return OCS_ERR_ARG;
    KaArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = d->nx; a.ny = d->ny;
    a.x = d->x_d; a.y = d->y_d;
    a.theta = d->theta_d; a.th_rs = d->theta_row_stride; a.th_cs = d->theta_col_stride;
    a.phi = d->phi_d; a.ph_rs = d->phi_row_stride; a.ph_cs = d->phi_col_stride;
    a.dz = d->dz_d; a.diffx = d->diffx_d; a.diffy = d->diffy_d;
    // the facet approach never reads the curvatures; give it valid pointers anyway
    a.diffxx = d->diffxx_d ? d->diffxx_d : d->diffx_d;
    a.diffyy = d->diffyy_d ? d->diffyy_d : d->diffx_d;
    a.diffxy = d->diffxy_d ? d->diffxy_d : d->diffx_d;
    a.kp.k0 = d->k0; a.kp.dx = d->dx; a.kp.dy = d->dy; a.kp.K_re = d->K_re; a.kp.K_im = d->K_im;
    a.kp.mode = d->mode;
    a.pol_i = d->pol_i; a.pol_s = d->pol_s;
    a.out = d->out_d;
    const long long n = (long long)d->nx * d->ny;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    ka_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? OCS_OK : OCS_ERR_CUDA;
}
