/*
 * On-device source generation: seafloor deformation of rectangular faults
 * (Okada 1985) applied to a layer, so a forecast request goes from fault
 * parameters to its initial state without a host upload of the surface.
 *
 * Follows the reference's GET_FLOOR_DEFORM / DEFORM_OKADA / STRIKE_SLIP /
 * DIP_SLIP / STEREO_PROJECTION (deform.f90:2-240, 494-586): per fault, the
 * vertical displacement US + UD of the free surface above a buried
 * dislocation (strike-slip and dip-slip parts, each a four-corner
 * combination F1 - F2 - F3 + F4), with cell positions mapped onto the fault
 * plane by an oblique stereographic projection on the WGS84 ellipsoid
 * (spherical layers) or from the layer origin and spacing (Cartesian
 * layers); non-finite values and |value| <= GX give 0; then Z += DEFORM and
 * H -= DEFORM in fault order.  The reference evaluates in single precision;
 * here every cell is evaluated in double (its float rounding jumps between
 * atan branches on the lines where a fault end is level with the cell) and
 * the per-fault result is rounded to float before it is applied, as the
 * reference's REAL DEFORM array is.
 */
#include <math.h>
#include <string.h>

#include "gc_internal.h"
#include "gcomcot.h"

namespace {

constexpr int MAX_FAULTS_PER_LAUNCH = 12;

/* per-fault constants, evaluated once on the host in double */
struct FaultDev {
    double hh, halfl, w, ang_l, sn, cs, st, ct, ds, dd, del_x, del_y, x0, y0, xl, yl;
};
struct FaultPack {
    int n;
    FaultDev f[MAX_FAULTS_PER_LAUNCH];
};

__host__ __device__ void stereo(double lonin, double latin, double lon0, double lat0, double &xo, double &yo) {
    const double rad = CC_RAD_DEG;
    const double pole = CC_PI / 2.0 - (double)CC_EPS;
    double lat = latin * rad, lon = lonin * rad, lt0 = lat0 * rad, ln0 = lon0 * rad;
    if (lat > pole) lat = pole;
    if (lat < -pole) lat = -pole;
    if (lt0 > pole) lt0 = pole;
    if (lt0 < -pole) lt0 = -pole;
    const double sn = sin(lat), cs0 = cos(lt0), sn0 = sin(lt0);
    const double a = 6378137.0, e = 0.08181919092891, f2 = 0.00669438000426, k0 = 0.9996;
    const double tmp0 = sqrt(1.0 - f2 * (sn0 * sn0));
    const double rho0 = a * (1.0 - f2) / (tmp0 * tmp0 * tmp0);
    /* the reference's NU0 is an INTEGER by implicit typing: truncated */
    const double nu0 = (double)(int)(a / tmp0);
    const double rr = sqrt(rho0 * nu0);
    const double n = sqrt(1.0 + f2 * ((cs0 * cs0) * (cs0 * cs0)) / (1.0 - f2));
    const double s1 = (1.0 + sn0) / (1.0 - sn0);
    const double s2 = (1.0 - e * sn0) / (1.0 + e * sn0);
    const double w1 = pow(s1 * pow(s2, e), n);
    const double sn_xi0 = (w1 - 1.0) / (w1 + 1.0);
    const double c = (n + sn0) * (1.0 - sn_xi0) / (n - sn0) / (1.0 + sn_xi0);
    const double w2 = c * w1;
    const double sa = (1.0 + sn) / (1.0 - sn);
    const double sb = (1.0 - e * sn) / (1.0 + e * sn);
    const double w = c * pow(sa * pow(sb, e), n);
    const double xi0 = asin((w2 - 1.0) / (w2 + 1.0));
    const double lm = n * (lon - ln0) + ln0;
    const double xi = asin((w - 1.0) / (w + 1.0));
    const double beta = 1.0 + sin(xi) * sin(xi0) + cos(xi) * cos(xi0) * cos(lm - ln0);
    yo = 2.0 * rr * k0 * (sin(xi) * cos(xi0) - cos(xi) * sin(xi0) * cos(lm - ln0)) / beta;
    xo = 2.0 * rr * k0 * cos(xi) * sin(lm - ln0) / beta;
}

/* STRIKE_SLIP corner term; x2 is the cell's across-strike coordinate */
__device__ double strike_slip(double y1, double y2, double x2, double sn, double cs, double dd) {
    const double q = x2 * sn - dd * cs;
    const double d_bar = y2 * sn - q * cs;
    const double r = sqrt(y1 * y1 + y2 * y2 + q * q);
    double t1 = r + d_bar, t2 = r + y2;
    if (t1 <= 1.0e-10) t1 = 1.0e-10;
    if (t2 <= 1.0e-10) t2 = 1.0e-10;
    const double a4 = 0.5 / cs * (log(t1) - sn * log(t2));
    return -(d_bar * q / r / (r + y2) + q * sn / (r + y2) + a4 * sn) / 2.0 / 3.14159;
}

/* DIP_SLIP corner term */
__device__ double dip_slip(double y1, double y2, double x2, double sn, double cs, double dd) {
    const double q = x2 * sn - dd * cs;
    const double d_bar = y2 * sn - q * cs;
    const double r = sqrt(y1 * y1 + y2 * y2 + q * q);
    const double xx = sqrt(y1 * y1 + q * q);
    const double a5 = 1.0 / cs * atan((y2 * (xx + q * cs) + xx * (r + xx) * sn) / y1 / (r + xx) / cs);
    return -(d_bar * q / r / (r + y1) + sn * atan(y1 * y2 / q / r) - a5 * sn * cs) / 2.0 / 3.14159;
}

__device__ float deform_cell(const FaultDev &f, int laycord, int i, int j, const float *x, const float *y, float dx,
                             float dy) {
    double xs, ys;
    if (laycord == 0) {
        stereo((double)x[i], (double)y[j], f.x0, f.y0, xs, ys);
        xs = xs - f.del_x;
        ys = ys + f.del_y;
    } else {
        const double yy = (double)dy * (double)j, xx = (double)dx * (double)i;
        xs = xx - f.xl - f.del_x;
        ys = yy - f.yl + f.del_y;
    }
    const double x1 = xs * f.st + ys * f.ct;
    const double x2 = -(xs * f.ct - ys * f.st);
    const double p = x2 * f.cs + f.hh * f.sn;
    const double f1 = strike_slip(x1 + f.halfl, p, x2, f.sn, f.cs, f.hh);
    const double f2 = strike_slip(x1 + f.halfl, p - f.w, x2, f.sn, f.cs, f.hh);
    const double f3 = strike_slip(x1 - f.halfl, p, x2, f.sn, f.cs, f.hh);
    const double f4 = strike_slip(x1 - f.halfl, p - f.w, x2, f.sn, f.cs, f.hh);
    const double g1 = dip_slip(x1 + f.halfl, p, x2, f.sn, f.cs, f.hh);
    const double g2 = dip_slip(x1 + f.halfl, p - f.w, x2, f.sn, f.cs, f.hh);
    const double g3 = dip_slip(x1 - f.halfl, p, x2, f.sn, f.cs, f.hh);
    const double g4 = dip_slip(x1 - f.halfl, p - f.w, x2, f.sn, f.cs, f.hh);
    double us = (f1 - f2 - f3 + f4) * f.ds;
    double ud = (g1 - g2 - g3 + g4) * f.dd;
    if (!isfinite(us)) us = 0.0;
    if (!isfinite(ud)) ud = 0.0;
    if (fabs(us) <= (double)CC_GX) us = 0.0;
    if (fabs(ud) <= (double)CC_GX) ud = 0.0;
    return (float)(us + ud);
}

__global__ void k_okada(FaultPack pk, int laycord, int nx, int ny, int pitch, const float *x, const float *y, float dx,
                        float dy, float *z, float *h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nx || j >= ny) return;
    const size_t c = (size_t)j * pitch + i;
    float zc = z ? z[c] : 0.0f, hc = h ? h[c] : 0.0f;
    for (int k = 0; k < pk.n; k++) {
        const float d = deform_cell(pk.f[k], laycord, i, j, x, y, dx, dy);
        zc = zc + d;
        hc = hc - d;
    }
    if (z) z[c] = zc;
    if (h) h[c] = hc;
}

FaultDev prepare_fault(const gc_fault &in, int laycord) {
    FaultDev f;
    const double rad = CC_RAD_DEG;
    const double ang_l = rad * in.dl, ang_r = rad * in.rd, ang_t = rad * in.th;
    f.halfl = 0.5 * in.l;
    f.w = in.w;
    if (in.sw == 9) {
        f.hh = in.hh + in.w * sin(ang_l);
        f.del_x = in.w * cos(ang_l) * cos(ang_t);
        f.del_y = in.w * cos(ang_l) * sin(ang_t);
    } else {
        f.hh = in.hh + 0.5 * in.w * sin(ang_l);
        f.del_x = 0.5 * in.w * cos(ang_l) * cos(ang_t);
        f.del_y = 0.5 * in.w * cos(ang_l) * sin(ang_t);
    }
    f.ang_l = ang_l;
    f.ds = in.d * cos(ang_r);
    f.dd = in.d * sin(ang_r);
    f.sn = sin(ang_l);
    f.cs = cos(ang_l);
    f.st = sin(ang_t);
    f.ct = cos(ang_t);
    f.x0 = in.x0;
    f.y0 = in.y0;
    f.xl = f.yl = 0.0;
    if (laycord != 0) stereo(in.xo, in.yo, in.x0, in.y0, f.xl, f.yl);
    return f;
}

} // namespace

extern "C" {

int gc_okada_apply(const gc_fault *faults, int nf, int laycord, int nx, int ny, int pitch, const float *d_x,
                   const float *d_y, float dx, float dy, float *d_z, float *d_h, void *stream) {
    if (!faults || nf < 0 || nx < 1 || ny < 1 || pitch < nx || (laycord != 0 && laycord != 1)) return GC_EINVAL;
    if (laycord == 0 && (!d_x || !d_y)) return GC_EINVAL;
    for (int k = 0; k < nf; k++)
        if (faults[k].sw != 0 && faults[k].sw != 9) return GC_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    for (int k0 = 0; k0 < nf; k0 += MAX_FAULTS_PER_LAUNCH) {
        FaultPack pk;
        memset(&pk, 0, sizeof pk);
        pk.n = nf - k0 < MAX_FAULTS_PER_LAUNCH ? nf - k0 : MAX_FAULTS_PER_LAUNCH;
        for (int k = 0; k < pk.n; k++) pk.f[k] = prepare_fault(faults[k0 + k], laycord);
        dim3 grid((unsigned)((nx + 127) / 128), (unsigned)ny, 1);
        k_okada<<<grid, 128, 0, s>>>(pk, laycord, nx, ny, pitch, d_x, d_y, dx, dy, d_z, d_h);
        GC_CUDA_OR_RET(cudaGetLastError());
    }
    return GC_OK;
}

} /* extern "C" */
