// forcing.cuh -- time-varying current and wind (WindAndCurrentInterpolator::SetTime,
// windandcurrentinterpolator.cpp:66-70, which the reference leaves unfinished,
// and get_wind_vector, kernels.cuh:580-622, which it keeps commented out).
//
// Two current frames a, b (vx block then vy block, as icempm_set_current) and
// a coarse wind grid of rows x cols samples {u_a, v_a, u_b, v_b} (the
// reference's wgrid[lat][lon][4]: row along y, column along x, spacing `cell`,
// sample (r, c) at world (x0 + c cell, y0 + r cell)) stay on the device.
// k_blend_forcing sets, for every node at world (x h, y h):
//   current = (1 - tc) a + tc b,
//   wind    = (1 - tw) W_a + tw W_b,  W bilinear in the four samples around
//             the node (weights (1-u)(1-v), u(1-v), (1-u)v, uv of the node's
//             position inside its wind cell; nodes outside the wind grid take
//             the nearest edge),
// and writes the current into the compat current table and {current, wind
// stress rho_a C_a |U| U} into the extended forcing table.  Every double
// operation is written with an explicit rounding (no contraction into FMA),
// so the tables equal a plain IEEE evaluation in the same order.
#pragma once
#include "engine.cuh"

namespace icempm {

struct WindGrid {
    const float4 *w;      // rows * cols samples, row-major; nullptr: keep the static wind stress
    int rows, cols;
    double cell, x0, y0;
};

// Wind at world (X, Y): bilinear in space, then linear in time.
__device__ __forceinline__ void wind_sample(const WindGrid &g, double X, double Y, double tw, double &ux,
                                            double &uy)
{
    double u = __ddiv_rn(__dsub_rn(X, g.x0), g.cell);
    double v = __ddiv_rn(__dsub_rn(Y, g.y0), g.cell);
    u = fmin(fmax(u, 0.0), (double)(g.cols - 1));
    v = fmin(fmax(v, 0.0), (double)(g.rows - 1));
    const int c = min((int)u, max(g.cols - 2, 0)), r = min((int)v, max(g.rows - 2, 0));
    const int c1 = min(c + 1, g.cols - 1), r1 = min(r + 1, g.rows - 1);
    const double ub = __dsub_rn(u, (double)c), vb = __dsub_rn(v, (double)r);
    const double w00 = __dmul_rn(__dsub_rn(1.0, ub), __dsub_rn(1.0, vb));
    const double w01 = __dmul_rn(ub, __dsub_rn(1.0, vb));
    const double w10 = __dmul_rn(__dsub_rn(1.0, ub), vb);
    const double w11 = __dmul_rn(ub, vb);
    const float4 s00 = g.w[(size_t)r * g.cols + c], s01 = g.w[(size_t)r * g.cols + c1];
    const float4 s10 = g.w[(size_t)r1 * g.cols + c], s11 = g.w[(size_t)r1 * g.cols + c1];
    auto bil = [&](float a, float b, float cc, float d) {
        return __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(w00, (double)a), __dmul_rn(w01, (double)b)),
                                   __dmul_rn(w10, (double)cc)),
                         __dmul_rn(w11, (double)d));
    };
    const double uxa = bil(s00.x, s01.x, s10.x, s11.x), uya = bil(s00.y, s01.y, s10.y, s11.y);
    const double uxb = bil(s00.z, s01.z, s10.z, s11.z), uyb = bil(s00.w, s01.w, s10.w, s11.w);
    ux = __dadd_rn(__dmul_rn(__dsub_rn(1.0, tw), uxa), __dmul_rn(tw, uxb));
    uy = __dadd_rn(__dmul_rn(__dsub_rn(1.0, tw), uya), __dmul_rn(tw, uyb));
}

template <class Real>
__global__ void __launch_bounds__(256) k_blend_forcing(long long G, int gy, double h, const double *__restrict__ ca_,
                                                       const double *__restrict__ cb_, double tc, WindGrid wg,
                                                       double tw, double air_ca, V2<Real> *cur, V4<Real> *frc)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= G) return;
    V4<Real> f = frc[i];
    if (ca_) {
        const double t1 = __dsub_rn(1.0, tc);
        const double cx = __dadd_rn(__dmul_rn(t1, ca_[i]), __dmul_rn(tc, cb_[i]));
        const double cy = __dadd_rn(__dmul_rn(t1, ca_[G + i]), __dmul_rn(tc, cb_[G + i]));
        V2<Real> c;
        c.x = Real(cx); c.y = Real(cy);
        cur[i] = c;
        f.x = Real(cx); f.y = Real(cy);
    }
    if (wg.w) {
        const double X = __dmul_rn((double)(i / gy), h), Y = __dmul_rn((double)(i % gy), h);
        double ux, uy;
        wind_sample(wg, X, Y, tw, ux, uy);
        const double um = __dsqrt_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)));
        const double k = __dmul_rn(air_ca, um);
        f.z = Real(__dmul_rn(k, ux));
        f.w = Real(__dmul_rn(k, uy));
    }
    frc[i] = f;
}

}  // namespace icempm
