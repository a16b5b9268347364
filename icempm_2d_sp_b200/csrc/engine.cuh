// engine.cuh -- device data layout, kernels and the per-variant engine of the
// B200-native 2D APIC MPM step.
//
// Step structure.  The reference runs, per sub-step, reset_grid -> P2G ->
// update_nodes -> G2P (model.cpp:18-39, gpu_partition.cpp:300-365).  Here G2P
// of step k and P2G of step k+1 are one kernel (k_g2p_p2g): the point state is
// read once and written once per step, and the scatter of step k+1 uses the
// state that G2P just produced in registers.  The grid update (k_grid_update)
// turns the accumulators into velocities and clears them for the next scatter,
// which replaces the per-step memset.  A standalone P2G (k_p2g) primes the
// accumulators after an upload or a parameter change.
//
// Point layout (one entry per point, SoA of 16-byte vectors, 128-bit loads):
//   A   {x, y, Jp_inv, thickness}  x, y cell-local in [-0.5, 0.5]
//   H   {H00, H01, H10, H11}       H = Fe - I
//   K   {cell, utility}            cell = (y << 16) | x, utility flags
//   V   {vx, vy}                   written each step, read only when priming
//   C   {C00, C01, C10, C11}       APIC affine matrix (the reference's Bp)
//   PQ  {P, Q}                     written on record steps only
//   slot, pid, thick64             host slot, point id row, f64 thickness
// Grid layout (node = y + x*GridY, the reference order):
//   acc {mass, px, py, area}       accumulators (int64 fixed point, f32 or f64)
//   vel {vx, vy}                   grid velocity after the update
//   status (u8), cur {vx, vy}, force {fx, fy} (f64, boundary reaction)
#pragma once
#include <cstdint>
#include <cstring>
#include <climits>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include "device_math.cuh"
#include "../../include/icempm.h"

namespace icempm {

template <class T> struct alignas(16) V4 { T x, y, z, w; };
template <class T> struct alignas(2 * sizeof(T) > 16 ? 16 : 2 * sizeof(T)) V2 { T x, y; };
template <class A> struct alignas(16) Acc4 { A m, px, py, area; };

struct DevStatus {
    uint32_t err;
    int32_t disabled;
    int32_t step;
    uint32_t done;        // CTA completion ticket of the fused kernel
    int32_t n_active;     // result slot of the compaction boundary search
    int32_t pad[3];
};

template <class Real> struct Pts {
    V4<Real> *A, *H, *C;
    V2<Real> *V, *PQ;
    uint2 *K;
    uint32_t *slot, *pid;
    double *thick64;
};

template <class Real, class Acc> struct Grid {
    Acc4<Acc> *acc;
    V2<Real> *vel;
    V2<Real> *cur;
    const uint8_t *status;
    double2 *force;
};

// Values the kernels read, prepared on the host from SimParams and the options.
template <class Real> struct KParams {
    int gx, gy, update_every;
    int forcing, wind_kind;
    Real h, h_inv, dt, dt_h_inv, four_h_inv, vmax2_01, particle_mass, dt_vol_Dpinv, particle_volume;
    double dt_d;                    // InitialTimeStep (double) for the simulation time
    double kL, kQ;                  // effective drag coefficients * dt (compat)
    double scale_m, scale_p, scale_a;           // fixed point: value * scale -> int64
    double inv_scale_m, inv_scale_p, inv_scale_a;
    double lim_m, lim_p;            // largest |value| a single term may carry in fixed point
    double rho_w_cd_dt, rho_a_ca_dt;            // extended forcing
    double wind_u, wind_v, wind_cx, wind_cy, wind_vmax, wind_radius;
    Material mat;
};

// ---- accumulator conversions -------------------------------------------
template <class Acc> struct AccOps;
template <> struct AccOps<long long> {
    template <class Real>
    static __device__ __forceinline__ long long from(Real v, double scale) {
        return (long long)__double2ll_rn(double(v) * scale);
    }
    template <class Real>
    static __device__ __forceinline__ Real to(long long v, double inv_scale) {
        return Real(double(v) * inv_scale);
    }
    static __device__ __forceinline__ void add_shared(long long *a, long long v) {
        atomicAdd(reinterpret_cast<unsigned long long *>(a), (unsigned long long)v);
    }
    static __device__ __forceinline__ void add_global(long long *a, long long v) {
        atomicAdd(reinterpret_cast<unsigned long long *>(a), (unsigned long long)v);
    }
};
template <> struct AccOps<float> {
    template <class Real> static __device__ __forceinline__ float from(Real v, double) { return float(v); }
    template <class Real> static __device__ __forceinline__ Real to(float v, double) { return Real(v); }
    static __device__ __forceinline__ void add_shared(float *a, float v) { atomicAdd(a, v); }
    static __device__ __forceinline__ void add_global(float *a, float v) { atomicAdd(a, v); }
};
template <> struct AccOps<double> {
    template <class Real> static __device__ __forceinline__ double from(Real v, double) { return double(v); }
    template <class Real> static __device__ __forceinline__ Real to(double v, double) { return Real(v); }
    static __device__ __forceinline__ void add_shared(double *a, double v) { atomicAdd(a, v); }
    static __device__ __forceinline__ void add_global(double *a, double v) { atomicAdd(a, v); }
};

__device__ __forceinline__ void warp_flush_status(DevStatus *st, uint32_t err, int ndis)
{
    const uint32_t e = __reduce_or_sync(0xffffffffu, err);
    const int d = (int)__reduce_add_sync(0xffffffffu, (unsigned)ndis);
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicOr(&st->err, e);
        if (d) atomicAdd(&st->disabled, d);
    }
}

// ---- P2G sources of one point --------------------------------------------
// The reference scatters, for node offsets (i, j) in {-1,0,1}^2 (kernels.cuh:76-95)
//   dM = w m_p,   dP = w (m_p v + S (i - x, j - y) h),
//   S = m_p C - dt_vol_Dpinv Jp_inv thickness tau.
// With A = m_p v - h S (x, y):  dP = w (A + h S (i, j)).
template <class Real> struct Src {
    bool active;
    int cx, cy;
    Real wx[3], wy[3];
    Real mp, ax, ay, s00, s01, s10, s11, area;
};

template <class Real>
__device__ __forceinline__ void make_src(const KParams<Real> &kp, Src<Real> &s, Real x, Real y, Real Jp,
                                         Real thick, const M2<Real> &H, Real vx, Real vy, Real c00,
                                         Real c01, Real c10, Real c11)
{
    const Kin<Real> k = kinematics(H);
    const M2<Real> tau = kirchhoff(k, Real(kp.mat.mu), Real(kp.mat.kappa));
    const Real mp = kp.particle_mass * thick;
    const Real sc = kp.dt_vol_Dpinv * Jp * thick;
    const Real S00 = mp * c00 - sc * tau.a00, S01 = mp * c01 - sc * tau.a01;
    const Real S10 = mp * c10 - sc * tau.a10, S11 = mp * c11 - sc * tau.a11;
    s.mp = mp;
    s.ax = mp * vx - kp.h * (S00 * x + S01 * y);
    s.ay = mp * vy - kp.h * (S10 * x + S11 * y);
    s.s00 = kp.h * S00; s.s01 = kp.h * S01; s.s10 = kp.h * S10; s.s11 = kp.h * S11;
    s.area = kp.particle_volume;
    bspline(x, s.wx);
    bspline(y, s.wy);
}

// ---- block-level scatter ---------------------------------------------------
// 1. the block's bounding box of point cells, widened by one node, is the
//    shared tile when it holds at most CAP nodes (points are kept sorted by a
//    tiled cell key, so a CTA's points cover a compact patch);
// 2. optionally, points of the same cell inside a warp are summed with a
//    segmented shuffle reduction (match_any finds the segments);
// 3. contributions go to the tile with shared atomics, then one global atomic
//    per non-zero node channel flushes the tile.
// A block whose box does not fit scatters with global atomics directly.
template <class Real, class Acc, int NCH, int BT, int CAP, bool WARPRED>
__device__ __forceinline__ void block_scatter(const KParams<Real> &kp, const Src<Real> &s,
                                              Acc4<Acc> *__restrict__ gacc, uint32_t &err)
{
    constexpr int NW = BT / 32;
    __shared__ Acc tile[NCH][CAP];
    __shared__ int wbox[NW][4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;

    unsigned xmn = s.active ? (unsigned)s.cx : 0xffffffffu, ymn = s.active ? (unsigned)s.cy : 0xffffffffu;
    unsigned xmx = s.active ? (unsigned)s.cx : 0u, ymx = s.active ? (unsigned)s.cy : 0u;
    const unsigned any = __ballot_sync(FULL, s.active);
    xmn = __reduce_min_sync(FULL, xmn); ymn = __reduce_min_sync(FULL, ymn);
    xmx = __reduce_max_sync(FULL, xmx); ymx = __reduce_max_sync(FULL, ymx);
    if (lane == 0) {
        wbox[warp][0] = any ? (int)xmn : INT_MAX; wbox[warp][1] = any ? (int)ymn : INT_MAX;
        wbox[warp][2] = any ? (int)xmx : -1;      wbox[warp][3] = any ? (int)ymx : -1;
    }
    __syncthreads();
    int x0 = INT_MAX, y0 = INT_MAX, x1 = -1, y1 = -1;
#pragma unroll
    for (int w = 0; w < NW; w++) {
        x0 = min(x0, wbox[w][0]); y0 = min(y0, wbox[w][1]);
        x1 = max(x1, wbox[w][2]); y1 = max(y1, wbox[w][3]);
    }
    if (x1 < 0) return;                       // no active point in the block (uniform)
    x0 -= 1; y0 -= 1; x1 += 1; y1 += 1;       // stencil reach
    const int tw = x1 - x0 + 1, th = y1 - y0 + 1;
    const bool use_tile = (long long)tw * th <= CAP;
    const int ntile = use_tile ? tw * th : 0;
    if (use_tile) {
        for (int k = tid; k < ntile; k += BT)
#pragma unroll
            for (int c = 0; c < NCH; c++) tile[c][k] = Acc(0);
        __syncthreads();
    }

    // warp segments of equal cells
    bool leader = s.active;
    int seg_end = lane, maxcnt = 1;
    if (WARPRED) {
        const unsigned key = s.active ? (((unsigned)s.cy << 16) | (unsigned)s.cx) : (0x80000000u | (unsigned)lane);
        const unsigned peers = __match_any_sync(FULL, key);
        const int first = __ffs(peers) - 1;
        const int cnt = __popc(peers);
        const unsigned run = (cnt == 32) ? FULL : (((1u << cnt) - 1u) << first);
        const bool contiguous = __all_sync(FULL, peers == run);
        maxcnt = (int)__reduce_max_sync(FULL, (unsigned)cnt);
        if (contiguous && maxcnt > 1) {
            leader = s.active && (lane == first);
            seg_end = first + cnt - 1;
        } else {
            maxcnt = 1;
        }
    }

    bool nan_m = false, nan_v = false, ovf = false;
#pragma unroll
    for (int a = 0; a < 3; a++) {
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const Real w = s.wx[a] * s.wy[b];
            Real vm = s.active ? w * s.mp : Real(0);
            Real vx = s.active ? w * (s.ax + s.s00 * Real(a - 1) + s.s01 * Real(b - 1)) : Real(0);
            Real vy = s.active ? w * (s.ay + s.s10 * Real(a - 1) + s.s11 * Real(b - 1)) : Real(0);
            Real va = (NCH == 4 && s.active) ? w * s.area : Real(0);
            if (WARPRED && maxcnt > 1) {
                for (int off = 1; off < maxcnt; off <<= 1) {
                    const Real om = __shfl_down_sync(FULL, vm, off);
                    const Real ox = __shfl_down_sync(FULL, vx, off);
                    const Real oy = __shfl_down_sync(FULL, vy, off);
                    Real oa = Real(0);
                    if (NCH == 4) oa = __shfl_down_sync(FULL, va, off);
                    if (lane + off <= seg_end) { vm += om; vx += ox; vy += oy; if (NCH == 4) va += oa; }
                }
            }
            if (leader) {
                nan_m |= isnan(vm);
                nan_v |= isnan(vx) || isnan(vy);
                if (sizeof(Acc) == 8 && !std::is_floating_point<Acc>::value)
                    ovf |= fabs(double(vm)) > kp.lim_m || fabs(double(vx)) > kp.lim_p || fabs(double(vy)) > kp.lim_p;
                const Acc am = AccOps<Acc>::from(vm, kp.scale_m);
                const Acc ax = AccOps<Acc>::from(vx, kp.scale_p);
                const Acc ay = AccOps<Acc>::from(vy, kp.scale_p);
                if (use_tile) {
                    const int li = (s.cx + a - 1 - x0) * th + (s.cy + b - 1 - y0);
                    AccOps<Acc>::add_shared(&tile[0][li], am);
                    AccOps<Acc>::add_shared(&tile[1][li], ax);
                    AccOps<Acc>::add_shared(&tile[2][li], ay);
                    if (NCH == 4) AccOps<Acc>::add_shared(&tile[NCH - 1][li], AccOps<Acc>::from(va, kp.scale_a));
                } else {
                    const size_t node = (size_t)(s.cx + a - 1) * kp.gy + (size_t)(s.cy + b - 1);
                    AccOps<Acc>::add_global(&gacc[node].m, am);
                    AccOps<Acc>::add_global(&gacc[node].px, ax);
                    AccOps<Acc>::add_global(&gacc[node].py, ay);
                    if (NCH == 4) AccOps<Acc>::add_global(&gacc[node].area, AccOps<Acc>::from(va, kp.scale_a));
                }
            }
        }
    }
    if (nan_m) err |= kErrP2gNanMass;
    if (nan_v) err |= kErrP2gNanVel;
    if (ovf) err |= kErrFixedOverflow;
    if (use_tile) {
        __syncthreads();
        for (int k = tid; k < ntile; k += BT) {
            const int lx = k / th, ly = k - lx * th;
            const size_t node = (size_t)(x0 + lx) * kp.gy + (size_t)(y0 + ly);
            const Acc m = tile[0][k], px = tile[1][k], py = tile[2][k];
            if (m != Acc(0)) AccOps<Acc>::add_global(&gacc[node].m, m);
            if (px != Acc(0)) AccOps<Acc>::add_global(&gacc[node].px, px);
            if (py != Acc(0)) AccOps<Acc>::add_global(&gacc[node].py, py);
            if (NCH == 4) {
                const Acc ar = tile[NCH - 1][k];
                if (ar != Acc(0)) AccOps<Acc>::add_global(&gacc[node].area, ar);
            }
        }
    }
}

__device__ __forceinline__ bool cell_in_range(int cx, int cy, int gx, int gy)
{
    return cx >= 1 && cx <= gx - 2 && cy >= 1 && cy <= gy - 2;
}

// ---- standalone P2G (priming) --------------------------------------------
// partition_kernel_p2g (kernels.cuh:39-104) on the current point state.
template <class Real, class Acc, int NCH, int BT, int CAP, bool WARPRED>
__global__ void __launch_bounds__(BT) k_p2g(KParams<Real> kp, Pts<Real> P, Grid<Real, Acc> G,
                                            DevStatus *st, int n)
{
    const int i = blockIdx.x * BT + threadIdx.x;
    Src<Real> s;
    s.active = false; s.cx = s.cy = 0;
    uint32_t err = 0;
    if (i < n) {
        const uint2 key = P.K[i];
        if (!(key.y & kDisabled)) {
            const V4<Real> A = P.A[i], Hv = P.H[i], Cv = P.C[i];
            const V2<Real> v = P.V[i];
            s.cx = (int)(key.x & 0xffff); s.cy = (int)(key.x >> 16);
            if (cell_in_range(s.cx, s.cy, kp.gx, kp.gy)) {
                const M2<Real> H = {Hv.x, Hv.y, Hv.z, Hv.w};
                make_src(kp, s, A.x, A.y, A.z, A.w, H, v.x, v.y, Cv.x, Cv.y, Cv.z, Cv.w);
                s.active = true;
            } else {
                err |= kErrLeftArea;
            }
        }
    }
    if (!s.active) {
#pragma unroll
        for (int k = 0; k < 3; k++) { s.wx[k] = Real(0); s.wy[k] = Real(0); }
        s.mp = s.ax = s.ay = s.s00 = s.s01 = s.s10 = s.s11 = s.area = Real(0);
    }
    block_scatter<Real, Acc, NCH, BT, CAP, WARPRED>(kp, s, G.acc, err);
    warp_flush_status(st, err, 0);
}

// ---- grid update (partition_kernel_update_nodes, kernels.cuh:109-177) ----
template <class Real>
__device__ __forceinline__ void wind_at(const KParams<Real> &kp, double x, double y, double &ux, double &uy)
{
    ux = 0; uy = 0;
    if (kp.wind_kind == ICEMPM_WIND_UNIFORM) { ux = kp.wind_u; uy = kp.wind_v; }
    else if (kp.wind_kind == ICEMPM_WIND_RANKINE) {
        const double dx = x - kp.wind_cx, dy = y - kp.wind_cy;
        const double r = sqrt(dx * dx + dy * dy);
        if (r > 0) {
            const double sp = (r < kp.wind_radius) ? kp.wind_vmax * r / kp.wind_radius
                                                   : kp.wind_vmax * kp.wind_radius / r;
            ux = -dy / r * sp; uy = dx / r * sp;
        }
    }
}

template <class Real, class Acc, bool EXT>
__global__ void __launch_bounds__(256) k_grid_update(KParams<Real> kp, Grid<Real, Acc> G, DevStatus *st,
                                                     long long nnodes)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nnodes) return;
    const Acc4<Acc> r = G.acc[idx];
    V2<Real> out;
    out.x = Real(0); out.y = Real(0);
    if (r.m == Acc(0) && r.px == Acc(0) && r.py == Acc(0) && (!EXT || r.area == Acc(0))) {
        G.vel[idx] = out;
        return;
    }
    Acc4<Acc> z;
    z.m = z.px = z.py = z.area = Acc(0);
    G.acc[idx] = z;
    const Real mass = AccOps<Acc>::template to<Real>(r.m, kp.inv_scale_m);
    uint32_t err = 0;
    if (mass != Real(0)) {
        const Real mx = AccOps<Acc>::template to<Real>(r.px, kp.inv_scale_p);
        const Real my = AccOps<Acc>::template to<Real>(r.py, kp.inv_scale_p);
        Real vx = mx / mass, vy = my / mass;
        if (G.status[idx] != 100) {
            vx = Real(0); vy = Real(0);
            double2 f = G.force[idx];
            f.x += double(mx); f.y += double(my);
            G.force[idx] = f;
        } else if (!EXT) {
            const V2<Real> c = G.cur[idx];
            const double t = (double)(float)(kp.dt_d * (double)st->step);
            const double ramp = (t < 300000) ? 1 + fmin(t / (3600 * 2), 2.) : 3 + fmin((t - 300000) / (3600 * 10), 2.);
            const Real wx = c.x * Real(ramp), wy = c.y * Real(ramp);
            const Real ux = wx - vx, uy = wy - vy;
            const Real um = tsqrt(ux * ux + uy * uy);
            Real k = Real(kp.kL) + Real(kp.kQ) * um;
            k = fmin(k, Real(0.1));
            vx += k * ux; vy += k * uy;
        } else {
            const Real area = AccOps<Acc>::template to<Real>(r.area, kp.inv_scale_a);
            const Real am = area / mass;
            double uxw, uyw;
            wind_at(kp, (double)(idx / kp.gy) * (double)kp.h, (double)(idx % kp.gy) * (double)kp.h, uxw, uyw);
            const Real ux = Real(uxw), uy = Real(uyw);
            const Real ta = Real(kp.rho_a_ca_dt) * tsqrt(ux * ux + uy * uy) * am;
            vx += ta * ux; vy += ta * uy;
            const V2<Real> c = G.cur[idx];
            const Real dx = c.x - vx, dy = c.y - vy;
            const Real k = Real(kp.rho_w_cd_dt) * tsqrt(dx * dx + dy * dy) * am;
            const Real f = k / (Real(1) + k);
            vx += f * dx; vy += f * dy;
        }
        if (vx * vx + vy * vy > kp.vmax2_01) { vx = Real(0); vy = Real(0); }
        if (isnan(vx) || isnan(vy)) err |= kErrGridNan;
        out.x = vx; out.y = vy;
    }
    G.vel[idx] = out;
    if (err) atomicOr(&st->err, err);
}

// ---- fused G2P (step k) + P2G (step k+1) -----------------------------------
// G2P follows partition_kernel_g2p (kernels.cuh:181-315).  C is accumulated
// from (v_i - v_p): identical to the reference's sum over v_i in exact
// arithmetic since sum_i w_ip (x_i - x_p) = 0, and free of the roundoff of a
// large uniform velocity in FP32.
template <class Real, class Acc, int NCH, int BT, int CAP, bool WARPRED>
__global__ void __launch_bounds__(BT) k_g2p_p2g(KParams<Real> kp, Pts<Real> P, Grid<Real, Acc> G,
                                                DevStatus *st, int n)
{
    const int i = blockIdx.x * BT + threadIdx.x;
    const int step = st->step;
    const bool recordPQ = kp.update_every > 0 && (step % kp.update_every) == 0;
    uint32_t err = 0;
    int ndis = 0;
    Src<Real> s;
    s.active = false; s.cx = s.cy = 0;
    if (i < n) {
        const uint2 key = P.K[i];
        uint32_t util = key.y;
        if (!(util & kDisabled)) {
            const V4<Real> A = P.A[i];
            const V4<Real> Hv = P.H[i];
            Real x = A.x, y = A.y, Jp = A.z;
            const Real thick = A.w;
            M2<Real> H = {Hv.x, Hv.y, Hv.z, Hv.w};
            int cx = (int)(key.x & 0xffff), cy = (int)(key.x >> 16);
            Real wx[3], wy[3];
            bspline(x, wx);
            bspline(y, wy);
            Real vx = 0, vy = 0, c00 = 0, c01 = 0, c10 = 0, c11 = 0;
            if (cell_in_range(cx, cy, kp.gx, kp.gy)) {
                V2<Real> nv[3][3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const size_t col = (size_t)(cx + a - 1) * kp.gy + (size_t)(cy - 1);
#pragma unroll
                    for (int b = 0; b < 3; b++) nv[a][b] = G.vel[col + b];
                }
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) {
                        const Real w = wx[a] * wy[b];
                        vx += w * nv[a][b].x;
                        vy += w * nv[a][b].y;
                    }
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) {
                        const Real cf = kp.four_h_inv * (wx[a] * wy[b]);
                        const Real dvx = nv[a][b].x - vx, dvy = nv[a][b].y - vy;
                        const Real dpx = Real(a - 1) - x, dpy = Real(b - 1) - y;
                        c00 += cf * (dvx * dpx); c01 += cf * (dvx * dpy);
                        c10 += cf * (dvy * dpx); c11 += cf * (dvy * dpy);
                    }
            } else {
                err |= kErrLeftArea;
            }
            x += vx * kp.dt_h_inv;
            y += vy * kp.dt_h_inv;
            if (isnan(vx) || isnan(vy)) err |= kErrVelNan;
            if (isnan(x) || isnan(y)) err |= kErrPosNan;
            if (isnan(c00) || isnan(c10) || isnan(c01) || isnan(c11)) err |= kErrBpNan;
            bool moved = false;
            if (x > Real(0.5)) { x -= Real(1); cx++; moved = true; }
            else if (x < Real(-0.5)) { x += Real(1); cx--; moved = true; }
            if (y > Real(0.5)) { y -= Real(1); cy++; moved = true; }
            else if (y < Real(-0.5)) { y += Real(1); cy--; moved = true; }
            if (moved && (cx <= 1 || cx >= kp.gx - 2 || cy <= 1 || cy >= kp.gy - 2)) {
                util |= kDisabled;
                ndis++;
            }
            if (x > Real(0.5) || x < Real(-0.5) || y > Real(0.5) || y < Real(-0.5)) err |= kErrJump;

            // Fe <- (I + dt C) Fe, i.e. H <- H + D + D H with D = dt C
            {
                const Real d00 = kp.dt * c00, d01 = kp.dt * c01, d10 = kp.dt * c10, d11 = kp.dt * c11;
                const M2<Real> h = H;
                H.a00 = h.a00 + d00 + (d00 * h.a00 + d01 * h.a10);
                H.a01 = h.a01 + d01 + (d00 * h.a01 + d01 * h.a11);
                H.a10 = h.a10 + d10 + (d10 * h.a00 + d11 * h.a10);
                H.a11 = h.a11 + d11 + (d10 * h.a01 + d11 * h.a11);
            }
            if (isnan(H.a00) || isnan(H.a10) || isnan(H.a01) || isnan(H.a11)) err |= kErrFeNan;
            const Kin<Real> k = kinematics(H);
            Real p_tr, q_tr;
            pq(k, Real(kp.mat.mu), Real(kp.mat.kappa), p_tr, q_tr);
            if (!(util & kCrushed)) util = failure_check(kp.mat, util, p_tr, q_tr);
            if (util & kCrushed) {
                const SvdH<Real> sv = svd_h(H);
                wolper_dp(kp.mat, thick, p_tr, q_tr, k, sv, H, Jp);
                if (isnan(H.a00) || isnan(H.a10) || isnan(H.a01) || isnan(H.a11)) err |= kErrFeNan;
            }

            V4<Real> Ao; Ao.x = x; Ao.y = y; Ao.z = Jp; Ao.w = thick;
            P.A[i] = Ao;
            V4<Real> Ho; Ho.x = H.a00; Ho.y = H.a01; Ho.z = H.a10; Ho.w = H.a11;
            P.H[i] = Ho;
            V2<Real> Vo; Vo.x = vx; Vo.y = vy;
            P.V[i] = Vo;
            V4<Real> Co; Co.x = c00; Co.y = c01; Co.z = c10; Co.w = c11;
            P.C[i] = Co;
            const uint32_t cell = ((uint32_t)cy << 16) | (uint32_t)cx;   // as kernels.cuh:305
            if (moved || util != key.y) {
                uint2 ko; ko.x = moved ? cell : key.x; ko.y = util;
                P.K[i] = ko;
            }
            if (recordPQ) { V2<Real> pqv; pqv.x = p_tr; pqv.y = q_tr; P.PQ[i] = pqv; }

            if (!(util & kDisabled)) {
                if (cell_in_range(cx, cy, kp.gx, kp.gy)) {
                    s.cx = cx; s.cy = cy;
                    make_src(kp, s, x, y, Jp, thick, H, vx, vy, c00, c01, c10, c11);
                    s.active = true;
                } else {
                    err |= kErrLeftArea;
                }
            }
        }
    }
    if (!s.active) {
#pragma unroll
        for (int k = 0; k < 3; k++) { s.wx[k] = Real(0); s.wy[k] = Real(0); }
        s.mp = s.ax = s.ay = s.s00 = s.s01 = s.s10 = s.s11 = s.area = Real(0);
    }
    block_scatter<Real, Acc, NCH, BT, CAP, WARPRED>(kp, s, G.acc, err);
    warp_flush_status(st, err, ndis);

    // the last CTA to finish advances the device step counter (no waiting)
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&st->done, 1u);
        if (t == gridDim.x - 1) {
            st->step = step + 1;
            st->done = 0;
            __threadfence();
        }
    }
}

// ---- host <-> device conversion ---------------------------------------------
__device__ __forceinline__ uint32_t lo32(double v) { return (uint32_t)(__double_as_longlong(v) & 0xffffffffll); }
__device__ __forceinline__ double from_lo32(uint32_t v) { return __longlong_as_double((long long)v); }

// stage: 19 rows of n doubles (reference HSSOA rows, pitch n)
template <class Real>
__global__ void k_upload(const double *__restrict__ stage, size_t pitch, int n, Pts<Real> P)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double *r = stage + i;
    V4<Real> A; A.x = Real(r[6 * pitch]); A.y = Real(r[7 * pitch]); A.z = Real(r[5 * pitch]); A.w = Real(r[18 * pitch]);
    V4<Real> H;
    H.x = Real(r[10 * pitch] - 1.0); H.y = Real(r[11 * pitch]); H.z = Real(r[12 * pitch]); H.w = Real(r[13 * pitch] - 1.0);
    V2<Real> V; V.x = Real(r[8 * pitch]); V.y = Real(r[9 * pitch]);
    V4<Real> C; C.x = Real(r[14 * pitch]); C.y = Real(r[15 * pitch]); C.z = Real(r[16 * pitch]); C.w = Real(r[17 * pitch]);
    V2<Real> PQ; PQ.x = Real(r[3 * pitch]); PQ.y = Real(r[4 * pitch]);
    uint2 K; K.x = lo32(r[1 * pitch]); K.y = lo32(r[0]);
    P.A[i] = A; P.H[i] = H; P.V[i] = V; P.C[i] = C; P.PQ[i] = PQ; P.K[i] = K;
    P.slot[i] = (uint32_t)i;
    P.pid[i] = lo32(r[2 * pitch]);
    P.thick64[i] = r[18 * pitch];
}

template <class Real>
__global__ void k_download(Pts<Real> P, int n, double *__restrict__ stage, size_t pitch)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t s = P.slot[i];
    double *r = stage + s;
    const V4<Real> A = P.A[i], H = P.H[i], C = P.C[i];
    const V2<Real> V = P.V[i], PQ = P.PQ[i];
    const uint2 K = P.K[i];
    r[0] = from_lo32(K.y); r[1 * pitch] = from_lo32(K.x); r[2 * pitch] = from_lo32(P.pid[i]);
    r[3 * pitch] = double(PQ.x); r[4 * pitch] = double(PQ.y); r[5 * pitch] = double(A.z);
    r[6 * pitch] = double(A.x); r[7 * pitch] = double(A.y);
    r[8 * pitch] = double(V.x); r[9 * pitch] = double(V.y);
    r[10 * pitch] = 1.0 + double(H.x); r[11 * pitch] = double(H.y);
    r[12 * pitch] = double(H.z); r[13 * pitch] = 1.0 + double(H.w);
    r[14 * pitch] = double(C.x); r[15 * pitch] = double(C.y); r[16 * pitch] = double(C.z); r[17 * pitch] = double(C.w);
    r[18 * pitch] = P.thick64[i];
}

// ---- sorting ---------------------------------------------------------------
// Locality key: cells grouped in TX x TY tiles, tiles in column order, cells
// column-major inside a tile; disabled points sort last.
struct TileKey { int tx, ty, ntiles_y; };
static __global__ void k_keys_tiled(const uint2 *__restrict__ K, int n, TileKey t, uint32_t *keys, uint32_t *vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint2 k = K[i];
    uint32_t key = 0xffffffffu;
    if (!(k.y & kDisabled)) {
        const uint32_t cx = k.x & 0xffffu, cy = k.x >> 16;
        const uint32_t tile = (cx / t.tx) * (uint32_t)t.ntiles_y + cy / t.ty;
        key = tile * (uint32_t)(t.tx * t.ty) + (cx % t.tx) * t.ty + cy % t.ty;
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
}

// The reference's HSSOA order key x*GridY + y (ProxyPoint::getCellIndex,
// proxypoint2d.cpp:117-123); disabled points last.
static __global__ void k_keys_reference(const uint2 *__restrict__ K, const uint32_t *__restrict__ slot, int n,
                                 int gy, uint64_t *keys, uint32_t *vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint2 k = K[i];
    uint64_t key = ~0ull;
    if (!(k.y & kDisabled)) {
        const uint64_t cx = k.x & 0xffffu, cy = k.x >> 16;
        key = ((cx * (uint64_t)gy + cy) << 32) | slot[i];   // ties keep the previous host order
    }
    keys[i] = key;
    vals[i] = (uint32_t)i;
}

template <class Real>
__global__ void k_gather(Pts<Real> src, Pts<Real> dst, const uint32_t *__restrict__ perm, int n, int reslot)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t j = perm[i];
    dst.A[i] = src.A[j]; dst.H[i] = src.H[j]; dst.C[i] = src.C[j];
    dst.V[i] = src.V[j]; dst.PQ[i] = src.PQ[j]; dst.K[i] = src.K[j];
    dst.slot[i] = reslot ? (uint32_t)i : src.slot[j];
    dst.pid[i] = src.pid[j];
    dst.thick64[i] = src.thick64[j];
}

// number of leading keys that are not ~0 (keys sorted ascending)
static __global__ void k_count_active(const uint64_t *__restrict__ keys, int n, DevStatus *st)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool act = keys[i] != ~0ull;
    const bool next_inact = (i == n - 1) || keys[i + 1] == ~0ull;
    if (act && next_inact) st->n_active = i + 1;
    if (i == 0 && !act) st->n_active = 0;
}

static __global__ void k_set_step(DevStatus *st, int step, int reset_done)
{
    st->step = step;
    if (reset_done) st->done = 0;
}

}  // namespace icempm
