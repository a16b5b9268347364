// engine.cuh -- device data layout and the step kernels of the B200-native
// 2D APIC MPM step.
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
// Error bits keep the reference's timing: bits raised by a scatter go to a
// pending word that the next grid update folds into the error word, exactly
// when the reference's P2G of that step would have raised them.
//
// Point layout (one entry per point, SoA of 16-byte vectors, 128-bit loads):
//   A   {x, y, Jp_inv, thickness}  x, y cell-local in [-0.5, 0.5]
//   H   {H00, H01, H10, H11}       H = Fe - I
//   K   {cell, utility}            cell = (y << 16) | x, utility flags
//   V   {vx, vy}                   read only when priming
//   C   {C00, C01, C10, C11}       APIC affine matrix (the reference's Bp)
// The fused kernel hands V and C from its G2P to its P2G in registers, so
// between the sub-steps of one icempm_step call they are dead: they are
// stored by the call's last sub-step (DevStatus::vc_step) and by the sub-step
// that disables a point (its last), which leaves the state after the call
// identical to storing them every sub-step.
//   PQ  {P, Q}                     written on record steps only
//   slot, pid, thick64             host slot, point id row, f64 thickness
// Grid layout (node = y + x*GridY, the reference order):
//   acc.m, acc.px, acc.py          accumulators, one array each (int64 fixed point, f32 or f64)
//   vel {vx, vy}                   grid velocity after the update
//   status (u8), cur {vx, vy}, force {fx, fy} (f64, boundary reaction)
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <climits>
#include <type_traits>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "device_math.cuh"
#include "icempm.h"
#include "mlp_device.cuh"

// Shape of the FP32-state fused kernel: threads per CTA, points per thread,
// nodes of the shared scatter tile (0: no tile, each warp's merged node sums
// go straight to the global accumulators), CTAs per SM it is compiled for
// (this caps registers at 96: occupancy is what hides its latencies).
#ifndef ICEMPM_FUSED_BT
#define ICEMPM_FUSED_BT 128
#endif
#ifndef ICEMPM_FUSED_PPT
#define ICEMPM_FUSED_PPT 4
#endif
#ifndef ICEMPM_FUSED_CAP
#define ICEMPM_FUSED_CAP 0
#endif
#ifndef ICEMPM_FUSED_MINB
#define ICEMPM_FUSED_MINB 5
#endif
// Stages of point state in shared memory (2: the next chunk is fetched while
// this one is computed; 1: it is fetched at the end of this one).
#ifndef ICEMPM_FUSED_STAGES
#define ICEMPM_FUSED_STAGES 2
#endif
// Nodes per thread of the grid update (1, 2 or 4; vector loads and stores).
#ifndef ICEMPM_UPDATE_NPT
#define ICEMPM_UPDATE_NPT 2
#endif
// 1: the fused kernel keeps the 3x3 node velocities of the last cell in
// registers for the thread's next point; 0: it loads them for every point.
#ifndef ICEMPM_VEL_CACHE
#define ICEMPM_VEL_CACHE 0
#endif
// 1: persistent grid of as many CTAs as fit; 0: one CTA per chunk.
#ifndef ICEMPM_FUSED_PERSIST
#define ICEMPM_FUSED_PERSIST 1
#endif

namespace icempm {

template <class T> struct alignas(16) V4 { T x, y, z, w; };
template <class T> struct alignas(2 * sizeof(T) > 16 ? 16 : 2 * sizeof(T)) V2 { T x, y; };
// Grid accumulators, one array per channel (node-major), so that a warp's
// atomics and the grid update's loads touch contiguous words.
template <class A> struct AccGrid { A *m, *px, *py; };

// Point arrays are read once and written once per step: load and store them
// with the streaming cache policy so they do not evict the grid velocities
// the 3x3 gathers reuse from L1.
__device__ __forceinline__ V4<float> ld_stream(const V4<float> *p)
{
    const float4 v = __ldcs(reinterpret_cast<const float4 *>(p));
    V4<float> r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = v.w;
    return r;
}
__device__ __forceinline__ V4<double> ld_stream(const V4<double> *p)
{
    const double2 a = __ldcs(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2 *>(p) + 1);
    V4<double> r; r.x = a.x; r.y = a.y; r.z = b.x; r.w = b.y;
    return r;
}
__device__ __forceinline__ uint2 ld_stream(const uint2 *p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(V4<float> *p, const V4<float> &v)
{
    __stcs(reinterpret_cast<float4 *>(p), make_float4(v.x, v.y, v.z, v.w));
}
__device__ __forceinline__ void st_stream(V4<double> *p, const V4<double> &v)
{
    __stcs(reinterpret_cast<double2 *>(p), make_double2(v.x, v.y));
    __stcs(reinterpret_cast<double2 *>(p) + 1, make_double2(v.z, v.w));
}
__device__ __forceinline__ void st_stream(V2<float> *p, const V2<float> &v)
{
    __stcs(reinterpret_cast<float2 *>(p), make_float2(v.x, v.y));
}
__device__ __forceinline__ void st_stream(V2<double> *p, const V2<double> &v)
{
    __stcs(reinterpret_cast<double2 *>(p), make_double2(v.x, v.y));
}
__device__ __forceinline__ void st_stream(uint2 *p, const uint2 &v) { __stcs(p, v); }

struct DevStatus {
    uint32_t err;          // the reference's gpu_error_indicator
    int32_t disabled;      // the reference's gpu_disabled_points_count
    int32_t step;          // index of the sub-step the next grid update runs
    uint32_t done;         // CTA completion ticket of the fused kernel
    int32_t n_active;      // result slot of the compaction boundary search
    uint32_t err_pending;  // bits of the scatter for the next sub-step
    int32_t vc_step;       // G2P sub-step whose point velocity and C are stored
    uint32_t chunk_ticket; // chunks of the fused kernel handed out beyond each CTA's first
};

template <class Real> struct Pts {
    V4<Real> *A, *H, *C;
    V2<Real> *V, *PQ;
    uint2 *K;
    uint32_t *slot, *pid;
    double *thick64;
};

template <class Real, class Acc> struct Grid {
    AccGrid<Acc> acc;
    V2<Real> *vel;
    V2<Real> *cur;
    const V4<Real> *frc;   // extended forcing per node: {current vx, vy, wind stress x, y}
    const uint8_t *status;
    double2 *force;
};

// The yield-surface and hardening constants of SimParams
// (GetParametersForGrain, kernels.cuh:538-566; tan is taken once here).
inline Material material_of(const icempm_simparams_t &p)
{
    Material m;
    m.mu = p.mu; m.kappa = p.kappa; m.DP_threshold_p = p.DP_threshold_p;
    m.pmax = p.IceCompressiveStrength; m.pmin = -p.IceTensileStrength;
    m.qmax = p.IceShearStrength; m.pmin2 = -p.IceTensileStrength2;
    m.beta = p.IceTensileStrength / p.IceCompressiveStrength;
    m.M_sq = (4. * m.qmax * m.qmax * (1. + 2. * m.beta)) / ((m.pmax - m.pmin) * (m.pmax - m.pmin));
    m.tan_phi = std::tan(p.DP_phi * ICEMPM_PI / 180);
    m.ridge_coeff_g_rho = p.RidgeFormationCoeff * ICEMPM_GRAVITY * p.IceDensity;
    return m;
}

// Trial/projected pairs of the return map recorded from a run (training data
// of the learned return map).  Record r is rec[2r] = {sigma1, sigma2, Jp_inv,
// thickness} of the trial state and rec[2r+1] = {sigma1', sigma2', Jp_inv', 3}
// after the projection; only projections onto the yield surface (case 3 of
// the return map) are recorded.
struct HarvestBuf {
    uint32_t count, cap;
    float4 *rec;
};

// Values the kernels read, prepared on the host from SimParams and the options.
template <class Real> struct KParams {
    int gx, gy, update_every;
    int ext, wind_kind;
    Real h, h_inv, dt, dt_h_inv, four_h_inv, vmax2_01, particle_mass, dt_vol_Dpinv;
    double dt_d;                    // InitialTimeStep (double) for the simulation time
    double kL, kQ;                  // effective drag coefficients * dt (compat)
    double scale_m, scale_p;        // fixed point: value * scale -> int64
    double inv_scale_m, inv_scale_p;
    float lim_m, lim_p;             // largest |value| a single term may carry in fixed point
    Real ext_impulse;               // dt * ParticleVolume (extended forcing)
    Real rho_w_cd;                  // rho_w * Cd (extended forcing)
    MatT<Real> mat;
    HarvestBuf *harvest;            // return-map pairs are recorded when not null
    int harvest_stride;             // ... for points with (index + step) % stride == 0
    uint32_t tx_extra;              // bytes each chunk's barrier expects beyond its copies (0; tests of the timeout)
    unsigned long long wait_ns;     // time limit of a barrier wait
    const mlp::Packed *mlp;         // learned return map (the LEARNED instance): packed network
    float mlp_tol;                  // ... accepted when its answer lies on the yield surface within this
    unsigned long long *mlp_counts; // ... [0] answers kept, [1] exact fallbacks
    // Broadcast pairs of the factors the packed arithmetic of the fused
    // kernel uses (one 8-byte constant load each, no register shuffling):
    // dt/h, -4/h, -h, 1, 1/2, the extended forcing's impulse factor, and the
    // fixed-point scales (1 for float accumulators): momentum scale, h times
    // it, mass scale (scalar).
    P2<Real> dt_h_inv2, neg_four_h_inv2, neg_h2, one2, half2, ext_impulse2, sp2, hsp2;
    Real sm_r;
};

// Fire-and-forget reductions into global memory (red.global: no value comes
// back, so the issuing thread does not wait for the L2).
// The int64 node sums are reduced with an L2 evict-last policy: the grid
// update reads every accumulator line right after the scatter, and more of
// them are then still in L2 (grid update -3.6 %).
__device__ __forceinline__ void red_global_add(long long *a, long long v)
{
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("red.relaxed.gpu.global.add.L2::cache_hint.u64 [%0], %1, %2;" ::"l"(a), "l"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void red_global_add(float *a, float v)
{
    asm volatile("red.relaxed.gpu.global.add.f32 [%0], %1;" ::"l"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void red_global_add(double *a, double v)
{
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(a), "d"(v) : "memory");
}

// ---- accumulator conversions -------------------------------------------
// Scatter values arrive already multiplied by the scale (sources are scaled
// once per point); `cvt` rounds them to the accumulator type.
template <class Acc> struct AccOps;
template <> struct AccOps<long long> {
    static constexpr bool fixed = true;
    static __device__ __forceinline__ long long cvt(float v) { return __float2ll_rn(v); }
    static __device__ __forceinline__ long long cvt(double v) { return __double2ll_rn(v); }
    template <class Real>
    static __device__ __forceinline__ Real to(long long v, double inv_scale) { return Real(double(v) * inv_scale); }
    // A 64-bit shared-memory atomic add is a compare-and-swap loop on sm_100a;
    // two native 32-bit adds give the same sum modulo 2^64: the low words add
    // with a returned old value, and each addition that wraps the low word
    // carries one into the high word.  The total carry is the same in every
    // order, so the tile sum stays exact and order-independent.
    static __device__ __forceinline__ void add_shared(long long *a, long long v) {
        unsigned *w = reinterpret_cast<unsigned *>(a);       // w[0] low word, w[1] high word
        const unsigned lo = (unsigned)(unsigned long long)v;
        const unsigned hi = (unsigned)((unsigned long long)v >> 32);
        const unsigned old = atomicAdd(w, lo);
        atomicAdd(w + 1, hi + ((old + lo < old) ? 1u : 0u));
    }
    static __device__ __forceinline__ void add_global(long long *a, long long v) { red_global_add(a, v); }
};
template <> struct AccOps<float> {
    static constexpr bool fixed = false;
    template <class R> static __device__ __forceinline__ float cvt(R v) { return float(v); }
    template <class Real> static __device__ __forceinline__ Real to(float v, double) { return Real(v); }
    static __device__ __forceinline__ void add_shared(float *a, float v) { atomicAdd(a, v); }
    static __device__ __forceinline__ void add_global(float *a, float v) { red_global_add(a, v); }
};
template <> struct AccOps<double> {
    static constexpr bool fixed = false;
    template <class R> static __device__ __forceinline__ double cvt(R v) { return double(v); }
    template <class Real> static __device__ __forceinline__ Real to(double v, double) { return Real(v); }
    static __device__ __forceinline__ void add_shared(double *a, double v) { atomicAdd(a, v); }
    static __device__ __forceinline__ void add_global(double *a, double v) { red_global_add(a, v); }
};

__device__ __forceinline__ void warp_flush_status(DevStatus *st, uint32_t err, uint32_t perr, int ndis)
{
    const uint32_t e = __reduce_or_sync(0xffffffffu, err);
    const uint32_t pe = __reduce_or_sync(0xffffffffu, perr);
    const int d = (int)__reduce_add_sync(0xffffffffu, (unsigned)ndis);
    if ((threadIdx.x & 31) == 0) {
        if (e) atomicOr(&st->err, e);
        if (pe) atomicOr(&st->err_pending, pe);
        if (d) atomicAdd(&st->disabled, d);
    }
}

__device__ __forceinline__ bool cell_in_range(int cx, int cy, int gx, int gy)
{
    // 1 <= cx <= gx - 2 and 1 <= cy <= gy - 2, as two unsigned compares (grids are >= 5 nodes a side)
    return (uint32_t)(cx - 1) <= (uint32_t)(gx - 3) && (uint32_t)(cy - 1) <= (uint32_t)(gy - 3);
}

// ---- P2G sources of one point --------------------------------------------
// The reference scatters, for node offsets (i, j) in {-1,0,1}^2 (kernels.cuh:76-95)
//   dM = w m_p,   dP = w (m_p v + S (i - x, j - y) h),
//   S = m_p C - dt_vol_Dpinv Jp_inv thickness tau.
// With A = m_p v - h S (x, y):  dP = w (A + h S (i, j)).  The extended
// forcing adds the impulse dt * area * (wind + water stress) to A, with the
// wind stress and the current of the point's cell node.  For fixed-point
// accumulation the sources carry the accumulator scale already.
template <class Real> struct Src {
    int cx, cy;
    Real wx[3], wy[3];
    Real mp, ax, ay, s00, s01, s10, s11;
};

template <class Real, class Acc>
__device__ __forceinline__ void make_src(const KParams<Real> &kp, const V4<Real> &f, Src<Real> &s,
                                         Real x, Real y, Real Jp, Real thick, const Kin<Real> &k, Real vx,
                                         Real vy, Real c00, Real c01, Real c10, Real c11, uint32_t &perr)
{
    const M2<Real> tau = kirchhoff(k, kp.mat.mu, kp.mat.kappa);
    const Real mp = kp.particle_mass * thick;
    const Real sc = kp.dt_vol_Dpinv * Jp * thick;
    const Real S00 = mp * c00 - sc * tau.a00, S01 = mp * c01 - sc * tau.a01;
    const Real S10 = mp * c10 - sc * tau.a10, S11 = mp * c11 - sc * tau.a11;
    Real ax = mp * vx - kp.h * (S00 * x + S01 * y);
    Real ay = mp * vy - kp.h * (S10 * x + S11 * y);
    if (kp.ext) {   // f = forcing entry of the point's cell node
        const Real dx = f.x - vx, dy = f.y - vy;
        const Real cw = kp.rho_w_cd * tsqrt(dx * dx + dy * dy);
        ax += kp.ext_impulse * (f.z + cw * dx);
        ay += kp.ext_impulse * (f.w + cw * dy);
    }
    const Real fm = AccOps<Acc>::fixed ? Real(kp.scale_m) : Real(1);
    const Real fp = AccOps<Acc>::fixed ? Real(kp.scale_p) : Real(1);
    if (AccOps<Acc>::fixed) {
        // a node term is at most max(w) <= 0.5625 times these bounds
        if (!(fabs(ax) + kp.h * (fabs(S00) + fabs(S01)) <= Real(kp.lim_p)) ||
            !(fabs(ay) + kp.h * (fabs(S10) + fabs(S11)) <= Real(kp.lim_p)) || !(mp <= Real(kp.lim_m)))
            perr |= kErrFixedOverflow;
    }
    s.mp = mp * fm;
    s.ax = ax * fp; s.ay = ay * fp;
    const Real hp = kp.h * fp;
    s.s00 = hp * S00; s.s01 = hp * S01; s.s10 = hp * S10; s.s11 = hp * S11;
    bspline(x, s.wx);
    bspline(y, s.wy);
}

// Node (a, b) terms of a source: mass, x- and y-momentum.
template <class Real>
__device__ __forceinline__ void src_terms(const Src<Real> &s, int a, int b, Real &m, Real &px, Real &py)
{
    const Real w = s.wx[a] * s.wy[b];
    m = s.mp * w;
    px = w * (s.ax + s.s00 * Real(a - 1) + s.s01 * Real(b - 1));
    py = w * (s.ay + s.s10 * Real(a - 1) + s.s11 * Real(b - 1));
}

// ---- shared scatter tile -----------------------------------------------------
// The tile covers nodes [x0, x0+tw) x [y0, y0+th) of the grid; entry
// (X - x0) * th + (Y - y0), three channels.
template <class Acc, int CAP> struct Tile {
    Acc (*t)[CAP > 0 ? CAP : 1];
    int x0, y0, tw, th;
    unsigned th_rcp;   // ceil(2^32 / th): entry k lies in column umulhi(k, th_rcp) (exact while k * th < 2^32)
    bool on;
};

__device__ __forceinline__ unsigned rcp32(int d) { return d > 0 ? 0xffffffffu / (unsigned)d + 1u : 0u; }

template <class Real, class Acc, int CAP>
__device__ __forceinline__ void node_add(const Tile<Acc, CAP> &T, bool in_tile, const AccGrid<Acc> &gacc,
                                         int gy, int X, int Y, Real m, Real px, Real py)
{
    const Acc am = AccOps<Acc>::cvt(m), ax = AccOps<Acc>::cvt(px), ay = AccOps<Acc>::cvt(py);
    if (in_tile) {
        const int li = (X - T.x0) * T.th + (Y - T.y0);
        AccOps<Acc>::add_shared(&T.t[0][li], am);
        AccOps<Acc>::add_shared(&T.t[1][li], ax);
        AccOps<Acc>::add_shared(&T.t[2][li], ay);
    } else {
        const uint32_t node = (uint32_t)X * (uint32_t)gy + (uint32_t)Y;
        AccOps<Acc>::add_global(gacc.m + node, am);
        AccOps<Acc>::add_global(gacc.px + node, ax);
        AccOps<Acc>::add_global(gacc.py + node, ay);
    }
}

// Zero the tile entries [0, tw*th) (all threads of the CTA).
template <class Acc, int CAP, int BT>
__device__ __forceinline__ void tile_zero(const Tile<Acc, CAP> &T)
{
    const int nt = T.tw * T.th;
    for (int k = threadIdx.x; k < nt; k += BT) {
        T.t[0][k] = Acc(0); T.t[1][k] = Acc(0); T.t[2][k] = Acc(0);
    }
}

// One global atomic per non-zero tile entry and channel (all threads of the CTA).
template <class Acc, int CAP, int BT>
__device__ __forceinline__ void tile_flush(const Tile<Acc, CAP> &T, const AccGrid<Acc> &gacc, int gx, int gy)
{
    const int nt = T.tw * T.th;
    for (int k = threadIdx.x; k < nt; k += BT) {
        const int lx = (int)__umulhi((unsigned)k, T.th_rcp), ly = k - lx * T.th;
        const int X = T.x0 + lx, Y = T.y0 + ly;
        const Acc m = T.t[0][k], px = T.t[1][k], py = T.t[2][k];
        if ((m != Acc(0) || px != Acc(0) || py != Acc(0)) && X >= 0 && X < gx && Y >= 0 && Y < gy) {
            const uint32_t node = (uint32_t)X * (uint32_t)gy + (uint32_t)Y;
            if (m != Acc(0)) AccOps<Acc>::add_global(gacc.m + node, m);
            if (px != Acc(0)) AccOps<Acc>::add_global(gacc.px + node, px);
            if (py != Acc(0)) AccOps<Acc>::add_global(gacc.py + node, py);
        }
    }
}

// CTA bounding box of cells widened by `reach` nodes -> tile; `box` holds
// {INT_MAX, INT_MAX, -1, -1} visible to all threads before the call.
template <class Acc, int CAP>
__device__ __forceinline__ Tile<Acc, CAP> make_tile(Acc (*t)[CAP], int *box, bool any_lane, unsigned xmn,
                                                    unsigned ymn, unsigned xmx, unsigned ymx, int reach)
{
    const unsigned FULL = 0xffffffffu;
    xmn = __reduce_min_sync(FULL, xmn); ymn = __reduce_min_sync(FULL, ymn);
    xmx = __reduce_max_sync(FULL, xmx); ymx = __reduce_max_sync(FULL, ymx);
    const bool warp_any = __any_sync(FULL, any_lane);
    if ((threadIdx.x & 31) == 0 && warp_any) {
        atomicMin(&box[0], (int)xmn); atomicMin(&box[1], (int)ymn);
        atomicMax(&box[2], (int)xmx); atomicMax(&box[3], (int)ymx);
    }
    __syncthreads();
    Tile<Acc, CAP> T;
    T.t = t;
    T.x0 = box[0] - reach; T.y0 = box[1] - reach;
    T.tw = box[2] - box[0] + 2 * reach + 1; T.th = box[3] - box[1] + 2 * reach + 1;
    // 64-bit product: a box spanning the whole grid must not wrap into range
    T.on = box[2] >= 0 && (long long)T.tw * (long long)T.th <= (long long)CAP;
    if (!T.on) { T.tw = 0; T.th = 0; }
    T.th_rcp = rcp32(T.th);
    return T;
}

template <class Acc, int CAP>
__device__ __forceinline__ bool cell_in_tile(const Tile<Acc, CAP> &T, int cx, int cy)
{
    return T.on && cx - 1 >= T.x0 && cx + 1 < T.x0 + T.tw && cy - 1 >= T.y0 && cy + 1 < T.y0 + T.th;
}

__device__ __forceinline__ void init_box(int *box)
{
    if (threadIdx.x == 0) { box[0] = INT_MAX; box[1] = INT_MAX; box[2] = -1; box[3] = -1; }
}

// ---- standalone P2G (priming) --------------------------------------------
// partition_kernel_p2g (kernels.cuh:39-104) on the current point state, one
// point per thread, contributions straight into the tile.
template <class Real, class Acc, int BT, int CAP>
__global__ void __launch_bounds__(BT) k_p2g(KParams<Real> kp, Pts<Real> P, Grid<Real, Acc> G,
                                            DevStatus *st, int n)
{
    __shared__ Acc tile[3][CAP];
    __shared__ int box[4];
    init_box(box);
    const int i = blockIdx.x * BT + threadIdx.x;
    Src<Real> s;
    s.cx = s.cy = 0;
    bool active = false;
    uint32_t perr = 0;
    if (i < n) {
        const uint2 key = P.K[i];
        if (!(key.y & kDisabled)) {
            s.cx = (int)(key.x & 0xffff); s.cy = (int)(key.x >> 16);
            if (cell_in_range(s.cx, s.cy, kp.gx, kp.gy)) {
                const V4<Real> A = P.A[i], Hv = P.H[i], Cv = P.C[i];
                const V2<Real> v = P.V[i];
                const M2<Real> H = {Hv.x, Hv.y, Hv.z, Hv.w};
                V4<Real> f{};
                if (kp.ext) f = G.frc[(uint32_t)s.cx * (uint32_t)kp.gy + (uint32_t)s.cy];
                make_src<Real, Acc>(kp, f, s, A.x, A.y, A.z, A.w, kinematics(H), v.x, v.y,
                                    Cv.x, Cv.y, Cv.z, Cv.w, perr);
                active = true;
            } else {
                perr |= kErrLeftArea;
            }
        }
    }
    __syncthreads();
    const Tile<Acc, CAP> T = make_tile<Acc, CAP>(tile, box, active, active ? s.cx : 0x7fffffffu,
                                                 active ? s.cy : 0x7fffffffu, active ? s.cx : 0u,
                                                 active ? s.cy : 0u, 1);
    tile_zero<Acc, CAP, BT>(T);
    __syncthreads();
    if (active) {
        const bool in_tile = cell_in_tile(T, s.cx, s.cy);
        bool nan_m = false, nan_v = false;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) {
                Real m, px, py;
                src_terms(s, a, b, m, px, py);
                nan_m |= isnan(m);
                nan_v |= isnan(px) || isnan(py);
                node_add<Real, Acc, CAP>(T, in_tile, G.acc, kp.gy, s.cx + a - 1, s.cy + b - 1, m, px, py);
            }
        if (nan_m) perr |= kErrP2gNanMass;
        if (nan_v) perr |= kErrP2gNanVel;
    }
    __syncthreads();
    tile_flush<Acc, CAP, BT>(T, G.acc, kp.gx, kp.gy);
    warp_flush_status(st, 0u, perr, 0);
}

// ---- the textbook step: the plain from-scratch FP32 baseline ---------------
// The MPM sub-step as three plain kernels, one point or node per thread,
// written the way the method is usually first put on a GPU: P2G straight into
// the global accumulators with one FP32 atomic per node and channel (27 per
// point), the grid update, and G2P with the 3x3 gather summed node by node;
// the whole point state (V and C included) is read and written every
// sub-step.  Same arithmetic helpers as the fused kernel (H = Fe - I, FP32),
// no fusion, no locality tiles, no warp-level merging, no fixed point.  It is
// the yardstick the fused kernel is measured against, not the product.
// P2G of the next sub-step (errors pending until its grid update, as in the
// fused kernel); `advance`: the sub-step counter moves on (not when priming).
template <class Real>
__global__ void __launch_bounds__(256) k_textbook_p2g(KParams<Real> kp, Pts<Real> P, Grid<Real, float> G,
                                                      DevStatus *st, int n, int advance)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (advance && i == 0) st->step += 1;   // G2P of this sub-step has finished reading it
    uint32_t perr = 0;
    if (i < n) {
        const uint2 key = P.K[i];
        if (!(key.y & kDisabled)) {
            Src<Real> s;
            s.cx = (int)(key.x & 0xffff); s.cy = (int)(key.x >> 16);
            if (cell_in_range(s.cx, s.cy, kp.gx, kp.gy)) {
                const V4<Real> A = P.A[i], Hv = P.H[i], Cv = P.C[i];
                const V2<Real> v = P.V[i];
                const M2<Real> H = {Hv.x, Hv.y, Hv.z, Hv.w};
                V4<Real> f{};
                if (kp.ext) f = G.frc[(uint32_t)s.cx * (uint32_t)kp.gy + (uint32_t)s.cy];
                make_src<Real, float>(kp, f, s, A.x, A.y, A.z, A.w, kinematics(H), v.x, v.y, Cv.x, Cv.y, Cv.z, Cv.w,
                                      perr);
                bool nan_m = false, nan_v = false;
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        Real m, px, py;
                        src_terms(s, a, b, m, px, py);
                        nan_m |= isnan(m);
                        nan_v |= isnan(px) || isnan(py);
                        const uint32_t node = (uint32_t)(s.cx + a - 1) * (uint32_t)kp.gy + (uint32_t)(s.cy + b - 1);
                        atomicAdd(G.acc.m + node, float(m));
                        atomicAdd(G.acc.px + node, float(px));
                        atomicAdd(G.acc.py + node, float(py));
                    }
                if (nan_m) perr |= kErrP2gNanMass;
                if (nan_v) perr |= kErrP2gNanVel;
            } else {
                perr |= kErrLeftArea;
            }
        }
    }
    warp_flush_status(st, 0u, perr, 0);
}

template <class Real>
__global__ void __launch_bounds__(256) k_textbook_g2p(KParams<Real> kp, Pts<Real> P, Grid<Real, float> G,
                                                      DevStatus *st, int n)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    uint32_t err = 0;
    int ndis = 0;
    const int step = st->step;
    if (i < n) {
        const uint2 key = P.K[i];
        uint32_t util = key.y;
        if (!(util & kDisabled)) {
            const V4<Real> A = P.A[i], Hv = P.H[i];
            Real x = A.x, y = A.y, Jp = A.z;
            const Real thick = A.w;
            M2<Real> H = {Hv.x, Hv.y, Hv.z, Hv.w};
            int cx = (int)(key.x & 0xffff), cy = (int)(key.x >> 16);
            Real vx = 0, vy = 0, c00 = 0, c01 = 0, c10 = 0, c11 = 0;
            if (cell_in_range(cx, cy, kp.gx, kp.gy)) {
                Real wx[3], wy[3];
                bspline(x, wx);
                bspline(y, wy);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        const V2<Real> nv = G.vel[(uint32_t)(cx + a - 1) * (uint32_t)kp.gy + (uint32_t)(cy + b - 1)];
                        const Real w = wx[a] * wy[b];
                        const Real dx = Real(a - 1) - x, dy = Real(b - 1) - y;
                        vx += w * nv.x; vy += w * nv.y;
                        c00 += w * nv.x * dx; c01 += w * nv.x * dy;
                        c10 += w * nv.y * dx; c11 += w * nv.y * dy;
                    }
                c00 *= kp.four_h_inv; c01 *= kp.four_h_inv; c10 *= kp.four_h_inv; c11 *= kp.four_h_inv;
            }
            x += vx * kp.dt_h_inv;
            y += vy * kp.dt_h_inv;
            if (isnan(vx + vy)) err |= kErrVelNan;
            if (isnan(x + y)) err |= kErrPosNan;
            if (isnan((c00 + c10) + (c01 + c11))) err |= kErrBpNan;
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
            const Real d00 = kp.dt * c00, d01 = kp.dt * c01, d10 = kp.dt * c10, d11 = kp.dt * c11;
            const M2<Real> h = H;
            H.a00 = h.a00 + d00 + (d00 * h.a00 + d01 * h.a10);
            H.a01 = h.a01 + d01 + (d00 * h.a01 + d01 * h.a11);
            H.a10 = h.a10 + d10 + (d10 * h.a00 + d11 * h.a10);
            H.a11 = h.a11 + d11 + (d10 * h.a01 + d11 * h.a11);
            if (isnan((H.a00 + H.a10) + (H.a01 + H.a11))) err |= kErrFeNan;
            Kin<Real> k = kinematics(H);
            Real p_tr, q_tr;
            pq(k, kp.mat.mu, kp.mat.kappa, p_tr, q_tr);
            if (!(util & kCrushed)) util = failure_check(kp.mat, util, p_tr, q_tr);
            if (util & kCrushed) {
                wolper_dp(kp.mat, thick, p_tr, q_tr, k, svd_h(H), H, Jp);
                if (isnan((H.a00 + H.a10) + (H.a01 + H.a11))) err |= kErrFeNan;
            }
            V4<Real> Ao; Ao.x = x; Ao.y = y; Ao.z = Jp; Ao.w = thick;
            P.A[i] = Ao;
            V4<Real> Ho; Ho.x = H.a00; Ho.y = H.a01; Ho.z = H.a10; Ho.w = H.a11;
            P.H[i] = Ho;
            V2<Real> Vo; Vo.x = vx; Vo.y = vy;
            P.V[i] = Vo;
            V4<Real> Co; Co.x = c00; Co.y = c01; Co.z = c10; Co.w = c11;
            P.C[i] = Co;
            uint2 ko; ko.x = ((uint32_t)cy << 16) | (uint32_t)cx; ko.y = util;
            P.K[i] = ko;
            if (kp.update_every > 0 && (step % kp.update_every) == 0) {
                V2<Real> pqv; pqv.x = p_tr; pqv.y = q_tr;
                P.PQ[i] = pqv;
            }
        }
    }
    warp_flush_status(st, err, 0u, ndis);
}

// ---- grid update (partition_kernel_update_nodes, kernels.cuh:109-177) ----
// Compat forcing follows the reference; the extended forcing's stresses are
// point impulses (make_src), so its node update is v = p/m with walls and clamp.
// One node of the update; `step` is the sub-step index (the compat current ramp).
template <class Real, class Acc, bool EXT>
__device__ __forceinline__ void grid_update_node(const KParams<Real> &kp, const Grid<Real, Acc> &G, DevStatus *st,
                                                 long long idx, int step)
{
    struct { Acc m, px, py; } r = {G.acc.m[idx], G.acc.px[idx], G.acc.py[idx]};
    V2<Real> out;
    out.x = Real(0); out.y = Real(0);
    if (r.m == Acc(0) && r.px == Acc(0) && r.py == Acc(0)) {
        G.vel[idx] = out;
        return;
    }
    G.acc.m[idx] = Acc(0); G.acc.px[idx] = Acc(0); G.acc.py[idx] = Acc(0);
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
            const double t = (double)(float)(kp.dt_d * (double)step);
            const double ramp = (t < 300000) ? 1 + fmin(t / (3600 * 2), 2.) : 3 + fmin((t - 300000) / (3600 * 10), 2.);
            const Real wx = c.x * Real(ramp), wy = c.y * Real(ramp);
            const Real ux = wx - vx, uy = wy - vy;
            const Real um = tsqrt(ux * ux + uy * uy);
            Real k = Real(kp.kL) + Real(kp.kQ) * um;
            k = fmin(k, Real(0.1));
            vx += k * ux; vy += k * uy;
        }
        if (vx * vx + vy * vy > kp.vmax2_01) { vx = Real(0); vy = Real(0); }
        if (isnan(vx) || isnan(vy)) err |= kErrGridNan;
        out.x = vx; out.y = vy;
    }
    G.vel[idx] = out;
    if (err) atomicOr(&st->err, err);
}

// this step's scatter errors become visible now, as in the reference
__device__ __forceinline__ void fold_pending(DevStatus *st)
{
    const uint32_t pe = st->err_pending;
    if (pe) { atomicOr(&st->err, pe); st->err_pending = 0; }
}

// Velocity of a node whose accumulators (am, apx, apy) are not all zero, from
// its status byte (grid_update_node after its loads); adds the wall reaction
// into the force accumulator and error bits into err.
template <class Real, class Acc, bool EXT>
__device__ __forceinline__ V2<Real> node_velocity(const KParams<Real> &kp, const Grid<Real, Acc> &G, long long idx,
                                                  int step, Acc am, Acc apx, Acc apy, uint8_t status, uint32_t &err)
{
    V2<Real> out;
    out.x = Real(0); out.y = Real(0);
    const Real mass = AccOps<Acc>::template to<Real>(am, kp.inv_scale_m);
    if (mass != Real(0)) {
        const Real mx = AccOps<Acc>::template to<Real>(apx, kp.inv_scale_p);
        const Real my = AccOps<Acc>::template to<Real>(apy, kp.inv_scale_p);
        Real vx = mx / mass, vy = my / mass;
        if (status != 100) {
            vx = Real(0); vy = Real(0);
            double2 f = G.force[idx];
            f.x += double(mx); f.y += double(my);
            G.force[idx] = f;
        } else if (!EXT) {
            const V2<Real> c = G.cur[idx];
            const double t = (double)(float)(kp.dt_d * (double)step);
            const double ramp = (t < 300000) ? 1 + fmin(t / (3600 * 2), 2.) : 3 + fmin((t - 300000) / (3600 * 10), 2.);
            const Real wx = c.x * Real(ramp), wy = c.y * Real(ramp);
            const Real ux = wx - vx, uy = wy - vy;
            const Real um = tsqrt(ux * ux + uy * uy);
            Real k = Real(kp.kL) + Real(kp.kQ) * um;
            k = fmin(k, Real(0.1));
            vx += k * ux; vy += k * uy;
        }
        if (vx * vx + vy * vy > kp.vmax2_01) { vx = Real(0); vy = Real(0); }
        if (isnan(vx) || isnan(vy)) err |= kErrGridNan;
        out.x = vx; out.y = vy;
    }
    return out;
}

// NPT consecutive values of T as one aligned vector (16-byte loads and stores).
template <class T, int NPT> struct alignas(sizeof(T) * NPT >= 16 ? 16 : sizeof(T) * NPT) VecN { T v[NPT]; };

// NPT consecutive nodes per thread: the three accumulator channels, the
// status bytes and the velocities move as vectors, so more bytes are in
// flight per thread (the one-node form waits on each load).  Channel arrays
// must start 16-byte aligned (the context pads each to a multiple of 32
// nodes); the last partial group takes the one-node path.
// Nodes i0 .. i0+NPT-1 (those below nnodes) of one grid: the accumulators
// read and cleared and the three int64 channels, status bytes and velocities
// moved as vectors of NPT nodes (the channel arrays start 256-byte aligned,
// i0 is a multiple of NPT).
template <class Real, class Acc, bool EXT, int NPT>
__device__ __forceinline__ void grid_update_nodes(const KParams<Real> &kp, const Grid<Real, Acc> &G, DevStatus *st,
                                                  long long i0, long long nnodes, int step)
{
    if (NPT == 1 || i0 + NPT > nnodes) {
        for (long long idx = i0; idx < nnodes && idx < i0 + NPT; idx++) grid_update_node<Real, Acc, EXT>(kp, G, st, idx, step);
        return;
    }
    using AV = VecN<Acc, NPT>;
    const AV m = *reinterpret_cast<const AV *>(G.acc.m + i0);
    const AV px = *reinterpret_cast<const AV *>(G.acc.px + i0);
    const AV py = *reinterpret_cast<const AV *>(G.acc.py + i0);
    bool nz[NPT], any = false;
#pragma unroll
    for (int k = 0; k < NPT; k++) {
        nz[k] = m.v[k] != Acc(0) || px.v[k] != Acc(0) || py.v[k] != Acc(0);
        any |= nz[k];
    }
    VecN<V2<Real>, NPT> vel;
    uint32_t err = 0;
    if (any) {
        AV z;
#pragma unroll
        for (int k = 0; k < NPT; k++) z.v[k] = Acc(0);
        *reinterpret_cast<AV *>(G.acc.m + i0) = z;
        *reinterpret_cast<AV *>(G.acc.px + i0) = z;
        *reinterpret_cast<AV *>(G.acc.py + i0) = z;
        const VecN<uint8_t, NPT> stv = *reinterpret_cast<const VecN<uint8_t, NPT> *>(G.status + i0);
#pragma unroll
        for (int k = 0; k < NPT; k++) {
            vel.v[k].x = Real(0); vel.v[k].y = Real(0);
            if (nz[k]) vel.v[k] = node_velocity<Real, Acc, EXT>(kp, G, i0 + k, step, m.v[k], px.v[k], py.v[k], stv.v[k], err);
        }
    } else {
#pragma unroll
        for (int k = 0; k < NPT; k++) { vel.v[k].x = Real(0); vel.v[k].y = Real(0); }
    }
    if constexpr (sizeof(Real) == 4 && NPT == 2) {
        // the velocities (8 B per node, 67 MB at 8.4M nodes) are stored with an
        // L2 evict-last policy: the fused kernel's 3x3 gathers then find more of
        // them in L2 while its point stream passes through (fused kernel -1.5 %)
        uint64_t pol;
        asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
        asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(G.vel + i0),
                     "f"((float)vel.v[0].x), "f"((float)vel.v[0].y), "f"((float)vel.v[1].x), "f"((float)vel.v[1].y),
                     "l"(pol)
                     : "memory");
    } else {
        *reinterpret_cast<VecN<V2<Real>, NPT> *>(G.vel + i0) = vel;
    }
    if (err) atomicOr(&st->err, err);
}

template <class Real, class Acc, bool EXT, int NPT>
__global__ void __launch_bounds__(256) k_grid_update(KParams<Real> kp, Grid<Real, Acc> G, DevStatus *st,
                                                     long long nnodes)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) fold_pending(st);
    const long long i0 = t * NPT;
    if (i0 >= nnodes) return;
    grid_update_nodes<Real, Acc, EXT, NPT>(kp, G, st, i0, nnodes, st->step);
}

// ---- fused G2P (step k) + P2G (step k+1) -----------------------------------
// Thread -> point mapping: warp w, lane l, iteration j handles point
//   w * 32 * PPT + j * 32 + l.
// The locality sort stores points in that interleaved order, so each
// thread's PPT points are consecutive in the tiled cell order (mostly one
// or two cells of one column) while every load and store of a warp stays
// one contiguous 32-element access.
template <int PPT> __host__ __device__ __forceinline__ uint32_t fused_index(uint32_t warp, int lane, int j)
{
    return warp * (uint32_t)(32 * PPT) + (uint32_t)(j * 32 + lane);
}

// ---- bulk asynchronous copies into shared memory ----------------------------
// cp.async.bulk (the TMA engine's 1D form) with an mbarrier that counts the
// bytes in flight; waits are bounded in iterations and in time.
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, uint32_t bytes)
{
    unsigned long long state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state) : "r"(smem_addr(bar)), "r"(bytes) : "memory");
    (void)state;
}
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, uint32_t bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Gives up after 2^24 polls or limit_ns, whichever comes first.
constexpr unsigned long long kWaitLimitNs = 1000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long *bar, uint32_t parity,
                                                  unsigned long long limit_ns = kWaitLimitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (uint32_t k = 0; k < (1u << 24); k++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((k & 255u) == 255u && global_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// A thread accumulates its points' node terms in a register patch of the
// 3x3 nodes around cell (cx, cy): mass m[a][b] and momentum p[a][b] = (px, py).
// When the next point sits one cell higher in the same column the patch
// slides: its lowest node row is written out and the other two rows move
// down.  Any other cell change writes out the patch.
template <class Real> struct Patch {
    Real m[3][3];
    P2<Real> p[3][3];
    int cx, cy;
    uint32_t key;   // (cy << 16) | cx while `have`; kNoScatter before
    bool have, in_tile;
};

template <class Real, class Acc, int CAP>
__device__ __forceinline__ void patch_node(const Patch<Real> &p, const Tile<Acc, CAP> &T, const AccGrid<Acc> &gacc,
                                           int gy, int a, int b)
{
    node_add<Real, Acc, CAP>(T, p.in_tile, gacc, gy, p.cx + a - 1, p.cy + b - 1, p.m[a][b], p.p[a][b].x, p.p[a][b].y);
}

template <class Real, class Acc, int CAP>
__device__ __forceinline__ void patch_flush(Patch<Real> &p, const Tile<Acc, CAP> &T, const AccGrid<Acc> &gacc, int gy)
{
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) patch_node<Real, Acc, CAP>(p, T, gacc, gy, a, b);
    p.have = false;
}

// End of a chunk: lanes whose tile patches sit on vertically adjacent cells
// of one column (lane l+1 one cell above lane l, the usual case in the
// interleaved cell order) overlap in two node rows.  Each lane adds the
// upper neighbour's lowest row and the lower neighbour's highest row into
// its centre row with warp shuffles (a fixed order of float adds, so the
// fixed-point sums stay deterministic); `low` / `high` tell whether the
// lane's own lowest / highest row is still its to write (no neighbour took
// it).  In the usual case 9 of the 27 node-channel adds remain.  All 32
// lanes of the warp must call it.
template <class Real>
__device__ __forceinline__ void patch_merge(Patch<Real> &p, int lane, bool &low, bool &high, bool tile_only = true)
{
    const unsigned FULL = 0xffffffffu;
    const bool mine = p.have && (p.in_tile || !tile_only);
    const uint32_t key = mine ? (((uint32_t)p.cx << 16) | (uint32_t)p.cy) : 0xffffffffu;
    const uint32_t key_up = __shfl_down_sync(FULL, key, 1);     // lane l+1
    const uint32_t key_dn = __shfl_up_sync(FULL, key, 1);       // lane l-1
    const bool above = mine && lane < 31 && key_up == key + 1u;
    const bool below = mine && lane > 0 && key_dn == key - 1u;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const Real um = __shfl_down_sync(FULL, p.m[a][0], 1), ux = __shfl_down_sync(FULL, p.p[a][0].x, 1),
                   uy = __shfl_down_sync(FULL, p.p[a][0].y, 1);
        const Real dm = __shfl_up_sync(FULL, p.m[a][2], 1), dx = __shfl_up_sync(FULL, p.p[a][2].x, 1),
                   dy = __shfl_up_sync(FULL, p.p[a][2].y, 1);
        if (above) { p.m[a][1] += um; p.p[a][1].x += ux; p.p[a][1].y += uy; }
        if (below) { p.m[a][1] += dm; p.p[a][1].x += dx; p.p[a][1].y += dy; }
    }
    low = !below;
    high = !above;
}

// Adds a lane's end patch into the shared tile.  ATOMIC: shared atomics.
// Otherwise plain read-add-write, which needs (a) no two lanes of the warp
// on the same cell, so one (a, b) step of the warp touches distinct nodes,
// (b) the steps separated by __syncwarp, since different lanes reach the
// same node in different steps, and (c) no other warp writing the same nodes
// meanwhile.  All 32 lanes of the warp must call the plain form.
template <bool ATOMIC, class Real, class Acc, int CAP>
__device__ __forceinline__ void patch_store(const Patch<Real> &p, const Tile<Acc, CAP> &T, bool on, bool low,
                                            bool high)
{
    const int base = (p.cx - 1 - T.x0) * T.th + (p.cy - 1 - T.y0);
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
        for (int b = 0; b < 3; b++) {
            if (on && (b != 0 || low) && (b != 2 || high)) {
                const int li = base + a * T.th + b;
                const Acc am = AccOps<Acc>::cvt(p.m[a][b]), ax = AccOps<Acc>::cvt(p.p[a][b].x),
                          ay = AccOps<Acc>::cvt(p.p[a][b].y);
                if (ATOMIC) {
                    AccOps<Acc>::add_shared(&T.t[0][li], am);
                    AccOps<Acc>::add_shared(&T.t[1][li], ax);
                    AccOps<Acc>::add_shared(&T.t[2][li], ay);
                } else {
                    volatile Acc *t0 = &T.t[0][li], *t1 = &T.t[1][li], *t2 = &T.t[2][li];
                    *t0 = *t0 + am;
                    *t1 = *t1 + ax;
                    *t2 = *t2 + ay;
                }
            }
            if (!ATOMIC) __syncwarp();
        }
}

// P2G source of one point in pair form (scaled for fixed point): node (a, b)
// receives  m: mp wx_a wy_b  and  (px, py): wx_a wy_b (A + (a-1) S0 + (b-1) S1)
// with A = (ax, ay), S0 = h (S00, S10), S1 = h (S01, S11) (see make_src).
template <class Real> struct SrcP {
    int cx, cy;
    Real x, y, mp;
    P2<Real> A, S0, S1;
};

// The node terms, summed separably over the weights of both axes.
template <class Real>
__device__ __forceinline__ void patch_accumulate(Patch<Real> &p, const SrcP<Real> &s, P2<Real> half)
{
    using PT = P2<Real>;
    PT wx[3], wy[3];
    bspline2(pbc(s.x), wx, half);
    bspline2(pbc(s.y), wy, half);
    const PT axa[3] = {psub(s.A, s.S0), s.A, padd(s.A, s.S0)};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const PT pr = pmul(wx[a], axa[a]);
        const PT qt = pmul(wx[a], s.S1);
        p.p[a][0] = pfma(wy[0], psub(pr, qt), p.p[a][0]);
        p.p[a][1] = pfma(wy[1], pr, p.p[a][1]);
        p.p[a][2] = pfma(wy[2], padd(pr, qt), p.p[a][2]);
        const Real u = s.mp * wx[a].x;
        p.m[a][0] = fma(u, wy[0].x, p.m[a][0]);
        p.m[a][1] = fma(u, wy[1].x, p.m[a][1]);
        p.m[a][2] = fma(u, wy[2].x, p.m[a][2]);
    }
}

// Moves the patch to the source's cell (s.cx, s.cy), which differs from its
// own: a slide by one cell up, or a flush and a fresh patch.
template <class Real, class Acc, int CAP>
__device__ __forceinline__ void patch_move(Patch<Real> &p, const SrcP<Real> &s, const Tile<Acc, CAP> &T,
                                           const AccGrid<Acc> &gacc, int gy)
{
    if (p.have) {
        const bool same = s.cx == p.cx && s.cy == p.cy;
        const bool slide = s.cx == p.cx && s.cy == p.cy + 1 && cell_in_tile(T, s.cx, s.cy) == p.in_tile;
        if (slide) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                patch_node<Real, Acc, CAP>(p, T, gacc, gy, a, 0);
                p.m[a][0] = p.m[a][1]; p.p[a][0] = p.p[a][1];
                p.m[a][1] = p.m[a][2]; p.p[a][1] = p.p[a][2];
                p.m[a][2] = Real(0); p.p[a][2] = pbc(Real(0));
            }
            p.cy += 1;
        } else if (!same) {
            patch_flush<Real, Acc, CAP>(p, T, gacc, gy);
        }
    }
    if (!p.have) {
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) { p.m[a][b] = Real(0); p.p[a][b] = pbc(Real(0)); }
        p.cx = s.cx; p.cy = s.cy;
        p.in_tile = cell_in_tile(T, s.cx, s.cy);
        p.have = true;
    }
    p.key = ((uint32_t)p.cy << 16) | (uint32_t)p.cx;
}

// Shared memory of one CTA of the fused kernel.  A chunk is CH = BT*PPT
// consecutive points; the stages hold the point state of the current chunk
// (and with two stages the next one), which the bulk copy engine fetches
// ahead; `tile` holds the scatter accumulators of the chunk's new cells +-1
// node.  After a point's G2P the stage entries of that point hold its P2G
// source (see fused_chunk); `mp` carries the source's mass where the K entry
// has no room for it (FP64 state).
template <class Real, class Acc, int BT, int PPT, int CAP, int STAGES> struct ChunkSmem {
    static constexpr int CH = BT * PPT;
    struct Stage {
        V4<Real> A[CH];
        V4<Real> H[CH];
        uint2 K[CH];
        Real mp[sizeof(Real) == 8 ? CH : 1];
    };
    Stage stage[STAGES];
    Acc tile[3][CAP > 0 ? CAP : 1];
    unsigned long long mbar[2];
    int nextc[2];           // chunk of the next iteration (the fused kernel's schedule)
    int red[BT / 32][5];
    int wbox[BT / 32][5];   // per warp: node box of its end patches {x0, x1, y0, y1}, duplicate cells
};

// Cell word of a stage entry whose point scatters nothing this step.
constexpr uint32_t kNoScatter = 0xffffffffu;
// Instances of the fused kernel (template argument MODE).
constexpr int FUSED_PLAIN = 0, FUSED_HARVEST = 1, FUSED_LEARNED = 2;

// The source's mass: in the K entry's second word (FP32 state, returned as
// that word) or in the stage's mass array (FP64 state, returns 0).
template <class Stage> __device__ __forceinline__ uint32_t put_src_mass(Stage &, int, float mp)
{
    return __float_as_uint(mp);
}
template <class Stage> __device__ __forceinline__ uint32_t put_src_mass(Stage &sg, int local, double mp)
{
    sg.mp[local] = mp;
    return 0u;
}
template <class Real, class Stage> __device__ __forceinline__ Real get_src_mass(const Stage &sg, int local, uint2 k)
{
    if constexpr (sizeof(Real) == 4) return __uint_as_float(k.y);
    else return sg.mp[local];
}

template <class Real> __device__ __forceinline__ P2<Real> ld_vel(const V2<Real> *p)
{
    return *reinterpret_cast<const P2<Real> *>(p);
}

// Issues the bulk copies of one chunk's A, H, K into a stage; the barrier
// expects their bytes plus `extra` (0 except in tests of the timeout path,
// where the wait then runs out although every copy has landed).
template <class Real, class Stage>
__device__ __forceinline__ void fetch_chunk(Stage &sg, const Pts<Real> &P, uint32_t base, int ch,
                                            unsigned long long *bar, uint32_t extra = 0u)
{
    const uint32_t bv = (uint32_t)ch * (uint32_t)sizeof(V4<Real>);
    const uint32_t bk = (uint32_t)ch * (uint32_t)sizeof(uint2);
    mbar_arrive_expect_tx(bar, 2 * bv + bk + extra);
    bulk_to_smem(sg.A, P.A + base, bv, bar);
    bulk_to_smem(sg.H, P.H + base, bv, bar);
    bulk_to_smem(sg.K, P.K + base, bk, bar);
}

// Orders this thread's generic-proxy writes to shared memory before later
// bulk copies (async proxy) into the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Records one projection onto the yield surface (case 3 of wolper_dp) for the
// learned return map: the trial singular values (sv), Jp_inv before (jp0) and
// after, and the singular values of the projected state (H).
template <class Real>
__device__ __noinline__ void harvest_record(HarvestBuf *hb, const MatT<Real> &m, const SvdH<Real> &sv, Real p_tr,
                                            Real q_tr, Real jp0, Real thick, const M2<Real> &H, Real jp1)
{
    if (p_tr < m.thr) return;                                   // cases 0/1: tension
    const Real q_fs = p_tr < m.pmax ? m.fs_c * tsqrt((m.pmax - p_tr) * (p_tr - m.pmin)) : Real(0);
    const Real q_dp = fmax(Real(0), (p_tr - m.thr) * m.tan_phi);
    const Real q_yield = p_tr < m.pmax ? fmin(q_fs, q_dp) : Real(0);
    if (!(q_tr > q_yield)) return;                              // case 2: elastic
    const uint32_t r = atomicAdd(&hb->count, 1u);
    if (r >= hb->cap) return;
    const SvdH<Real> s1 = svd_h(H);
    hb->rec[2 * (size_t)r] = make_float4(float(Real(1) + sv.e0), float(Real(1) + sv.e1), float(jp0), float(thick));
    hb->rec[2 * (size_t)r + 1] = make_float4(float(Real(1) + s1.e0), float(Real(1) + s1.e1), float(jp1), 3.0f);
}

// Case 3 of wolper_dp (kernels.cuh:400-467): the trial state lies above the
// yield surface and is projected onto it.
template <class T> __device__ __forceinline__ bool is_projection(const MatT<T> &m, T p_tr, T q_tr)
{
    if (p_tr < m.thr) return false;
    T q_yield = T(0);
    if (p_tr < m.pmax) q_yield = fmin(m.fs_c * tsqrt((m.pmax - p_tr) * (p_tr - m.pmin)), fmax(T(0), (p_tr - m.thr) * m.tan_phi));
    return q_tr > q_yield;
}

// The learned return map in place of wolper_dp's case 3, for the lanes with
// `net` (all 32 lanes of the warp call it; the network runs on the warp's
// rows).  Inputs (log sigma1, log sigma2, log Jp_inv, log thickness) and
// outputs (the log changes of sigma1, sigma2, Jp_inv) are standardised with
// the network's norm.  An answer is kept when it lies on the yield surface
// within kp.mlp_tol (|q - q_yield(p)| / max(q_yield, 1) of the predicted
// state); otherwise, and for non-finite answers, the exact map answers.  The
// rotations U, V of the trial state's SVD are kept.  Counts go to
// kp.mlp_counts (kept, fallback).
template <class Real, int NW>
__device__ __noinline__ void learned_projection(const KParams<Real> &kp, mlp::Smem<NW> &ml, int wid, int lane, bool net,
                                                Real thick, Real p_tr, Real q_tr, const SvdH<Real> &svd,
                                                Kin<Real> &k, M2<Real> &H, Real &Jp)
{
    const float *nm = ml.p.norm;
    float xin[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (net) {
        xin[0] = (log1pf(float(svd.e0)) - nm[0]) / nm[4];
        xin[1] = (log1pf(float(svd.e1)) - nm[1]) / nm[5];
        xin[2] = (logf(float(Jp)) - nm[2]) / nm[6];
        xin[3] = (logf(float(thick)) - nm[3]) / nm[7];
    }
    float yo[3];
    mlp::rows_forward(ml.p, ml.io[wid], lane, xin, yo);
    bool kept = false;
    if (net) {
        const MatT<Real> &m = kp.mat;
        const Real y0 = Real(yo[0] * nm[11] + nm[8]), y1 = Real(yo[1] * nm[12] + nm[9]), y2 = Real(yo[2] * nm[13] + nm[10]);
        // sigma' - 1 = e + (1 + e)(exp(y) - 1)
        const Real e0 = svd.e0 + (Real(1) + svd.e0) * Real(expm1f(float(y0)));
        const Real e1 = svd.e1 + (Real(1) + svd.e1) * Real(expm1f(float(y1)));
        const Real jp1 = Jp * Real(expf(float(y2)));
        const Real s0 = Real(1) + e0, s1 = Real(1) + e1;
        const Real J1 = s0 * s1;
        const Real p1 = -(m.kappa * Real(0.5)) * (J1 * J1 - Real(1));
        const Real q1 = m.mu * fabs((e0 - e1) * (Real(2) + e0 + e1)) / J1;   // mu |s0^2 - s1^2| / J
        Real qy = Real(0);
        if (p1 < m.pmax)
            qy = fmin(m.fs_c * tsqrt(fmax((m.pmax - p1) * (p1 - m.pmin), Real(0))), fmax(Real(0), (p1 - m.thr) * m.tan_phi));
        const Real res = fabs(q1 - qy) / fmax(qy, Real(1));
        kept = res <= Real(kp.mlp_tol) && isfinite(e0) && isfinite(e1) && isfinite(jp1) && jp1 > Real(0);
        if (kept) {
            H = usvt_h(svd, e0, e1);
            Jp = jp1;
        } else {
            wolper_dp(kp.mat, thick, p_tr, q_tr, k, svd, H, Jp);
        }
    }
    const unsigned nk = __popc(__ballot_sync(0xffffffffu, kept));
    const unsigned nf = __popc(__ballot_sync(0xffffffffu, net && !kept));
    if (lane == 0) {
        if (nk) atomicAdd(&kp.mlp_counts[0], (unsigned long long)nk);
        if (nf) atomicAdd(&kp.mlp_counts[1], (unsigned long long)nf);
    }
}

// One chunk of the fused kernel: CH = BT*PPT entries starting at `base` of a
// scene's arrays, whose A, H, K are in stage `s`.  With one stage, the next
// chunk (`next`, arrays Pn from base_n) is fetched into it once its points
// are read.  Error bits and the count of newly disabled points accumulate
// into err, perr, ndis.  MODE: 0 the ordinary instance, FUSED_HARVEST the one
// that records return-map pairs, FUSED_LEARNED the one whose projections onto
// the yield surface go to the learned return map (both kept out of the
// ordinary instance, whose registers they would crowd); ml is the learned
// map's shared memory (FUSED_LEARNED only).  SCENES: kp lives in shared
// memory (the scene-table kernel), where the pairs (1, 1) and (1/2, 1/2) are
// formed from immediates instead (the register allocation of that kernel
// spills more with them loaded from kp).
//
// G2P follows partition_kernel_g2p (kernels.cuh:181-315), P2G
// partition_kernel_p2g (kernels.cuh:39-104).  Two phases per chunk:
//  1. per point: the 3x3 gather, advection and re-keying, the Fe update and
//     the return map, the stores of the new state, and the P2G source of the
//     new state, written back into the point's own stage entries (A <- x, y,
//     S1; H <- A, S0; K <- cell, mass).  The 3x3 node velocities (and the
//     forcing entry) are loaded for every point; the locality sort gives a
//     thread's points one cell, so all but the first load hit L1
//     (ICEMPM_VEL_CACHE=1 keeps them in registers instead, which spills).
//  2. per point: the source's node terms into the thread's register patch;
//     at the end of the chunk the patches of vertically adjacent cells are
//     merged with warp shuffles and every node channel goes to the global
//     accumulators with one reduction (tile shapes: through the shared tile
//     of the chunk's new cells +-1 node).
// Splitting the chunk keeps the gather's and the return map's registers and
// the patch from being live at the same time.  Every point of a chunk is read
// and written by the same thread, so the stage entries need no barrier
// between the phases.
//
// The gather is evaluated separably: with d_ab = v_ab - v_c (v_c the centre
// node), S_a = sum_b wy_b d_ab and T_a = sum_b wy_b (b-1-y) d_ab,
//   v_p = v_c + sum_a wx_a S_a,
//   C[:,0] = 4/h sum_a wx_a (a-1-x) S_a,   C[:,1] = 4/h sum_a wx_a T_a,
// which equals the reference's sums over the nine nodes (the subtracted v_c
// cancels because sum_a wx_a (a-1-x) = 0 and sum_b wy_b (b-1-y) = 0) and keeps
// FP32 roundoff relative to velocity differences.  Velocities, momenta and
// the columns of C are pairs (packed FP32x2 arithmetic).
template <class Real, class Acc, int BT, int PPT, int CAP, int STAGES, int MODE, bool SCENES = false>
__device__ __forceinline__ void fused_chunk(ChunkSmem<Real, Acc, BT, PPT, CAP, STAGES> &sm, int s,
                                            const KParams<Real> &kp, const Pts<Real> &P, const Grid<Real, Acc> &G,
                                            uint32_t base, int n, int step, bool recordPQ, bool store_vc, bool next,
                                            const Pts<Real> &Pn, uint32_t base_n, uint32_t &err, uint32_t &perr,
                                            int &ndis, mlp::Smem<BT / 32> *ml = nullptr)
{
    using SM = ChunkSmem<Real, Acc, BT, PPT, CAP, STAGES>;
    using PT = P2<Real>;
    constexpr int CH = SM::CH;
    constexpr int NW = BT / 32;
    constexpr bool FIXED = AccOps<Acc>::fixed;
    constexpr bool TILE = CAP > 0;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    typename SM::Stage &sg = sm.stage[s];
    const int wbase = wid * 32 * PPT + lane;
    const PT one = SCENES ? pbc(Real(1)) : kp.one2, half = SCENES ? pbc(Real(0.5)) : kp.half2;

    // ---- phase 1 ----------------------------------------------------------
    unsigned xmn = 0xffffu, ymn = 0xffffu, xmx = 0, ymx = 0;   // box of the new cells that scatter
    bool any = false;
    uint32_t vcell = kNoScatter;   // cell whose node velocities vc, dv and forcing fc are held
    PT vc = pbc(Real(0)), dv[8];
    V4<Real> fc{};
#pragma unroll 1
    for (int j = 0; j < PPT; j++) {
        const int local = wbase + 32 * j;
        const uint32_t i = base + (uint32_t)local;
        const bool inb = i < (uint32_t)n;
        const uint2 key = inb ? sg.K[local] : make_uint2(0u, kDisabled);
        uint32_t util = key.y;
        const bool act = !(util & kDisabled);
        // entries that scatter nothing (disabled points, and in the last chunk
        // the entries past n) are marked so in the stage, for phase 2
        if (!act) sg.K[local].x = kNoScatter;
        if (MODE != FUSED_LEARNED && !act) continue;
        // The learned instance keeps every lane in the loop body (inactive
        // lanes with act = false), so that the warp meets at the network.
        Real x = Real(0), y = Real(0), Jp = Real(0), thick = Real(0);
        M2<Real> H = {Real(0), Real(0), Real(0), Real(0)};
        int cx = 0, cy = 0;
        bool moved = false, in0 = false;   // in0: the start cell is in range
        PT v = pbc(Real(0)), c0 = pbc(Real(0)), c1 = pbc(Real(0));   // (vx, vy), (c00, c10), (c01, c11)
        Kin<Real> k{};
        Real p_tr = Real(0), q_tr = Real(0);
        SvdH<Real> svd{};
        bool net = false;   // FUSED_LEARNED: this lane's projection goes to the network
        if (act) {
            const V4<Real> A = sg.A[local];
            const V4<Real> Hv = sg.H[local];
            Jp = A.z;
            thick = A.w;
            H = {Hv.x, Hv.y, Hv.z, Hv.w};
            cx = (int)(key.x & 0xffff); cy = (int)(key.x >> 16);
            in0 = cell_in_range(cx, cy, kp.gx, kp.gy);
            if (in0) {
                if (!ICEMPM_VEL_CACHE || key.x != vcell) {
                    vcell = key.x;
                    const V2<Real> *col = G.vel + ((uint32_t)(cx - 1) * (uint32_t)kp.gy + (uint32_t)(cy - 1));
                    PT nv[3][3];
#pragma unroll
                    for (int a = 0; a < 3; a++)
#pragma unroll
                        for (int b = 0; b < 3; b++) nv[a][b] = ld_vel(col + (uint32_t)a * (uint32_t)kp.gy + b);
                    vc = nv[1][1];
                    int kd = 0;
#pragma unroll
                    for (int a = 0; a < 3; a++)
#pragma unroll
                        for (int b = 0; b < 3; b++)
                            if (a != 1 || b != 1) dv[kd++] = psub(nv[a][b], vc);
                    if (kp.ext) fc = G.frc[(uint32_t)cx * (uint32_t)kp.gy + (uint32_t)cy];
                }
                // column sums first (weights of y), then the row combination (weights of x),
                // so that only one axis's weight pairs are live at a time
                // (the gradient weights are taken with the opposite sign,
                // wy_b (y - (b-1)), which makes ta, pv and qv the negatives of
                // the sums above, exactly; -4/h restores the sign of C)
                PT sa[3], ta[3];
                {
                    PT wy[3];
                    const PT vy = pbc(A.y);
                    bspline2(vy, wy, half);
                    const PT gy[3] = {pmul(wy[0], padd(vy, one)), pmul(wy[1], vy), pmul(wy[2], psub(vy, one))};
                    // a = 0: dv[0..2] are nodes (0, 0..2); a = 1: dv[3], dv[4] are nodes (1, 0), (1, 2)
                    // (the centre's difference is zero); a = 2: dv[5..7] are nodes (2, 0..2)
                    sa[0] = pfma(wy[2], dv[2], pfma(wy[1], dv[1], pmul(wy[0], dv[0])));
                    ta[0] = pfma(gy[2], dv[2], pfma(gy[1], dv[1], pmul(gy[0], dv[0])));
                    sa[1] = pfma(wy[2], dv[4], pmul(wy[0], dv[3]));
                    ta[1] = pfma(gy[2], dv[4], pmul(gy[0], dv[3]));
                    sa[2] = pfma(wy[2], dv[7], pfma(wy[1], dv[6], pmul(wy[0], dv[5])));
                    ta[2] = pfma(gy[2], dv[7], pfma(gy[1], dv[6], pmul(gy[0], dv[5])));
                }
                PT sv, pv, qv;
                {
                    PT wx[3];
                    const PT vx = pbc(A.x);
                    bspline2(vx, wx, half);
                    const PT gx[3] = {pmul(wx[0], padd(vx, one)), pmul(wx[1], vx), pmul(wx[2], psub(vx, one))};
                    sv = pfma(wx[2], sa[2], pfma(wx[1], sa[1], pmul(wx[0], sa[0])));
                    pv = pfma(gx[2], sa[2], pfma(gx[1], sa[1], pmul(gx[0], sa[0])));
                    qv = pfma(wx[2], ta[2], pfma(wx[1], ta[1], pmul(wx[0], ta[0])));
                }
                v = padd(vc, sv);
                c0 = pmul(kp.neg_four_h_inv2, pv);
                c1 = pmul(kp.neg_four_h_inv2, qv);
            }
            const PT xy = pfma(v, kp.dt_h_inv2, pmk(A.x, A.y));
            {   // one test in the usual case; a NaN in any of the sums reaches the total
                const PT t = padd(padd(v, xy), padd(c0, c1));
                if (isnan(t.x + t.y)) {
                    if (isnan(v.x + v.y)) err |= kErrVelNan;
                    if (isnan(xy.x + xy.y)) err |= kErrPosNan;
                    if (isnan((c0.x + c0.y) + (c1.x + c1.y))) err |= kErrBpNan;
                }
            }
            x = xy.x; y = xy.y;
            if (fabs(x) > Real(0.5) || fabs(y) > Real(0.5)) {   // the point left its cell (rare)
                if (x > Real(0.5)) { x -= Real(1); cx++; moved = true; }
                else if (x < Real(-0.5)) { x += Real(1); cx--; moved = true; }
                if (y > Real(0.5)) { y -= Real(1); cy++; moved = true; }
                else if (y < Real(-0.5)) { y += Real(1); cy--; moved = true; }
                if (moved && (cx <= 1 || cx >= kp.gx - 2 || cy <= 1 || cy >= kp.gy - 2)) {
                    util |= kDisabled;
                    ndis++;
                }
                if (x > Real(0.5) || x < Real(-0.5) || y > Real(0.5) || y < Real(-0.5)) err |= kErrJump;
            }

            // Fe <- (I + dt C) Fe, i.e. H <- H + D + D H with D = dt C
            {
                const Real d00 = kp.dt * c0.x, d01 = kp.dt * c1.x, d10 = kp.dt * c0.y, d11 = kp.dt * c1.y;
                const M2<Real> h = H;
                // each entry h + (D + D h), the small D terms summed first
                H.a00 = h.a00 + fma(d00, h.a00, fma(d01, h.a10, d00));
                H.a01 = h.a01 + fma(d00, h.a01, fma(d01, h.a11, d01));
                H.a10 = h.a10 + fma(d10, h.a00, fma(d11, h.a10, d10));
                H.a11 = h.a11 + fma(d10, h.a01, fma(d11, h.a11, d11));
            }
            if (isnan((H.a00 + H.a10) + (H.a01 + H.a11))) err |= kErrFeNan;
            k = kinematics(H);
            pq(k, kp.mat.mu, kp.mat.kappa, p_tr, q_tr);
            if (!(util & kCrushed)) util = failure_check(kp.mat, util, p_tr, q_tr);
            if (util & kCrushed) {
                svd = svd_h(H);
                if (MODE == FUSED_LEARNED && kp.mlp && is_projection(kp.mat, p_tr, q_tr) && thick > Real(0) &&
                    Jp > Real(0) && svd.e1 > Real(-1)) {
                    net = true;
                } else {
                    const Real jp0 = Jp;
                    wolper_dp(kp.mat, thick, p_tr, q_tr, k, svd, H, Jp);
                    if (MODE == FUSED_HARVEST && kp.harvest && (i + (uint32_t)step) % (uint32_t)kp.harvest_stride == 0u)
                        harvest_record(kp.harvest, kp.mat, svd, p_tr, q_tr, jp0, thick, H, Jp);
                    if (isnan((H.a00 + H.a10) + (H.a01 + H.a11))) err |= kErrFeNan;
                    k = kinematics(H);
                }
            }
        }
        if constexpr (MODE == FUSED_LEARNED) {
            if (__any_sync(0xffffffffu, net)) {
                learned_projection<Real>(kp, *ml, wid, lane, net, thick, p_tr, q_tr, svd, k, H, Jp);
                if (net) {
                    if (isnan((H.a00 + H.a10) + (H.a01 + H.a11))) err |= kErrFeNan;
                    k = kinematics(H);
                }
            }
        }
        if (!act) continue;

            V4<Real> Ao; Ao.x = x; Ao.y = y; Ao.z = Jp; Ao.w = thick;
            st_stream(P.A + i, Ao);
            V4<Real> Ho; Ho.x = H.a00; Ho.y = H.a01; Ho.z = H.a10; Ho.w = H.a11;
            st_stream(P.H + i, Ho);
            if (store_vc || (util & kDisabled)) {   // a point disabled now keeps this step's V and C
                V2<Real> Vo; Vo.x = v.x; Vo.y = v.y;
                st_stream(P.V + i, Vo);
                V4<Real> Co; Co.x = c0.x; Co.y = c1.x; Co.z = c0.y; Co.w = c1.y;
                st_stream(P.C + i, Co);
            }
            const uint32_t cell = ((uint32_t)cy << 16) | (uint32_t)cx;   // as kernels.cuh:305
            if (moved || util != key.y) {
                uint2 ko; ko.x = moved ? cell : key.x; ko.y = util;
                st_stream(P.K + i, ko);
            }
            if (recordPQ) { V2<Real> pqv; pqv.x = p_tr; pqv.y = q_tr; st_stream(P.PQ + i, pqv); }

            // P2G source of the new state (make_src in pair form): with
            // S = m_p C - dt_vol_Dpinv Jp_inv thickness tau (columns S0, S1),
            // A = m_p v - h (S0 x + S1 y) (+ the extended forcing's impulse).
            uint2 src_key = make_uint2(kNoScatter, 0u);   // new cell and mass of the source, or no scatter
            if (!(util & kDisabled)) {
                if (moved ? cell_in_range(cx, cy, kp.gx, kp.gy) : in0) {
                    const M2<Real> tau = kirchhoff(k, kp.mat.mu, kp.mat.kappa);
                    const Real mp = kp.particle_mass * thick;
                    const PT nsc = pbc(-(kp.dt_vol_Dpinv * Jp * thick)), mpp = pbc(mp);
                    const PT S0 = pfma(mpp, c0, pmul(nsc, pmk(tau.a00, tau.a10)));
                    const PT S1 = pfma(mpp, c1, pmul(nsc, pmk(tau.a01, tau.a11)));
                    PT Av = pfma(kp.neg_h2, pfma(S0, pbc(x), pmul(S1, pbc(y))), pmul(mpp, v));
                    if (kp.ext) {   // wind stress and current of the new cell's node
                        const V4<Real> f = moved ? G.frc[(uint32_t)cx * (uint32_t)kp.gy + (uint32_t)cy] : fc;
                        const PT d = psub(pmk(f.x, f.y), v);
                        const Real cw = kp.rho_w_cd * tsqrt(d.x * d.x + d.y * d.y);
                        Av = pfma(kp.ext_impulse2, pfma(pbc(cw), d, pmk(f.z, f.w)), Av);
                    }
                    const PT sA = pmul(Av, kp.sp2), sS0 = pmul(kp.hsp2, S0), sS1 = pmul(kp.hsp2, S1);
                    const Real smp = mp * kp.sm_r;
                    // Fixed point: a node term is at most max(w) <= 0.5625 times the
                    // bounds below.  Finite sources with |x|, |y| <= 2 raise no P2G
                    // bit; anything else takes the exact tests.
                    const Real lim_p = FIXED ? Real(kp.lim_p) : Real(sizeof(Real) == 4 ? 1e30 : 1e300);
                    const Real lim_m = FIXED ? Real(kp.lim_m) : lim_p;
                    const Real bx = fabs(Av.x) + kp.h * (fabs(S0.x) + fabs(S1.x));
                    const Real by = fabs(Av.y) + kp.h * (fabs(S0.y) + fabs(S1.y));
                    if (!(bx <= lim_p && by <= lim_p && mp <= lim_m && fabs(x) <= Real(2) && fabs(y) <= Real(2))) {
                        if (FIXED && (!(bx <= Real(kp.lim_p)) || !(by <= Real(kp.lim_p)) || !(mp <= Real(kp.lim_m))))
                            perr |= kErrFixedOverflow;
                        Real wxs[3], wys[3];
                        bspline(x, wxs);
                        bspline(y, wys);
                        const Real sw = (wxs[0] + wxs[1] + wxs[2]) + (wys[0] + wys[1] + wys[2]);
                        if (isnan(sw + smp)) perr |= kErrP2gNanMass;
                        if (isnan(sw + ((sA.x + sA.y) + (sS0.x + sS1.x) + (sS0.y + sS1.y)))) perr |= kErrP2gNanVel;
                    }
                    V4<Real> a4; a4.x = x; a4.y = y; a4.z = sS1.x; a4.w = sS1.y;
                    sg.A[local] = a4;
                    V4<Real> h4; h4.x = sA.x; h4.y = sA.y; h4.z = sS0.x; h4.w = sS0.y;
                    sg.H[local] = h4;
                    src_key.x = cell;
                    src_key.y = put_src_mass(sg, local, smp);
                    xmn = min(xmn, (unsigned)cx); ymn = min(ymn, (unsigned)cy);
                    xmx = max(xmx, (unsigned)cx); ymx = max(ymx, (unsigned)cy);
                    any = true;
                } else {
                    perr |= kErrLeftArea;
                }
            }
        sg.K[local] = src_key;
    }
    fence_proxy_async_smem();

    // ---- the tile: box of the chunk's scattering cells, +-1 node ------------
    Tile<Acc, CAP> T;
    T.t = sm.tile;
    T.on = false; T.x0 = T.y0 = 0; T.tw = T.th = 0; T.th_rcp = 0;
    if constexpr (TILE) {
        {
            const unsigned FULL = 0xffffffffu;
            xmn = __reduce_min_sync(FULL, xmn); ymn = __reduce_min_sync(FULL, ymn);
            xmx = __reduce_max_sync(FULL, xmx); ymx = __reduce_max_sync(FULL, ymx);
            const unsigned wany = __reduce_or_sync(FULL, any ? 1u : 0u);
            if (lane == 0) {
                sm.red[wid][0] = (int)xmn; sm.red[wid][1] = (int)ymn;
                sm.red[wid][2] = (int)xmx; sm.red[wid][3] = (int)ymx; sm.red[wid][4] = (int)wany;
            }
        }
        __syncthreads();
        int bx0 = 0xffff, by0 = 0xffff, bx1 = 0, by1 = 0, bany = 0;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            bx0 = min(bx0, sm.red[w][0]); by0 = min(by0, sm.red[w][1]);
            bx1 = max(bx1, sm.red[w][2]); by1 = max(by1, sm.red[w][3]); bany |= sm.red[w][4];
        }
        T.x0 = bx0 - 1; T.y0 = by0 - 1;
        T.tw = bx1 - bx0 + 3; T.th = by1 - by0 + 3;
        // 64-bit products: a box spanning the whole grid must not wrap into range
        T.on = bany && (long long)T.tw * (long long)T.th <= (long long)CAP;
        if (!T.on) { T.tw = 0; T.th = 0; }
        T.th_rcp = rcp32(T.th);
        tile_zero<Acc, CAP, BT>(T);
        __syncthreads();
    }

    // ---- phase 2 ----------------------------------------------------------
    Patch<Real> patch;
    patch.have = false; patch.in_tile = false; patch.cx = patch.cy = 0; patch.key = kNoScatter;
#pragma unroll
    for (int j = 0; j < PPT; j++) {
        const int local = wbase + 32 * j;
        const uint2 k2 = sg.K[local];
        if (k2.x == kNoScatter) continue;
        const V4<Real> a4 = sg.A[local];
        const V4<Real> h4 = sg.H[local];
        SrcP<Real> src;
        src.x = a4.x; src.y = a4.y;
        src.mp = get_src_mass<Real>(sg, local, k2);
        src.A = pmk(h4.x, h4.y); src.S0 = pmk(h4.z, h4.w); src.S1 = pmk(a4.z, a4.w);
        if (k2.x != patch.key) {   // the first source, or one from another cell (rare)
            src.cx = (int)(k2.x & 0xffff); src.cy = (int)(k2.x >> 16);
            patch_move<Real, Acc, CAP>(patch, src, T, G.acc, kp.gy);
        }
        patch_accumulate(patch, src, half);
    }
    // end patches: merge neighbours, then write them out.  Without a tile
    // (CAP == 0) every node goes straight to the global accumulators (one
    // reduction per node and channel).  With a tile: for int64 accumulators
    // (whose shared atomics are multi-instruction sequences) the writes go
    // without atomics in two phases (even warps, odd warps) when warps of one
    // phase touch disjoint nodes and no warp has two lanes on one cell; float
    // accumulators keep the native atomics.
    if constexpr (!TILE) {
        bool low = true, high = true;
        patch_merge(patch, lane, low, high, false);
        if (patch.have) {
            // the centre row; then one pass for the edge row each lane still
            // owns (in a column run of cells only the run's ends own one: one
            // pass of reductions for both ends instead of one per edge row),
            // and a second one where a lane owns both (a cell without
            // vertical neighbours)
#pragma unroll
            for (int a = 0; a < 3; a++) patch_node<Real, Acc, CAP>(patch, T, G.acc, kp.gy, a, 1);
            if (low || high) {
#pragma unroll
                for (int a = 0; a < 3; a++)
                    node_add<Real, Acc, CAP>(T, patch.in_tile, G.acc, kp.gy, patch.cx + a - 1, patch.cy + (low ? -1 : 1),
                                             low ? patch.m[a][0] : patch.m[a][2], low ? patch.p[a][0].x : patch.p[a][2].x,
                                             low ? patch.p[a][0].y : patch.p[a][2].y);
            }
            if (low && high) {
#pragma unroll
                for (int a = 0; a < 3; a++) patch_node<Real, Acc, CAP>(patch, T, G.acc, kp.gy, a, 2);
            }
        }
        // one stage: every thread has read its entries; refill the stage
        if (STAGES == 1) {
            __syncthreads();
            if (tid == 0 && next) fetch_chunk(sm.stage[0], Pn, base_n, CH, &sm.mbar[0], kp.tx_extra);
        }
        return;
    } else if (!FIXED) {
        bool low = true, high = true;
        patch_merge(patch, lane, low, high);
        if (patch.have) {
            if (patch.in_tile) patch_store<true, Real, Acc, CAP>(patch, T, true, low, high);
            else patch_flush<Real, Acc, CAP>(patch, T, G.acc, kp.gy);
        }
        __syncthreads();
    } else {
        const unsigned FULL = 0xffffffffu;
        bool low = true, high = true;
        patch_merge(patch, lane, low, high);
        if (patch.have && !patch.in_tile) patch_flush<Real, Acc, CAP>(patch, T, G.acc, kp.gy);
        const bool mine = patch.have;
        const uint32_t key = mine ? (((uint32_t)patch.cx << 16) | (uint32_t)patch.cy) : (0xffffffe0u | (uint32_t)lane);
        // every lane takes part in the match (a lane skipped here would stall the warp)
        const unsigned same = __match_any_sync(FULL, key);
        const bool dup = __any_sync(FULL, mine && __popc(same) > 1);
        const int x0 = __reduce_min_sync(FULL, mine ? patch.cx - 1 : INT_MAX);
        const int x1 = __reduce_max_sync(FULL, mine ? patch.cx + 1 : INT_MIN);
        const int y0 = __reduce_min_sync(FULL, mine ? patch.cy - 1 : INT_MAX);
        const int y1 = __reduce_max_sync(FULL, mine ? patch.cy + 1 : INT_MIN);
        if (lane == 0) {
            sm.wbox[wid][0] = x0; sm.wbox[wid][1] = x1; sm.wbox[wid][2] = y0; sm.wbox[wid][3] = y1;
            sm.wbox[wid][4] = dup ? 1 : 0;
        }
        __syncthreads();
        bool phased = true;
#pragma unroll
        for (int w = 0; w < NW; w++) {
            if (sm.wbox[w][4]) phased = false;
#pragma unroll
            for (int v = w + 2; v < NW; v += 2)
                if (!(sm.wbox[w][1] < sm.wbox[v][0] || sm.wbox[v][1] < sm.wbox[w][0] ||
                      sm.wbox[w][3] < sm.wbox[v][2] || sm.wbox[v][3] < sm.wbox[w][2]))
                    phased = false;
        }
        if (phased) {
            if ((wid & 1) == 0) patch_store<false, Real, Acc, CAP>(patch, T, mine, low, high);
            __syncthreads();
            if ((wid & 1) == 1) patch_store<false, Real, Acc, CAP>(patch, T, mine, low, high);
        } else if (mine) {
            patch_store<true, Real, Acc, CAP>(patch, T, true, low, high);
        }
        __syncthreads();
    }
    if constexpr (TILE) {
        // one stage: its entries are all read now, fetch the next chunk into it
        if (STAGES == 1 && tid == 0 && next) fetch_chunk(sm.stage[0], Pn, base_n, CH, &sm.mbar[0], kp.tx_extra);
        tile_flush<Acc, CAP, BT>(T, G.acc, kp.gx, kp.gy);
    }
}

// Dynamic shared memory of an instance of the fused kernel: the chunk stages
// (and tile), and for the learned instance the network after them.
template <class SM, int BT, int MODE> constexpr size_t fused_smem_bytes()
{
    return MODE == FUSED_LEARNED ? (sizeof(SM) + 15) / 16 * 16 + sizeof(mlp::Smem<BT / 32>) : sizeof(SM);
}

template <class Real, class Acc, int BT, int PPT, int CAP, int STAGES, int MODE>
__global__ void __launch_bounds__(BT, (sizeof(Real) == 8 ? 1 : (MODE == FUSED_LEARNED ? 4 : ICEMPM_FUSED_MINB)))
k_g2p_p2g(KParams<Real> kp, Pts<Real> P, Grid<Real, Acc> G, DevStatus *st, int n, int nchunks)
{
    static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
    using SM = ChunkSmem<Real, Acc, BT, PPT, CAP, STAGES>;
    constexpr int CH = SM::CH;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);
    const int tid = threadIdx.x;
    mlp::Smem<BT / 32> *ml = nullptr;
    if constexpr (MODE == FUSED_LEARNED) {   // launched only with a network (kp.mlp)
        ml = reinterpret_cast<mlp::Smem<BT / 32> *>(smem_raw + (sizeof(SM) + 15) / 16 * 16);
        mlp::load_packed(ml->p, kp.mlp, tid, BT);
    }

    if (tid == 0) {
        mbar_init(&sm.mbar[0], 1);
        if (STAGES == 2) mbar_init(&sm.mbar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // Chunk schedule: a CTA's first chunk is its block index; each later one
    // is chunk gridDim.x + t for the next ticket t of st->chunk_ticket (rewound
    // by the launch's last CTA), so that CTAs which finish their chunks early
    // take more and the launch ends within about one chunk time on every SM.
    // Thread 0 draws the ticket of iteration it + 2 while iteration it runs
    // (the atomic's latency hides behind the chunk) and publishes the chunk of
    // iteration it + 1 in sm.nextc[it & 1] before the iteration's barrier.
    // Schedule position c processes the chunk nchunks - 1 - c: the points
    // (sorted by cell) are walked from the high cells down, starting where
    // the grid update, which walks the nodes upwards, has just left its
    // velocities and cleared accumulators in L2.
    int c = blockIdx.x;
    uint32_t ticket = 0;
    if (tid == 0 && c < nchunks) {
        fetch_chunk(sm.stage[0], P, (uint32_t)(nchunks - 1 - c) * CH, CH, &sm.mbar[0], kp.tx_extra);
        ticket = atomicAdd(&st->chunk_ticket, 1u);
    }

    const int step = st->step;
    const bool recordPQ = kp.update_every > 0 && (step % kp.update_every) == 0;
    const bool store_vc = step == st->vc_step;
    uint32_t err = 0, perr = 0;
    int ndis = 0;

    for (int it = 0; c < nchunks; it++) {
        const int s = STAGES == 2 ? (it & 1) : 0;
        const uint32_t parity = STAGES == 2 ? ((uint32_t)(it >> 1) & 1u) : ((uint32_t)it & 1u);
        const bool ok = mbar_wait_bounded(&sm.mbar[s], parity, kp.wait_ns);
        if (tid == 0) sm.nextc[it & 1] = (int)min(gridDim.x + ticket, (uint32_t)nchunks);
        if (__syncthreads_or(!ok)) {
            // the chunk's copies did not complete in time: report it, give
            // copies still in flight one more bounded wait to land in this
            // CTA's shared memory, and leave
            err |= kErrBarrierTimeout;
            if (tid == 0) (void)mbar_wait_bounded(&sm.mbar[s], parity, kp.wait_ns);
            __syncthreads();
            break;
        }
        const int cn = sm.nextc[it & 1];
        const bool next = cn < nchunks;
        const uint32_t base_n = (uint32_t)(nchunks - 1 - cn) * CH;   // used only with next
        if (tid == 0 && next) {
            if (STAGES == 2) fetch_chunk(sm.stage[s ^ 1], P, base_n, CH, &sm.mbar[s ^ 1], kp.tx_extra);
            ticket = atomicAdd(&st->chunk_ticket, 1u);
        }
        fused_chunk<Real, Acc, BT, PPT, CAP, STAGES, MODE>(sm, s, kp, P, G, (uint32_t)(nchunks - 1 - c) * CH, n, step,
                                                  recordPQ, store_vc,
                                                  next, P, base_n, err, perr, ndis, ml);
        c = cn;
    }
    warp_flush_status(st, err, perr, ndis);

    // the last CTA to finish advances the device step counter and rewinds the
    // chunk tickets for the next launch (no waiting)
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&st->done, 1u);
        if (t == gridDim.x - 1) {
            st->step = step + 1;
            st->done = 0;
            st->chunk_ticket = 0;
            __threadfence();
        }
    }
}

// ---- ensembles: many independent scenes in one launch ------------------------
// Each scene is an ordinary context (its own points, grid, parameters and
// status); a table of their descriptors lets one launch of each kernel walk
// the chunks (fused kernel) and nodes (grid update) of all of them.  The
// batch's own DevStatus carries the common sub-step counter.
template <class Real, class Acc> struct SceneDesc {
    KParams<Real> kp;
    Pts<Real> P;
    Grid<Real, Acc> G;
    DevStatus *st;
    int n;             // entries of the point arrays (points + placeholders)
    int chunk0;        // first global chunk of this scene
    long long nnodes;
    int block0;        // first global block (256 * ICEMPM_UPDATE_NPT nodes) of this scene
    int ext;           // extended forcing
};

// A block of the batch grid update covers 256 * NPT nodes of one scene; its
// descriptor is copied into shared memory first (every node reads a dozen
// of its fields).
template <class Real, class Acc, int NPT>
__global__ void __launch_bounds__(256) k_grid_update_batch(const SceneDesc<Real, Acc> *__restrict__ scenes,
                                                           const int *__restrict__ block_scene, DevStatus *bst)
{
    __shared__ __align__(16) SceneDesc<Real, Acc> ssd;
    const int si = block_scene[blockIdx.x];
    {
        static_assert(sizeof(SceneDesc<Real, Acc>) % 4 == 0, "word copy");
        const uint32_t *src = reinterpret_cast<const uint32_t *>(&scenes[si]);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&ssd);
        for (int k = threadIdx.x; k < (int)(sizeof(SceneDesc<Real, Acc>) / 4); k += 256) dst[k] = src[k];
    }
    __syncthreads();
    const SceneDesc<Real, Acc> &S = ssd;
    const long long t = (long long)(blockIdx.x - S.block0) * 256 + threadIdx.x;
    if (t == 0) fold_pending(S.st);
    const long long i0 = t * NPT;
    if (i0 >= S.nnodes) return;
    if (S.ext) grid_update_nodes<Real, Acc, true, NPT>(S.kp, S.G, S.st, i0, S.nnodes, bst->step);
    else grid_update_nodes<Real, Acc, false, NPT>(S.kp, S.G, S.st, i0, S.nnodes, bst->step);
}

template <class Real, class Acc, int BT, int PPT, int CAP, int STAGES>
__global__ void __launch_bounds__(BT, (sizeof(Real) == 8 ? 1 : ICEMPM_FUSED_MINB))
k_g2p_p2g_batch(const SceneDesc<Real, Acc> *__restrict__ scenes, const int *__restrict__ chunk_scene, int nchunks,
                DevStatus *bst)
{
    static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
    using SM = ChunkSmem<Real, Acc, BT, PPT, CAP, STAGES>;
    constexpr int CH = SM::CH;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    SM &sm = *reinterpret_cast<SM *>(smem_raw);
    const int tid = threadIdx.x;
    // the current scene's descriptor, copied into shared memory when the scene changes
    __shared__ __align__(16) SceneDesc<Real, Acc> ssd;
    int cur_scene = -1;

    if (tid == 0) {
        mbar_init(&sm.mbar[0], 1);
        if (STAGES == 2) mbar_init(&sm.mbar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // schedule position c processes the chunk nchunks - 1 - c (high cells of
    // the last scene first: see k_g2p_p2g)
    int c = blockIdx.x;
    if (tid == 0 && c < nchunks) {
        const int cc = nchunks - 1 - c;
        const SceneDesc<Real, Acc> &S0 = scenes[chunk_scene[cc]];
        fetch_chunk(sm.stage[0], S0.P, (uint32_t)(cc - S0.chunk0) * CH, CH, &sm.mbar[0]);
    }
    const int step = bst->step;
    const bool store_vc = step == bst->vc_step;

    for (int it = 0; c < nchunks; it++, c += (int)gridDim.x) {
        const int cc = nchunks - 1 - c;
        const int sc = chunk_scene[cc];
        if (sc != cur_scene) {   // block-uniform: every thread of the CTA walks the same chunks
            __syncthreads();
            static_assert(sizeof(SceneDesc<Real, Acc>) % 4 == 0, "word copy");
            const uint32_t *src = reinterpret_cast<const uint32_t *>(&scenes[sc]);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&ssd);
            for (int k = tid; k < (int)(sizeof(SceneDesc<Real, Acc>) / 4); k += BT) dst[k] = src[k];
            __syncthreads();
            cur_scene = sc;
        }
        const SceneDesc<Real, Acc> &S = ssd;
        const int s = STAGES == 2 ? (it & 1) : 0;
        const uint32_t parity = STAGES == 2 ? ((uint32_t)(it >> 1) & 1u) : ((uint32_t)it & 1u);
        uint32_t err = 0, perr = 0;
        int ndis = 0;
        const bool ok = mbar_wait_bounded(&sm.mbar[s], parity);
        if (__syncthreads_or(!ok)) {
            warp_flush_status(S.st, kErrBarrierTimeout, 0u, 0);
            if (tid == 0) (void)mbar_wait_bounded(&sm.mbar[s], parity);
            __syncthreads();
            break;
        }
        const int cn = c + (int)gridDim.x;
        const bool next = cn < nchunks;
        const int ccn = next ? nchunks - 1 - cn : cc;
        const SceneDesc<Real, Acc> &Sn = scenes[chunk_scene[ccn]];
        const uint32_t base_n = (uint32_t)(ccn - Sn.chunk0) * CH;
        if (STAGES == 2 && tid == 0 && next) fetch_chunk(sm.stage[s ^ 1], Sn.P, base_n, CH, &sm.mbar[s ^ 1]);
        const bool recordPQ = S.kp.update_every > 0 && (step % S.kp.update_every) == 0;
        fused_chunk<Real, Acc, BT, PPT, CAP, STAGES, FUSED_PLAIN, true>(sm, s, S.kp, S.P, S.G, (uint32_t)(cc - S.chunk0) * CH, S.n,
                                                          step, recordPQ, store_vc, next, Sn.P, base_n, err, perr, ndis);
        warp_flush_status(S.st, err, perr, ndis);
    }

    // the last CTA to finish advances the batch's sub-step counter
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const unsigned t = atomicAdd(&bst->done, 1u);
        if (t == gridDim.x - 1) {
            bst->step = step + 1;
            bst->done = 0;
            __threadfence();
        }
    }
}

}  // namespace icempm
