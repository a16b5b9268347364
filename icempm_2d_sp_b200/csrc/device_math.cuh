// device_math.cuh -- per-point constitutive math of the 2D APIC MPM step,
// written for sm_100a.  Templated on the arithmetic type T (float or double).
//
// The deformation gradient is carried as H = Fe - I (the displacement
// gradient) instead of Fe.  Every quantity the reference derives from Fe --
// det, b = Fe Fe^T, the Kirchhoff stress, p/q, the polar rotation and the
// Jacobi rotation of the 2x2 SVD, the Drucker-Prager projection -- is
// rewritten algebraically in terms of H so that differences from identity
// (strains ~1e-4) keep full relative precision in FP32.  In exact arithmetic
// each function equals its reference counterpart (cited per function,
// simulation/kernels.cuh, helper_math.cuh, givens.cuh of igorg520b/iceMPM_2d_sp).
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace icempm {

constexpr uint32_t kCrushed = 0x10000u;
constexpr uint32_t kDisabled = 0x20000u;
constexpr uint32_t kErrPosNan = 0x0001u, kErrVelNan = 0x0002u, kErrJump = 0x0004u,
                   kErrLeftArea = 0x0008u, kErrBpNan = 0x0010u, kErrFeNan = 0x0020u,
                   kErrP2gNanVel = 0x0100u, kErrP2gNanMass = 0x0200u, kErrGridNan = 0x0400u,
                   kErrFixedOverflow = 0x1000u, kErrBarrierTimeout = 0x2000u;

template <class T> struct M2 { T a00, a01, a10, a11; };

template <class T> __device__ __forceinline__ T tsqrt(T x);
template <> __device__ __forceinline__ float tsqrt<float>(float x) { return sqrtf(x); }
template <> __device__ __forceinline__ double tsqrt<double>(double x) { return sqrt(x); }

// Quadratic B-spline weights of the three nodes -1, 0, +1 around a point at
// cell-local coordinate x in [-0.5, 0.5] (CalculateWeightCoeffs, kernels.cuh:323-332).
template <class T> __device__ __forceinline__ void bspline(T x, T w[3])
{
    const T v0 = T(0.5) - x, v2 = x + T(0.5);
    w[0] = T(0.5) * v0 * v0;
    w[1] = T(0.75) - x * x;
    w[2] = T(0.5) * v2 * v2;
}

// ---- pairs -----------------------------------------------------------------
// Two values that take the same arithmetic (the x and y components of a
// velocity, a momentum or a matrix column) travel as one pair.  For float the
// pair operations are sm_100's packed FP32x2 instructions (one instruction,
// two lanes, each rounded exactly as the scalar operation); for double they
// are two scalar operations.
template <class T> struct PairOf;
template <> struct PairOf<float> { using type = float2; };
template <> struct PairOf<double> { using type = double2; };
template <class T> using P2 = typename PairOf<T>::type;

__device__ __forceinline__ float2 pbc(float s) { return make_float2(s, s); }
__device__ __forceinline__ double2 pbc(double s) { return make_double2(s, s); }
__device__ __forceinline__ float2 pmk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 pmk(double a, double b) { return make_double2(a, b); }

__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 psub(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pr;\n\t"
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "sub.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ double2 padd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 psub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 pfma(double2 a, double2 b, double2 c)
{
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}

// B-spline weights of both components of a pair: w[k] = (w_k(v.x), w_k(v.y)).
// With v = (x, x) every w[k] is a broadcast pair.  w[1] = 0.75 - x^2 is
// formed as (0.5 - x)(x + 0.5) + 0.5.  `half` is the pair (0.5, 0.5).
template <class PT> __device__ __forceinline__ void bspline2(PT v, PT w[3], PT half)
{
    const PT v0 = psub(half, v), v2 = padd(v, half);
    w[0] = pmul(pmul(half, v0), v0);
    w[1] = pfma(v0, v2, half);
    w[2] = pmul(pmul(half, v2), v2);
}

// Kinematic invariants of F = I + H.
//   Jm1 = det(F) - 1 = tr H + det H
//   dev(b) = [[d, b01], [b01, -d]] with b = F F^T  (b - I = H + H^T + H H^T)
template <class T> struct Kin { T Jm1, J, d, b01; };
template <class T> __device__ __forceinline__ Kin<T> kinematics(const M2<T> &H)
{
    Kin<T> k;
    k.Jm1 = fma(H.a00, H.a11, fma(-H.a01, H.a10, H.a00 + H.a11));
    k.J = T(1) + k.Jm1;
    const T bm00 = fma(H.a00, H.a00, fma(H.a01, H.a01, T(2) * H.a00));
    const T bm11 = fma(H.a10, H.a10, fma(H.a11, H.a11, T(2) * H.a11));
    k.b01 = fma(H.a00, H.a10, fma(H.a01, H.a11, H.a01 + H.a10));
    k.d = T(0.5) * (bm00 - bm11);
    return k;
}

// p = -(kappa/2)(J^2-1), q = sqrt(2) mu/J |dev b|_F   (ComputePQ, kernels.cuh:337-343)
template <class T> __device__ __forceinline__ void pq(const Kin<T> &k, T mu, T kappa, T &p, T &q)
{
    p = -(kappa * T(0.5)) * (k.Jm1 * (T(2) + k.Jm1));
    const T nrm = tsqrt(T(2) * (k.d * k.d + k.b01 * k.b01));
    q = T(1.4142135623730950) * mu / k.J * nrm;
}

// Kirchhoff stress tau = mu/J dev(b) + kappa/2 (J^2-1) I = mu/J dev(b) - p I
// (KirchhoffStress_Wolper, kernels.cuh:525-535).
template <class T> __device__ __forceinline__ M2<T> kirchhoff(const Kin<T> &k, T mu, T kappa)
{
    const T a = mu / k.J;
    const T c = (kappa * T(0.5)) * (k.Jm1 * (T(2) + k.Jm1));
    M2<T> t;
    t.a00 = a * k.d + c;
    t.a01 = a * k.b01;
    t.a10 = a * k.b01;
    t.a11 = -a * k.d + c;
    return t;
}

// 2x2 SVD of F = I + H in the reference's conventions (svd2x2 over
// polar_decomposition and singular_value_decomposition, kernels.cuh:486-499,
// helper_math.cuh:24-44,78-143, givens.cuh:117-154,190-197):
//   U = [[uc, us], [-us, uc]], V = [[vc, vs], [-vs, vc]], sigma_k = 1 + e_k,
//   sigma sorted descending, the sign (if any) on the smaller one.
// The polar rotation G = [[c,-s],[s,c]] gives S = G F; E = S - I is formed
// from H directly (c - 1 = -s^2/(1+c)), and the symmetric Jacobi rotation
// acts on E, whose eigenvectors are those of S.
template <class T> struct SvdH { T uc, us, vc, vs, e0, e1; };

template <class T, class J>
__device__ __forceinline__ void jacobi_sym(T E00, T E01, T E11, T &cs, T &sn, T &e0, T &e1)
{
    const J x = J(E00), y = J(E01), z = J(E11);
    const J y2 = y * y;
    if (y2 == J(0)) {
        cs = T(1); sn = T(0); e0 = E00; e1 = E11;
        return;
    }
    const J tau = J(0.5) * (x - z);
    const J w = tsqrt<J>(tau * tau + y2);
    const J t = (tau > J(0)) ? y / (tau + w) : y / (tau - w);
    const J c = J(1) / tsqrt<J>(t * t + J(1));
    const J s = -t * c;
    const J c2 = c * c, csy = J(2) * c * s * y, s2 = s * s;
    cs = T(c); sn = T(s);
    e0 = T(c2 * x - csy + s2 * z);
    e1 = T(s2 * x + csy + c2 * z);
}

template <class T> __device__ __forceinline__ SvdH<T> svd_h(const M2<T> &H)
{
    const T x0 = T(2) + H.a00 + H.a11;   // F00 + F11
    const T x1 = H.a10 - H.a01;          // F10 - F01
    const T den = tsqrt(x0 * x0 + x1 * x1);
    T c = T(1), s = T(0);
    if (den != T(0)) { c = x0 / den; s = -x1 / den; }
    const T cm1 = (c > T(0)) ? -(s * s) / (T(1) + c) : c - T(1);
    const T E00 = cm1 + c * H.a00 - s * H.a10;
    const T E01 = -s + c * H.a01 - s * H.a11;
    const T E11 = cm1 + s * H.a01 + c * H.a11;
    T cs, sn, e0, e1;
    // Near-degenerate singular values (gap below 1e-5): the Jacobi rotation is
    // evaluated in FP64 for the FP32 variants.
    if (sizeof(T) == 4 && fabs(double(E00) - double(E11)) + fabs(double(E01)) < 1e-5)
        jacobi_sym<T, double>(E00, E01, E11, cs, sn, e0, e1);
    else
        jacobi_sym<T, T>(E00, E01, E11, cs, sn, e0, e1);
    SvdH<T> r;
    if (e0 < e1) {
        const T tmp = e0; e0 = e1; e1 = tmp;
        r.vc = -sn; r.vs = cs;
    } else {
        r.vc = cs; r.vs = sn;
    }
    r.uc = c * r.vc - s * r.vs;
    r.us = s * r.vc + c * r.vs;
    r.e0 = e0; r.e1 = e1;
    return r;
}

// H of U diag(1+a, 1+b) V^T (a, b are sigma - 1), i.e. U diag(a,b) V^T + (U V^T - I).
template <class T> __device__ __forceinline__ M2<T> usvt_h(const SvdH<T> &s, T a, T b)
{
    const T rc = s.uc * s.vc + s.us * s.vs;       // U V^T = [[rc, rs], [-rs, rc]]
    const T rs = s.us * s.vc - s.uc * s.vs;
    const T rcm1 = (rc > T(0)) ? -(rs * rs) / (T(1) + rc) : rc - T(1);
    M2<T> H;
    H.a00 = s.uc * a * s.vc + s.us * b * s.vs + rcm1;
    H.a01 = -s.uc * a * s.vs + s.us * b * s.vc + rs;
    H.a10 = -s.us * a * s.vc + s.uc * b * s.vs - rs;
    H.a11 = s.us * a * s.vs + s.uc * b * s.vc + rcm1;
    return H;
}

// sqrt(1 + x) - 1 without cancellation
template <class T> __device__ __forceinline__ T sqrt1pm1(T x) { return x / (tsqrt(T(1) + x) + T(1)); }

struct Material {
    double mu, kappa, DP_threshold_p, pmin, pmax, qmax, pmin2, beta, M_sq, tan_phi, ridge_coeff_g_rho;
};

// The material constants in the arithmetic type of the kernels, with the
// combinations the yield tests use formed once on the host in FP64.
template <class T> struct MatT {
    T mu, kappa, thr, pmin, pmax, qmax, pmin2, tan_phi, ridge;
    T one_2beta;   // 1 + 2 beta
    T beta_pmax;   // beta pmax
    T M_sq;
    T cone_k;      // slope of the tension cone: -q0 / pmin2, q0 = 2 sqrt(-pmax pmin) qmax / (pmax - pmin)
    T fs_c;        // 2 qmax / (pmax - pmin) of the elliptic failure surface
};

template <class T> inline MatT<T> mat_of(const Material &m)
{
    MatT<T> r;
    r.mu = T(m.mu); r.kappa = T(m.kappa); r.thr = T(m.DP_threshold_p);
    r.pmin = T(m.pmin); r.pmax = T(m.pmax); r.qmax = T(m.qmax); r.pmin2 = T(m.pmin2);
    r.tan_phi = T(m.tan_phi); r.ridge = T(m.ridge_coeff_g_rho);
    r.one_2beta = T(1.0 + 2.0 * m.beta);
    r.beta_pmax = T(m.beta * m.pmax);
    r.M_sq = T(m.M_sq);
    const double q0 = 2.0 * std::sqrt(-m.pmax * m.pmin) * m.qmax / (m.pmax - m.pmin);
    r.cone_k = T(-q0 / m.pmin2);
    r.fs_c = T(2.0 * m.qmax / (m.pmax - m.pmin));
    return r;
}

// One-way latch of the crushed flag (CheckIfPointIsInsideFailureSurface with
// GetParametersForGrain, kernels.cuh:349-369,538-566).
template <class T>
__device__ __forceinline__ uint32_t failure_check(const MatT<T> &m, uint32_t util, T p, T q)
{
    if (p < T(0)) {
        if (p < m.pmin2) return util | kCrushed;
        const T q_limit = m.cone_k * (p - m.pmin2);
        if (q > q_limit) return util | kCrushed;
    } else {
        const T y = m.one_2beta * q * q + m.M_sq * (p + m.beta_pmax) * (p - m.pmax);
        if (y > T(0)) return util | kCrushed;
    }
    return util;
}

// Drucker-Prager / Wolper return map on H (Wolper_Drucker_Prager, kernels.cuh:374-483).
// The plastic volume ratio Jp_inv is updated in FP64.
template <class T>
__device__ __forceinline__ void wolper_dp(const MatT<T> &m, T thickness, T p_tr, T q_tr, const Kin<T> &k,
                                          const SvdH<T> &sv, M2<T> &H, T &Jp_inv)
{
    const T mu = m.mu, kappa = m.kappa;
    const T thr = m.thr;
    const T pmin = m.pmin, pmax = m.pmax;
    const T tan_phi = m.tan_phi;
    if (p_tr < thr) {
        if (Jp_inv < T(0.1)) {                       // case 0: Fe = sqrt(J) U V^T
            const T a = sqrt1pm1(k.Jm1);
            H = usvt_h(sv, a, a);
        } else {                                     // case 1: Fe = U V^T, Jp_inv /= J
            H = usvt_h(sv, T(0), T(0));
            Jp_inv = T(double(Jp_inv) / double(k.J));
        }
        return;
    }
    T q_yield;
    if (p_tr < pmax) {
        const T q_fs = m.fs_c * tsqrt((pmax - p_tr) * (p_tr - pmin));
        const T q_dp = fmax(T(0), (p_tr - thr) * tan_phi);
        q_yield = fmin(q_fs, q_dp);
    } else {
        q_yield = T(0);
    }
    if (!(q_tr > q_yield)) return;                   // case 2: elastic
    // case 3: project onto the yield surface
    const T p_ridge_max = m.ridge * thickness * Jp_inv;
    const T p_n_1 = fmin(p_tr, p_ridge_max);
    T q_n_1;
    if (p_n_1 < pmax) {
        const T q_dp = fmax(T(0), (p_n_1 - thr) * tan_phi);
        const T q_fs = m.fs_c * tsqrt((pmax - p_n_1) * (p_n_1 - pmin));
        q_n_1 = fmin(q_fs, q_dp);
    } else {
        q_n_1 = T(0);
    }
    const T Jnew_m1 = sqrt1pm1(T(-2) * p_n_1 / kappa);
    const T s_hat_norm = q_n_1 * T(0.7071067811865475);
    // v_s_hat_tr = mu/J dev_d(sigma^2) is (dd, -dd) with dd ~ (e0-e1)(2+e0+e1);
    // its normalisation is +-(1,-1)/sqrt(2), or 0 when dd == 0.
    const T dd = (sv.e0 - sv.e1) * (T(2) + sv.e0 + sv.e1);
    T n0 = T(0);
    if (dd > T(0)) n0 = T(0.7071067811865475);
    else if (dd < T(0)) n0 = T(-0.7071067811865475);
    const T f = s_hat_norm * ((T(1) + k.Jm1) / mu);
    const T b0m1 = f * n0 + Jnew_m1;
    const T b1m1 = -f * n0 + Jnew_m1;
    H = usvt_h(sv, sqrt1pm1(b0m1), sqrt1pm1(b1m1));
    Jp_inv = T(double(Jp_inv) * ((1.0 + double(Jnew_m1)) / (1.0 + double(k.Jm1))));
}

}  // namespace icempm
