// surrogate.cu -- the learned return map (an MLP in place of the Drucker-Prager projection).
//
// An MLP 4 -> 64 -> 64 -> 3 with SiLU stands in for the projection of a
// trial state onto the Drucker-Prager yield surface (case 3 of wolper_dp,
// kernels.cuh:411-467).  A trial state is (sigma1, sigma2, Jp_inv, thickness)
// -- the singular values of Fe after the G2P update, the plastic volume ratio
// and the thickness; the rotations U, V of the SVD are kept as they are.
//   inputs   x = (log sigma1, log sigma2, log Jp_inv, log thickness)
//   outputs  y = (log sigma1' - log sigma1, log sigma2' - log sigma2,
//                 log Jp_inv' - log Jp_inv)
// both standardised with per-feature mean and standard deviation
// (norm[14] = x mean[4], x std[4], y mean[3], y std[3]).  The thickness takes
// the input slot of the friction angle, which is one constant per material
// (one network per material) while the projection depends on the thickness
// through the ridging pressure bound.
//
// Parameters (FP32 master copy, row-major W[out][in]): W1[64][4] b1[64]
// W2[64][64] b2[64] W3[3][64] b3[3], 4675 floats.
//
//   k_mlp_grad      one sample per thread: forward, loss, backward; the
//                   block's 128 samples are reduced into the parameter
//                   gradient in shared memory, one atomic per parameter
//   k_mlp_adam      Adam update of the master parameters
//   k_mlp_forward   FP32 forward (evaluation, gradient checks)
//   k_return_map_exact<Real>   the exact map on a batch of trial states
//   k_return_map_learned       BF16 tensor-core inference (mma.sync
//                   m16n8k16, FP32 accumulate, 32 samples per warp); trial
//                   states of cases 0-2 take the exact closed forms, case 3
//                   takes the network, whose answer is kept only if it lies
//                   on the yield surface within the tolerance, else the
//                   exact map answers (fallback).
#include <cstdint>
#include <string>

#include <cuda_bf16.h>

#include "engine.cuh"
#include "engine_iface.h"
#include "mlp_device.cuh"

namespace icempm {
namespace mlp {

constexpr int BLK = 128, LD = HID + 1;

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

struct GradSmem {
    float P[NPARAM];
    float H1[BLK][LD], H2[BLK][LD], D1[BLK][LD], D2[BLK][LD];
    float X[BLK][IN], DY[BLK][OUT];
    float red[BLK / 32];
};

// Mean over the n samples of sum_o (y_o - t_o)^2; G += its gradient over
// this block's samples, *loss += this block's share of it.
__global__ void __launch_bounds__(BLK) k_mlp_grad(const float *__restrict__ P, const float *__restrict__ X,
                                                  const float *__restrict__ Y, int n, float inv_n, float *G,
                                                  float *loss)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    GradSmem &sm = *reinterpret_cast<GradSmem *>(smraw);
    const int tid = threadIdx.x;
    for (int k = tid; k < NPARAM; k += BLK) sm.P[k] = P[k];
    __syncthreads();
    const long long s = (long long)blockIdx.x * BLK + tid;
    const bool valid = s < n;
    float x[IN];
#pragma unroll
    for (int i = 0; i < IN; i++) x[i] = valid ? X[s * IN + i] : 0.0f;
    for (int j = 0; j < HID; j++) {
        float z = sm.P[B1 + j];
#pragma unroll
        for (int i = 0; i < IN; i++) z += sm.P[W1 + j * IN + i] * x[i];
        const float g = sigm(z);
        sm.H1[tid][j] = z * g;
        sm.D1[tid][j] = g * (1.0f + z * (1.0f - g));   // SiLU'(z)
    }
    for (int j = 0; j < HID; j++) {
        float z = sm.P[B2 + j];
        for (int k = 0; k < HID; k++) z += sm.P[W2 + j * HID + k] * sm.H1[tid][k];
        const float g = sigm(z);
        sm.H2[tid][j] = z * g;
        sm.D2[tid][j] = g * (1.0f + z * (1.0f - g));
    }
    float dy[OUT], lsum = 0.0f;
#pragma unroll
    for (int o = 0; o < OUT; o++) {
        float y = sm.P[B3 + o];
        for (int j = 0; j < HID; j++) y += sm.P[W3 + o * HID + j] * sm.H2[tid][j];
        const float d = valid ? y - Y[s * OUT + o] : 0.0f;
        lsum += d * d;
        dy[o] = 2.0f * d * inv_n;
        sm.DY[tid][o] = dy[o];
    }
    for (int j = 0; j < HID; j++) {   // dL/dz2
        float g = 0.0f;
#pragma unroll
        for (int o = 0; o < OUT; o++) g += sm.P[W3 + o * HID + j] * dy[o];
        sm.D2[tid][j] *= g;
    }
    for (int k = 0; k < HID; k++) {   // dL/dz1
        float g = 0.0f;
        for (int j = 0; j < HID; j++) g += sm.P[W2 + j * HID + k] * sm.D2[tid][j];
        sm.D1[tid][k] *= g;
    }
#pragma unroll
    for (int i = 0; i < IN; i++) sm.X[tid][i] = x[i];
    __syncthreads();
    for (int e = tid; e < NPARAM; e += BLK) {
        float acc = 0.0f;
        if (e < B1) {
            const int j = e / IN, i = e - j * IN;
            for (int t = 0; t < BLK; t++) acc += sm.D1[t][j] * sm.X[t][i];
        } else if (e < W2) {
            for (int t = 0; t < BLK; t++) acc += sm.D1[t][e - B1];
        } else if (e < B2) {
            const int j = (e - W2) / HID, k = (e - W2) - j * HID;
            for (int t = 0; t < BLK; t++) acc += sm.D2[t][j] * sm.H1[t][k];
        } else if (e < W3) {
            for (int t = 0; t < BLK; t++) acc += sm.D2[t][e - B2];
        } else if (e < B3) {
            const int o = (e - W3) / HID, j = (e - W3) - o * HID;
            for (int t = 0; t < BLK; t++) acc += sm.DY[t][o] * sm.H2[t][j];
        } else {
            for (int t = 0; t < BLK; t++) acc += sm.DY[t][e - B3];
        }
        atomicAdd(&G[e], acc);
    }
    float l = lsum;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) l += __shfl_down_sync(0xffffffffu, l, off);
    if ((tid & 31) == 0) sm.red[tid >> 5] = l;
    __syncthreads();
    if (tid == 0) {
        float b = 0.0f;
        for (int w2 = 0; w2 < BLK / 32; w2++) b += sm.red[w2];
        atomicAdd(loss, b * inv_n);
    }
}

__global__ void k_mlp_adam(float *P, const float *__restrict__ G, float *M, float *V, float lr, float b1, float b2,
                           float eps, float c1, float c2)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NPARAM) return;
    const float g = G[e];
    const float m = b1 * M[e] + (1.0f - b1) * g;
    const float v = b2 * V[e] + (1.0f - b2) * g * g;
    M[e] = m;
    V[e] = v;
    P[e] -= lr * (m * c1) / (sqrtf(v * c2) + eps);
}

__global__ void __launch_bounds__(128) k_mlp_forward(const float *__restrict__ P, const float *__restrict__ X, int n,
                                                     float *Y)
{
    __shared__ float sp[NPARAM];
    for (int k = threadIdx.x; k < NPARAM; k += blockDim.x) sp[k] = P[k];
    __syncthreads();
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    float x[IN], h1[HID];
#pragma unroll
    for (int i = 0; i < IN; i++) x[i] = X[s * IN + i];
#pragma unroll 4
    for (int j = 0; j < HID; j++) {
        float z = sp[B1 + j];
#pragma unroll
        for (int i = 0; i < IN; i++) z += sp[W1 + j * IN + i] * x[i];
        h1[j] = z * sigm(z);
    }
    float y[OUT];
#pragma unroll
    for (int o = 0; o < OUT; o++) y[o] = sp[B3 + o];
    for (int j = 0; j < HID; j++) {
        float z = sp[B2 + j];
#pragma unroll 8
        for (int k = 0; k < HID; k++) z += sp[W2 + j * HID + k] * h1[k];
        const float h = z * sigm(z);
#pragma unroll
        for (int o = 0; o < OUT; o++) y[o] += sp[W3 + o * HID + j] * h;
    }
#pragma unroll
    for (int o = 0; o < OUT; o++) Y[s * OUT + o] = y[o];
}

// Case of the return map for a trial state (wolper_dp's branches): 0/1
// tension, 2 elastic, 3 projection onto the yield surface.
template <class T>
__device__ __forceinline__ int return_map_case(const MatT<T> &m, T p, T q, T jp)
{
    if (p < m.thr) return jp < T(0.1) ? 0 : 1;
    T q_yield = T(0);
    if (p < m.pmax) q_yield = fmin(m.fs_c * tsqrt((m.pmax - p) * (p - m.pmin)), fmax(T(0), (p - m.thr) * m.tan_phi));
    return q > q_yield ? 3 : 2;
}

// The exact map on singular values: U = V = I, so H stays diagonal and the
// projected singular values are 1 + H00, 1 + H11.
template <class T>
__device__ __forceinline__ void exact_map(const MatT<T> &m, T s1, T s2, T jp, T thick, T &o1, T &o2, T &ojp)
{
    M2<T> H = {s1 - T(1), T(0), T(0), s2 - T(1)};
    const Kin<T> k = kinematics(H);
    T p, q;
    pq(k, m.mu, m.kappa, p, q);
    SvdH<T> sv;
    sv.uc = T(1); sv.us = T(0); sv.vc = T(1); sv.vs = T(0);
    sv.e0 = s1 - T(1); sv.e1 = s2 - T(1);
    wolper_dp(m, thick, p, q, k, sv, H, jp);
    o1 = T(1) + H.a00;
    o2 = T(1) + H.a11;
    ojp = jp;
}

template <class T>
__global__ void k_return_map_exact(MatT<T> m, const float4 *__restrict__ trial, int n, float4 *out)
{
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const float4 t = trial[s];
    T o1, o2, ojp;
    exact_map<T>(m, T(t.x), T(t.y), T(t.z), T(t.w), o1, o2, ojp);
    out[s] = make_float4(float(o1), float(o2), float(ojp), 0.0f);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ float silu(float z) { return z * sigm(z); }

constexpr int IWARPS = 8;

struct InferSmem {
    __nv_bfloat16 w1[HID][16];      // K padded 4 -> 16
    __nv_bfloat16 w2[HID][HID];
    __nv_bfloat16 w3[8][HID];       // N padded 3 -> 8
    float b1[HID], b2[HID], b3[8];
    float norm[14];
    float x[IWARPS][32][IN];
    float y[IWARPS][32][4];
};

// Learned map on a batch; out[s] = {sigma1', sigma2', Jp_inv', how} with how
// 0 = exact closed form (cases 0-2), 1 = network accepted, 2 = exact after the
// network's answer left the yield surface by more than `tol` (relative).
__global__ void __launch_bounds__(IWARPS * 32) k_return_map_learned(MatT<float> m, const float *__restrict__ P,
                                                                   const float *__restrict__ norm,
                                                                   const float4 *__restrict__ trial, int n,
                                                                   float tol, float4 *out, unsigned *fallbacks)
{
    __shared__ InferSmem sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int e = tid; e < HID * 16; e += blockDim.x) {
        const int j = e / 16, i = e % 16;
        sm.w1[j][i] = __float2bfloat16(i < IN ? P[W1 + j * IN + i] : 0.0f);
    }
    for (int e = tid; e < HID * HID; e += blockDim.x) sm.w2[e / HID][e % HID] = __float2bfloat16(P[W2 + e]);
    for (int e = tid; e < 8 * HID; e += blockDim.x) {
        const int o = e / HID, j = e % HID;
        sm.w3[o][j] = __float2bfloat16(o < OUT ? P[W3 + o * HID + j] : 0.0f);
    }
    for (int e = tid; e < HID; e += blockDim.x) { sm.b1[e] = P[B1 + e]; sm.b2[e] = P[B2 + e]; }
    if (tid < 8) sm.b3[tid] = tid < OUT ? P[B3 + tid] : 0.0f;
    if (tid < 14) sm.norm[tid] = norm[tid];
    __syncthreads();

    const int g = lane >> 2, tg = lane & 3;
    const long long nwarps = (long long)gridDim.x * IWARPS;
    for (long long base = ((long long)blockIdx.x * IWARPS + wid) * 32; base < n; base += nwarps * 32) {
        const long long s = base + lane;
        const bool valid = s < n;
        float4 t = valid ? trial[s] : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
        // exact classification; only projections go to the network
        const float J = t.x * t.y;
        const float p = -(m.kappa * 0.5f) * (J * J - 1.0f);
        const float q = 2.0f * m.mu * fabsf(0.5f * (t.x * t.x - t.y * t.y)) / J;
        const int cs = return_map_case<float>(m, p, q, t.z);
        const bool use_net = valid && cs == 3 && t.x > 0.0f && t.y > 0.0f && t.z > 0.0f && t.w > 0.0f;
        float xv[IN] = {logf(fmaxf(t.x, 1e-30f)), logf(fmaxf(t.y, 1e-30f)), logf(fmaxf(t.z, 1e-30f)),
                        logf(fmaxf(t.w, 1e-30f))};
#pragma unroll
        for (int i = 0; i < IN; i++) sm.x[wid][lane][i] = (xv[i] - sm.norm[i]) / fmaxf(sm.norm[4 + i], 1e-30f);
        __syncwarp();
        if (__any_sync(0xffffffffu, use_net)) {
            // layer 1: [32 x 16] x [16 x 64]
            uint32_t a[2][4][4];     // A fragments of the next layer (k-tiles of 16)
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                uint32_t ax[4];
                const int r0 = mt * 16 + g, r1 = r0 + 8;
                ax[0] = tg < 2 ? pack_bf16(sm.x[wid][r0][2 * tg], sm.x[wid][r0][2 * tg + 1]) : 0u;
                ax[1] = tg < 2 ? pack_bf16(sm.x[wid][r1][2 * tg], sm.x[wid][r1][2 * tg + 1]) : 0u;
                ax[2] = 0u;
                ax[3] = 0u;
                float c[8][4];
#pragma unroll
                for (int nt = 0; nt < 8; nt++) {
                    const int col = nt * 8 + 2 * tg;
                    c[nt][0] = sm.b1[col]; c[nt][1] = sm.b1[col + 1];
                    c[nt][2] = sm.b1[col]; c[nt][3] = sm.b1[col + 1];
                    const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&sm.w1[nt * 8 + g][2 * tg]);
                    const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&sm.w1[nt * 8 + g][2 * tg + 8]);
                    mma_bf16(c[nt], ax, b0, b1);
                }
#pragma unroll
                for (int kt = 0; kt < 4; kt++) {
                    a[mt][kt][0] = pack_bf16(silu(c[2 * kt][0]), silu(c[2 * kt][1]));
                    a[mt][kt][1] = pack_bf16(silu(c[2 * kt][2]), silu(c[2 * kt][3]));
                    a[mt][kt][2] = pack_bf16(silu(c[2 * kt + 1][0]), silu(c[2 * kt + 1][1]));
                    a[mt][kt][3] = pack_bf16(silu(c[2 * kt + 1][2]), silu(c[2 * kt + 1][3]));
                }
            }
            // layer 2: [32 x 64] x [64 x 64], then layer 3: [32 x 64] x [64 x 8]
#pragma unroll
            for (int mt = 0; mt < 2; mt++) {
                float c[8][4];
#pragma unroll
                for (int nt = 0; nt < 8; nt++) {
                    const int col = nt * 8 + 2 * tg;
                    c[nt][0] = sm.b2[col]; c[nt][1] = sm.b2[col + 1];
                    c[nt][2] = sm.b2[col]; c[nt][3] = sm.b2[col + 1];
#pragma unroll
                    for (int kt = 0; kt < 4; kt++) {
                        const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&sm.w2[nt * 8 + g][kt * 16 + 2 * tg]);
                        const uint32_t b1 =
                            *reinterpret_cast<const uint32_t *>(&sm.w2[nt * 8 + g][kt * 16 + 2 * tg + 8]);
                        mma_bf16(c[nt], a[mt][kt], b0, b1);
                    }
                }
                float d[4] = {sm.b3[2 * tg], sm.b3[2 * tg + 1], sm.b3[2 * tg], sm.b3[2 * tg + 1]};
#pragma unroll
                for (int kt = 0; kt < 4; kt++) {
                    uint32_t a2[4];
                    a2[0] = pack_bf16(silu(c[2 * kt][0]), silu(c[2 * kt][1]));
                    a2[1] = pack_bf16(silu(c[2 * kt][2]), silu(c[2 * kt][3]));
                    a2[2] = pack_bf16(silu(c[2 * kt + 1][0]), silu(c[2 * kt + 1][1]));
                    a2[3] = pack_bf16(silu(c[2 * kt + 1][2]), silu(c[2 * kt + 1][3]));
                    const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&sm.w3[g][kt * 16 + 2 * tg]);
                    const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&sm.w3[g][kt * 16 + 2 * tg + 8]);
                    mma_bf16(d, a2, b0, b1);
                }
                if (tg < 2) {   // columns 0..3 of rows g and g+8 of this m-tile
                    sm.y[wid][mt * 16 + g][2 * tg] = d[0];
                    sm.y[wid][mt * 16 + g][2 * tg + 1] = d[1];
                    sm.y[wid][mt * 16 + g + 8][2 * tg] = d[2];
                    sm.y[wid][mt * 16 + g + 8][2 * tg + 1] = d[3];
                }
            }
        }
        __syncwarp();
        float o1 = t.x, o2 = t.y, ojp = t.z, how = 0.0f;
        bool fb = false;
        if (use_net) {
            float yv[OUT];
#pragma unroll
            for (int o = 0; o < OUT; o++) yv[o] = sm.y[wid][lane][o] * sm.norm[11 + o] + sm.norm[8 + o];
            o1 = t.x * expf(yv[0]);
            o2 = t.y * expf(yv[1]);
            ojp = t.z * expf(yv[2]);
            // on the yield surface?  q' against q_yield(p') of the predicted state
            const float J1 = o1 * o2;
            const float p1 = -(m.kappa * 0.5f) * (J1 * J1 - 1.0f);
            const float q1 = 2.0f * m.mu * fabsf(0.5f * (o1 * o1 - o2 * o2)) / J1;
            float qy = 0.0f;
            if (p1 < m.pmax) qy = fminf(m.fs_c * sqrtf(fmaxf((m.pmax - p1) * (p1 - m.pmin), 0.0f)),
                                        fmaxf(0.0f, (p1 - m.thr) * m.tan_phi));
            const float res = fabsf(q1 - qy) / fmaxf(qy, 1.0f);
            fb = !(res <= tol);
            how = fb ? 2.0f : 1.0f;
        }
        if (valid && (cs != 3 || fb || !use_net)) exact_map<float>(m, t.x, t.y, t.z, t.w, o1, o2, ojp);
        if (valid) out[s] = make_float4(o1, o2, ojp, how);
        const unsigned nf = __popc(__ballot_sync(0xffffffffu, valid && fb));
        if (lane == 0 && nf) atomicAdd(fallbacks, nf);
        __syncwarp();
    }
}

// FP32 master parameters and normalisation -> the packed network
// (mlp_device.cuh), one thread per word.
__global__ void k_mlp_pack(const float *__restrict__ P, const float *__restrict__ norm, Packed *out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < HID * 8) {                       // w1: k 2c, 2c+1 of row n (k >= IN is padding)
        const int n = e / 8, c = e % 8, k = 2 * c;
        out->w1[n][c] = pack_bf16x2(k < IN ? P[W1 + n * IN + k] : 0.0f, k + 1 < IN ? P[W1 + n * IN + k + 1] : 0.0f);
    }
    if (e < HID * HID / 2) {
        const int n = e / (HID / 2), c = e % (HID / 2);
        out->w2[n][c] = pack_bf16x2(P[W2 + n * HID + 2 * c], P[W2 + n * HID + 2 * c + 1]);
    }
    if (e < 8 * HID / 2) {                   // w3: rows n >= OUT are padding
        const int n = e / (HID / 2), c = e % (HID / 2);
        out->w3[n][c] = n < OUT ? pack_bf16x2(P[W3 + n * HID + 2 * c], P[W3 + n * HID + 2 * c + 1]) : 0u;
    }
    if (e < HID) { out->b1[e] = P[B1 + e]; out->b2[e] = P[B2 + e]; }
    if (e < 8) out->b3[e] = e < OUT ? P[B3 + e] : 0.0f;
    if (e < 16) out->norm[e] = e < 14 ? norm[e] : 0.0f;
}

}  // namespace mlp

int mlp_pack(const float *d_params, const float *d_norm, void *d_packed, cudaStream_t stream)
{
    mlp::k_mlp_pack<<<(mlp::HID * mlp::HID / 2 + 255) / 256, 256, 0, stream>>>(d_params, d_norm,
                                                                             (mlp::Packed *)d_packed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string("k_mlp_pack: ") + cudaGetErrorString(e));
    return ICEMPM_OK;
}

size_t mlp_packed_bytes() { return sizeof(mlp::Packed); }

}  // namespace icempm

using icempm::fail;

#define ICEMPM_CK(call, what)                                                                              \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

int icempm_mlp_param_count(void) { return icempm::mlp::NPARAM; }

int icempm_mlp_grad(const float *d_params, const float *d_x, const float *d_y, uint32_t n, float *d_grad,
                    float *d_loss, void *stream)
{
    using namespace icempm::mlp;
    if (!d_params || !d_x || !d_y || !d_grad || !d_loss) return fail(ICEMPM_E_ARG, "null device pointer");
    if (n == 0 || n > (1u << 30)) return fail(ICEMPM_E_ARG, "n must be in 1 .. 2^30");
    ICEMPM_CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(GradSmem)),
              "k_mlp_grad shared memory");
    const unsigned nb = (n + BLK - 1) / BLK;
    k_mlp_grad<<<nb, BLK, sizeof(GradSmem), (cudaStream_t)stream>>>(d_params, d_x, d_y, (int)n, 1.0f / (float)n,
                                                                    d_grad, d_loss);
    ICEMPM_CK(cudaGetLastError(), "k_mlp_grad");
    return ICEMPM_OK;
}

int icempm_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int32_t t, float lr, void *stream)
{
    using namespace icempm::mlp;
    if (!d_params || !d_grad || !d_m || !d_v || t < 1) return fail(ICEMPM_E_ARG, "bad arguments");
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - std::pow(b1, (float)t)), c2 = 1.0f / (1.0f - std::pow(b2, (float)t));
    k_mlp_adam<<<(NPARAM + 255) / 256, 256, 0, (cudaStream_t)stream>>>(d_params, d_grad, d_m, d_v, lr, b1, b2, 1e-8f,
                                                                        c1, c2);
    ICEMPM_CK(cudaGetLastError(), "k_mlp_adam");
    return ICEMPM_OK;
}

int icempm_mlp_forward(const float *d_params, const float *d_x, uint32_t n, float *d_y, void *stream)
{
    using namespace icempm::mlp;
    if (!d_params || !d_x || !d_y) return fail(ICEMPM_E_ARG, "null device pointer");
    if (n == 0) return ICEMPM_OK;
    k_mlp_forward<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(d_params, d_x, (int)n, d_y);
    ICEMPM_CK(cudaGetLastError(), "k_mlp_forward");
    return ICEMPM_OK;
}

int icempm_return_map_exact(const icempm_simparams_t *prms, const float *d_trial, uint32_t n, float *d_out,
                            int32_t fp64, void *stream)
{
    using namespace icempm;
    if (!prms || !d_trial || !d_out) return fail(ICEMPM_E_ARG, "null argument");
    if (n == 0) return ICEMPM_OK;
    const Material m = material_of(*prms);
    const unsigned nb = (n + 255) / 256;
    if (fp64)
        mlp::k_return_map_exact<double><<<nb, 256, 0, (cudaStream_t)stream>>>(
            mat_of<double>(m), (const float4 *)d_trial, (int)n, (float4 *)d_out);
    else
        mlp::k_return_map_exact<float><<<nb, 256, 0, (cudaStream_t)stream>>>(
            mat_of<float>(m), (const float4 *)d_trial, (int)n, (float4 *)d_out);
    ICEMPM_CK(cudaGetLastError(), "k_return_map_exact");
    return ICEMPM_OK;
}

int icempm_return_map_learned(const icempm_simparams_t *prms, const float *d_params, const float *d_norm,
                              const float *d_trial, uint32_t n, float tol, float *d_out, uint32_t *d_fallbacks,
                              void *stream)
{
    using namespace icempm;
    if (!prms || !d_params || !d_norm || !d_trial || !d_out || !d_fallbacks) return fail(ICEMPM_E_ARG, "null argument");
    if (n == 0) return ICEMPM_OK;
    int dev = 0, sms = 0;
    ICEMPM_CK(cudaGetDevice(&dev), "cudaGetDevice");
    ICEMPM_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    const long long groups = ((long long)n + 31) / 32;
    const unsigned nb = (unsigned)std::min<long long>((groups + mlp::IWARPS - 1) / mlp::IWARPS, (long long)sms * 8);
    mlp::k_return_map_learned<<<nb, mlp::IWARPS * 32, 0, (cudaStream_t)stream>>>(
        mat_of<float>(material_of(*prms)), d_params, d_norm, (const float4 *)d_trial, (int)n, tol, (float4 *)d_out,
        d_fallbacks);
    ICEMPM_CK(cudaGetLastError(), "k_return_map_learned");
    return ICEMPM_OK;
}

}  // extern "C"
