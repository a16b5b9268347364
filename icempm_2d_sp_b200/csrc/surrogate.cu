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
//                   m16n8k16, FP32 accumulate, 32 samples per warp, the
//                   fused kernel's network code, mlp_device.cuh); trial
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

constexpr int IWARPS = 8;

// Learned map on a batch; out[s] = {sigma1', sigma2', Jp_inv', how} with how
// 0 = exact closed form (cases 0-2), 1 = network accepted, 2 = exact after the
// network's answer left the yield surface by more than `tol` (relative).  The
// network runs warp by warp on 32 trial states at a time (mlp::rows_forward,
// the same code the fused kernel runs), the CTA's copy of it packed into
// shared memory from the FP32 parameters at the start.
__global__ void __launch_bounds__(IWARPS * 32, 2) k_return_map_learned(MatT<float> m, const float *__restrict__ P,
                                                                   const float *__restrict__ norm,
                                                                   const float4 *__restrict__ trial, int n,
                                                                   float tol, float4 *out, unsigned *fallbacks)
{
    __shared__ Smem<IWARPS> sm;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int e = tid; e < PACK_ENTRIES; e += blockDim.x) pack_entry(e, P, norm, sm.p);
    __syncthreads();
    const float *nm = sm.p.norm;
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
        float xin[IN] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (use_net) {
            xin[0] = (logf(t.x) - nm[0]) / nm[4];
            xin[1] = (logf(t.y) - nm[1]) / nm[5];
            xin[2] = (logf(t.z) - nm[2]) / nm[6];
            xin[3] = (logf(t.w) - nm[3]) / nm[7];
        }
        float yo[OUT] = {0.0f, 0.0f, 0.0f};
        if (__any_sync(0xffffffffu, use_net)) rows_forward(sm.p, sm.io[wid], lane, xin, yo);
        float o1 = t.x, o2 = t.y, ojp = t.z, how = 0.0f;
        bool fb = false;
        if (use_net) {
            float yv[OUT];
#pragma unroll
            for (int o = 0; o < OUT; o++) yv[o] = yo[o] * nm[11 + o] + nm[8 + o];
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
// (mlp_device.cuh), one thread per entry.
__global__ void k_mlp_pack(const float *__restrict__ P, const float *__restrict__ norm, Packed *out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < PACK_ENTRIES) pack_entry(e, P, norm, *out);
}

}  // namespace mlp

int mlp_pack(const float *d_params, const float *d_norm, void *d_packed, cudaStream_t stream)
{
    mlp::k_mlp_pack<<<(mlp::PACK_ENTRIES + 255) / 256, 256, 0, stream>>>(d_params, d_norm, (mlp::Packed *)d_packed);
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
