// mlp_device.cuh -- the learned return map's network inside other kernels.
//
// The MLP 4 -> 64 -> 64 -> 3 with SiLU (parameters: see surrogate.cu) is
// evaluated by one warp on the 32 rows its lanes hold, with BF16 tensor-core
// MMAs (mma.sync m16n8k16, FP32 accumulate): rows 0-15 and 16-31 are two
// m-tiles, the 64 hidden features eight n-tiles, and each layer's FP32
// outputs become, after the activation, the BF16 A fragments of the next
// layer in registers.  The weights sit in shared memory as B fragments: for
// output row n and the k-tile of 16 inputs, lane (g, tg) = (lane / 4, lane % 4)
// needs the BF16 pairs of inputs (2tg, 2tg+1) and (2tg+8, 2tg+9), which are
// stored side by side as one 8-byte entry (one shared load per MMA operand).
// The 16 entries of a row of W2 and W3 are swizzled, entry c at
// c ^ 4 (n mod 4), so that the eight rows g a warp reads in one load fall on
// different banks.  Packed once per network by k_mlp_pack.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace icempm {
namespace mlp {

constexpr int IN = 4, HID = 64, OUT = 3;
// FP32 master parameters, row-major W[out][in]
constexpr int W1 = 0, B1 = W1 + HID * IN, W2 = B1 + HID, B2 = W2 + HID * HID, W3 = B2 + HID, B3 = W3 + OUT * HID;
constexpr int NPARAM = B3 + OUT;   // 4675

// The packed network: what a CTA copies into shared memory.
struct alignas(16) Packed {
    uint2 w1[HID][4];         // W1 fragments, K padded 4 -> 16 (one k-tile)
    uint2 w2[HID][16];        // W2 fragments: 4 k-tiles x 4 lanes, swizzled
    uint2 w3[8][16];          // W3 fragments, N padded 3 -> 8, swizzled
    float b1[HID], b2[HID], b3[8];
    float norm[16];           // x mean[4], x std[4], y mean[3], y std[3], 2 unused
};
static_assert(sizeof(Packed) % 16 == 0, "16-byte copies");

// Shared memory of the in-kernel network: the packed weights and one row
// exchange area (32 rows x 4 floats) per warp.
template <int NWARPS> struct Smem {
    Packed p;
    float io[NWARPS][32][4];
};

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Position of fragment entry c (k-tile c / 4, lane tg = c % 4) in row n.
__host__ __device__ __forceinline__ int frag_slot(int n, int c) { return c ^ ((n & 3) << 2); }

// One entry e of the packing of FP32 master parameters P and the
// normalisation into a Packed network (entries 0 .. PACK_ENTRIES-1; every
// word of the result is written by exactly one entry).
constexpr int PACK_ENTRIES = HID * 16;
__device__ __forceinline__ void pack_entry(int e, const float *__restrict__ P, const float *__restrict__ norm,
                                           Packed &out)
{
    if (e < HID * 4) {                       // w1: inputs 2tg, 2tg+1 (and 2tg+8.. = padding) of row n
        const int n = e / 4, k = 2 * (e % 4);
        out.w1[n][e % 4] = make_uint2(pack_bf16x2(k < IN ? P[W1 + n * IN + k] : 0.0f,
                                                  k + 1 < IN ? P[W1 + n * IN + k + 1] : 0.0f), 0u);
    }
    {                                        // w2: row n, k-tile kt, lane tg
        const int n = e / 16, c = e % 16, k = 16 * (c / 4) + 2 * (c % 4);
        const float *w = P + W2 + n * HID;
        out.w2[n][frag_slot(n, c)] = make_uint2(pack_bf16x2(w[k], w[k + 1]), pack_bf16x2(w[k + 8], w[k + 9]));
    }
    if (e < 8 * 16) {                        // w3: rows n >= OUT are padding
        const int n = e / 16, c = e % 16, k = 16 * (c / 4) + 2 * (c % 4);
        const float *w = P + W3 + n * HID;
        out.w3[n][frag_slot(n, c)] = n < OUT ? make_uint2(pack_bf16x2(w[k], w[k + 1]), pack_bf16x2(w[k + 8], w[k + 9]))
                                             : make_uint2(0u, 0u);
    }
    if (e < HID) { out.b1[e] = P[B1 + e]; out.b2[e] = P[B2 + e]; }
    if (e < 8) out.b3[e] = e < OUT ? P[B3 + e] : 0.0f;
    if (e < 16) out.norm[e] = e < 14 ? norm[e] : 0.0f;
}

// SiLU z / (1 + exp(-z)) of two accumulator values with the fast exponential
// and division intrinsics (a few ulp; the network is trained with the exact
// form, and the hardware tanh approximation's ~2^-11 error measurably raised
// the fallback rate), packed to a BF16 pair, the next layer's A-fragment word.
__device__ __forceinline__ uint32_t silu_pack(float z0, float z1)
{
    return pack_bf16x2(__fdividef(z0, 1.0f + __expf(-z0)), __fdividef(z1, 1.0f + __expf(-z1)));
}

// Copies the packed network into shared memory (all threads of the CTA; a
// barrier must follow before use).
__device__ __forceinline__ void load_packed(Packed &dst, const Packed *src, int tid, int nthreads)
{
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(&dst);
    for (int k = tid; k < (int)(sizeof(Packed) / 16); k += nthreads) d[k] = s[k];
}

// The network on the warp's 32 rows: lane l supplies its standardised input
// row x (4 values) and receives its standardised output row y (3 values).
// All 32 lanes of the warp must call it together; io is the warp's exchange
// area.
__device__ __forceinline__ void rows_forward(const Packed &P, float (*io)[4], int lane, const float x[4], float y[3])
{
    const int g = lane >> 2, tg = lane & 3;
    io[lane][0] = x[0]; io[lane][1] = x[1]; io[lane][2] = x[2]; io[lane][3] = x[3];
    __syncwarp();
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        uint32_t ax[4];
        ax[0] = tg < 2 ? pack_bf16x2(io[r0][2 * tg], io[r0][2 * tg + 1]) : 0u;
        ax[1] = tg < 2 ? pack_bf16x2(io[r1][2 * tg], io[r1][2 * tg + 1]) : 0u;
        ax[2] = 0u;
        ax[3] = 0u;
        // layer 1: [16 x 16] x [16 x 64] -> SiLU -> A fragments of layer 2
        uint32_t a[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            float c0[4], c1[4];
            const int n0 = (2 * kt) * 8, n1 = n0 + 8;
            c0[0] = P.b1[n0 + 2 * tg]; c0[1] = P.b1[n0 + 2 * tg + 1]; c0[2] = c0[0]; c0[3] = c0[1];
            c1[0] = P.b1[n1 + 2 * tg]; c1[1] = P.b1[n1 + 2 * tg + 1]; c1[2] = c1[0]; c1[3] = c1[1];
            const uint2 b0 = P.w1[n0 + g][tg], b1 = P.w1[n1 + g][tg];
            mma_bf16_16816(c0, ax, b0.x, b0.y);
            mma_bf16_16816(c1, ax, b1.x, b1.y);
            a[kt][0] = silu_pack(c0[0], c0[1]);
            a[kt][1] = silu_pack(c0[2], c0[3]);
            a[kt][2] = silu_pack(c1[0], c1[1]);
            a[kt][3] = silu_pack(c1[2], c1[3]);
        }
        // layer 2: [16 x 64] x [64 x 64] -> SiLU, two n-tiles at a time into
        // the A fragment of layer 3 ([16 x 64] x [64 x 8])
        float d[4] = {P.b3[2 * tg], P.b3[2 * tg + 1], P.b3[2 * tg], P.b3[2 * tg + 1]};
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            float c0[4], c1[4];
            const int n0 = (2 * kt) * 8, n1 = n0 + 8;
            c0[0] = P.b2[n0 + 2 * tg]; c0[1] = P.b2[n0 + 2 * tg + 1]; c0[2] = c0[0]; c0[3] = c0[1];
            c1[0] = P.b2[n1 + 2 * tg]; c1[1] = P.b2[n1 + 2 * tg + 1]; c1[2] = c1[0]; c1[3] = c1[1];
#pragma unroll
            for (int k2 = 0; k2 < 4; k2++) {
                const int slot = frag_slot(g, 4 * k2 + tg);   // rows n0 + g, n1 + g: n0, n1 multiples of 8
                const uint2 b0 = P.w2[n0 + g][slot], b1 = P.w2[n1 + g][slot];
                mma_bf16_16816(c0, a[k2], b0.x, b0.y);
                mma_bf16_16816(c1, a[k2], b1.x, b1.y);
            }
            uint32_t a2[4];
            a2[0] = silu_pack(c0[0], c0[1]);
            a2[1] = silu_pack(c0[2], c0[3]);
            a2[2] = silu_pack(c1[0], c1[1]);
            a2[3] = silu_pack(c1[2], c1[3]);
            const uint2 b3 = P.w3[g][frag_slot(g, 4 * kt + tg)];
            mma_bf16_16816(d, a2, b3.x, b3.y);
        }
        // this m-tile's rows were read into the A fragments before its first MMA:
        // its outputs replace them (columns 2tg, 2tg+1 of rows g and g+8;
        // outputs 0..2 are in the lanes with tg < 2)
        __syncwarp();
        if (tg < 2) {
            io[r0][2 * tg] = d[0]; io[r0][2 * tg + 1] = d[1];
            io[r1][2 * tg] = d[2]; io[r1][2 * tg + 1] = d[3];
        }
    }
    __syncwarp();
    y[0] = io[lane][0]; y[1] = io[lane][1]; y[2] = io[lane][2];
    __syncwarp();
}

}  // namespace mlp
}  // namespace icempm
