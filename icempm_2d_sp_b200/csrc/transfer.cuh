// transfer.cuh -- host<->device conversion of the reference HSSOA layout,
// locality sorting keys, permutation gather and compaction helpers.
#pragma once
#include "engine.cuh"

namespace icempm {

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

// Position of the point of sorted rank r when each warp-chunk of 32*ppt points
// is interleaved for the fused kernel (lane l, iteration j reads
// chunk*32*ppt + j*32 + l; rank chunk*32*ppt + l*ppt + j goes there).  The
// last, partial chunk keeps rank order.  ppt = 0 or 1: identity.
__host__ __device__ __forceinline__ size_t interleaved_position(size_t r, size_t n, int ppt)
{
    if (ppt <= 1) return r;
    const size_t chunk = (size_t)32 * ppt;
    const size_t c = r / chunk;
    if ((c + 1) * chunk > n) return r;
    const size_t rem = r - c * chunk;
    return c * chunk + (rem % ppt) * 32 + rem / ppt;
}

// dst[position(r)] = src[perm[r]]; with reslot, host slots become the rank.
template <class Real>
__global__ void k_gather(Pts<Real> src, Pts<Real> dst, const uint32_t *__restrict__ perm, int n, int reslot,
                         int ppt)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const uint32_t j = perm[r];
    const size_t i = interleaved_position((size_t)r, (size_t)n, ppt);
    dst.A[i] = src.A[j]; dst.H[i] = src.H[j]; dst.C[i] = src.C[j];
    dst.V[i] = src.V[j]; dst.PQ[i] = src.PQ[j]; dst.K[i] = src.K[j];
    dst.slot[i] = reslot ? (uint32_t)r : src.slot[j];
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

// Sets the index of the next sub-step (step >= 0; step < 0 keeps it) and
// marks the last G2P sub-step of the coming nsteps as the one that stores
// the point velocity and C.
static __global__ void k_set_step(DevStatus *st, int step, int reset_done, int nsteps)
{
    if (step >= 0) st->step = step;
    st->vc_step = st->step + nsteps - 1;
    if (reset_done) st->done = 0;
}

}  // namespace icempm
