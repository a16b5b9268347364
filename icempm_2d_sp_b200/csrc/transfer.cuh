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

// Slot of a placeholder point (cell padding of the locality order): it
// belongs to no host slot and is never written back.
constexpr uint32_t kSlotNone = 0xffffffffu;

template <class Real>
__global__ void k_download(Pts<Real> P, int n, double *__restrict__ stage, size_t pitch)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t s32 = P.slot[i];
    if (s32 == kSlotNone) return;
    const size_t s = s32;
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

// Boundary forces per node divided by elapsed steps * dt, into the layout of
// GPU_Implementation5::grid_boundary_forces (fx block, then fy block).
static __global__ void __launch_bounds__(256) k_forces_out(const double2 *__restrict__ force, long long G,
                                                           double div, double *__restrict__ out)
{
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= G) return;
    const double2 f = force[i];
    out[i] = __ddiv_rn(f.x, div);
    out[G + i] = __ddiv_rn(f.y, div);
}

// ---- sorting ---------------------------------------------------------------
// Locality key: cells grouped in TX x TY tiles, tiles in column order, cells
// column-major inside a tile; disabled points sort after the enabled ones and
// placeholders last.
struct TileKey { int tx, ty, ntiles_y; };
constexpr uint32_t kKeyDisabled = 0xfffffffeu, kKeyPlaceholder = 0xffffffffu;
static __global__ void k_keys_tiled(const uint2 *__restrict__ K, const uint32_t *__restrict__ slot, int n, TileKey t,
                                    uint32_t *keys, uint32_t *vals)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint2 k = K[i];
    uint32_t key = slot[i] == kSlotNone ? kKeyPlaceholder : kKeyDisabled;
    if (key == kKeyDisabled && !(k.y & kDisabled)) {
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

// ---- cell-aligned padding of the locality order ------------------------------
// The fused kernel gives each thread PPT consecutive points.  With four points
// per cell, padding every cell's run of points to a multiple of four with
// disabled placeholders puts each thread's points in one cell, which is what
// lets neighbouring threads merge their scatter patches and write them
// without shared atomics.  Runs are found on the sorted keys: start flags,
// an inclusive scan numbers the runs, each run's padded length is scanned to
// its padded start.

// first index whose key reaches each bound: bounds[0] = enabled count,
// bounds[1] = enabled + disabled count (keys sorted ascending)
static __global__ void k_key_bounds(const uint32_t *__restrict__ keys, int n, int *bounds)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    const uint32_t prev = i == 0 ? 0u : keys[i - 1];
    const uint32_t cur = i == n ? kKeyPlaceholder : keys[i];
    const bool prev_en = i > 0 && prev < kKeyDisabled, cur_en = i < n && cur < kKeyDisabled;
    const bool prev_real = i > 0 && prev != kKeyPlaceholder, cur_real = i < n && cur != kKeyPlaceholder;
    if ((i == 0 || prev_en) && !cur_en) bounds[0] = i;
    if ((i == 0 || prev_real) && !cur_real) bounds[1] = i;
}

static __global__ void k_run_flags(const uint32_t *__restrict__ keys, int n, uint32_t *flags)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    flags[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// run_id: inclusive scan of the flags (1-based run number of each entry)
static __global__ void k_run_begin(const uint32_t *__restrict__ run_id, int n, uint32_t *begin)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0 || run_id[i] != run_id[i - 1]) begin[run_id[i] - 1] = (uint32_t)i;
}

static __global__ void k_run_padded(const uint32_t *__restrict__ begin, int runs, int n, uint32_t *padded)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= runs) return;
    const uint32_t end = s + 1 < runs ? begin[s + 1] : (uint32_t)n;
    padded[s] = (end - begin[s] + 3u) & ~3u;
}

// Padded rank of sorted rank r: enabled points at their run's padded start
// plus their offset in the run, disabled points after all padded runs.
__device__ __forceinline__ size_t padded_rank(uint32_t r, uint32_t n_en, uint32_t n_pad_en,
                                              const uint32_t *__restrict__ run_id, const uint32_t *__restrict__ begin,
                                              const uint32_t *__restrict__ pstart)
{
    if (r >= n_en) return (size_t)n_pad_en + (r - n_en);
    const uint32_t s = run_id[r] - 1;
    return (size_t)pstart[s] + (r - begin[s]);
}

// dst[interleaved(padded_rank(r))] = src[perm[r]] for the n_real real points
template <class Real>
__global__ void k_gather_padded(Pts<Real> src, Pts<Real> dst, const uint32_t *__restrict__ perm, int n_real,
                                uint32_t n_en, uint32_t n_pad_en, uint32_t n_pad, const uint32_t *__restrict__ run_id,
                                const uint32_t *__restrict__ begin, const uint32_t *__restrict__ pstart, int ppt)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_real) return;
    const uint32_t j = perm[r];
    const size_t i = interleaved_position(padded_rank((uint32_t)r, n_en, n_pad_en, run_id, begin, pstart), n_pad, ppt);
    dst.A[i] = src.A[j]; dst.H[i] = src.H[j]; dst.C[i] = src.C[j];
    dst.V[i] = src.V[j]; dst.PQ[i] = src.PQ[j]; dst.K[i] = src.K[j];
    dst.slot[i] = src.slot[j];
    dst.pid[i] = src.pid[j];
    dst.thick64[i] = src.thick64[j];
}

// placeholders in the padding of each run (at most three per run)
template <class Real>
__global__ void k_fill_placeholders(Pts<Real> dst, int runs, uint32_t n_en, uint32_t n_pad, const uint32_t *__restrict__ begin,
                                    const uint32_t *__restrict__ pstart, const uint32_t *__restrict__ padded, int ppt)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= runs) return;
    const uint32_t end = s + 1 < runs ? begin[s + 1] : n_en;
    const uint32_t cnt = end - begin[s];
    for (uint32_t k = cnt; k < padded[s]; k++) {
        const size_t i = interleaved_position((size_t)pstart[s] + k, n_pad, ppt);
        V4<Real> z; z.x = z.y = z.z = z.w = Real(0);
        V2<Real> z2; z2.x = z2.y = Real(0);
        dst.A[i] = z; dst.H[i] = z; dst.C[i] = z; dst.V[i] = z2; dst.PQ[i] = z2;
        dst.K[i] = make_uint2(0u, kDisabled);
        dst.slot[i] = kSlotNone;
        dst.pid[i] = 0u;
        dst.thick64[i] = 0.0;
    }
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
    if (reset_done) { st->done = 0; st->chunk_ticket = 0; }
}

}  // namespace icempm
