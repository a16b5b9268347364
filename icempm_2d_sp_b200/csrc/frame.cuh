// frame.cuh -- the saved frame's grid arrays on the GPU
// (SnapshotManager::PrepareFrameArrays, snapshotmanager.cpp:623-765).
//
// Per enabled point, quadratic B-spline weights w of its 3x3 nodes spread
//   density += w, mass += w m_p, mass*vx += w m_p vx, mass*vy += w m_p vy,
//   Jp_inv, P, Q, r, g, b += w * value          (r, g, b: the point's colour)
// and the point counts in its cell; per node the sums become averages
// (velocity by mass, the rest by density; Jp_inv - 1), nodes with density
// <= 0.1 or a status other than 100 are zeroed, and the colour is blended
// with the water colour by alpha = clamp(density, 0, 1).  The boundary
// reaction of each node, divided by elapsed steps * dt, is summed per region
// (status >= 100 -> status - 99, else status).
//
// k_frame_scatter: one point per thread over the locality-sorted points; a
// CTA's nodes are accumulated in a shared tile (FP32 shared atomics) and
// flushed with one global atomic per non-zero node and channel.
// k_frame_finish: one node per thread; region sums reduced in shared memory.
#pragma once
#include "engine.cuh"

namespace icempm {

constexpr int kFrameChannels = 10;   // density, mass, m vx, m vy, Jp_inv, P, Q, r, g, b
constexpr int kFrameTile = 1024;     // nodes of a CTA's shared tile
// water colour (ColorMap::rgb_water, gui/colormap.h:36)
__host__ __device__ constexpr float water_rgb(int k) { return k == 0 ? 21.0f : (k == 1 ? 31.0f : 47.0f); }

struct FrameOut {
    float *ch[kFrameChannels];   // G each: the accumulated, then finished channels
    uint32_t *count;             // G: points per cell (the reference keeps the low 8 bits)
    uint8_t *rgb, *mask, *count8;
    float *region_force;         // 2 * ICEMPM_MAX_REGIONS
};

template <class Real>
__global__ void __launch_bounds__(256) k_frame_scatter(Pts<Real> P, int n, int gx, int gy, Real particle_mass,
                                                       const uint32_t *__restrict__ colors, uint32_t ncolors,
                                                       FrameOut F)
{
    __shared__ float tile[kFrameChannels][kFrameTile];
    __shared__ int box[4];
    if (threadIdx.x == 0) { box[0] = INT_MAX; box[1] = INT_MAX; box[2] = -1; box[3] = -1; }
    __syncthreads();
    const int i = blockIdx.x * 256 + threadIdx.x;
    bool active = false;
    int cx = 0, cy = 0;
    uint2 key = make_uint2(0u, kDisabled);
    if (i < n) {
        key = P.K[i];
        cx = (int)(key.x & 0xffff); cy = (int)(key.x >> 16);
        active = !(key.y & kDisabled) && cx >= 1 && cx <= gx - 2 && cy >= 1 && cy <= gy - 2;
    }
    {
        const unsigned FULL = 0xffffffffu;
        const unsigned xmn = __reduce_min_sync(FULL, active ? (unsigned)cx : 0x7fffffffu);
        const unsigned ymn = __reduce_min_sync(FULL, active ? (unsigned)cy : 0x7fffffffu);
        const unsigned xmx = __reduce_max_sync(FULL, active ? (unsigned)cx : 0u);
        const unsigned ymx = __reduce_max_sync(FULL, active ? (unsigned)cy : 0u);
        const bool warp_any = __any_sync(FULL, active);   // every lane votes (a skipped lane stalls the warp)
        if ((threadIdx.x & 31) == 0 && warp_any) {
            atomicMin(&box[0], (int)xmn); atomicMin(&box[1], (int)ymn);
            atomicMax(&box[2], (int)xmx); atomicMax(&box[3], (int)ymx);
        }
    }
    __syncthreads();
    const int x0 = box[0] - 1, y0 = box[1] - 1;
    const int tw = box[2] - box[0] + 3, th = box[3] - box[1] + 3;
    const bool on = box[2] >= 0 && (long long)tw * (long long)th <= (long long)kFrameTile;
    const int nt = on ? tw * th : 0;
    for (int k = threadIdx.x; k < nt; k += 256)
#pragma unroll
        for (int c = 0; c < kFrameChannels; c++) tile[c][k] = 0.0f;
    __syncthreads();
    if (active) {
        const V4<Real> A = P.A[i];
        const V2<Real> v = P.V[i], pq = P.PQ[i];
        const uint32_t pid = P.pid[i];
        const uint32_t col = (colors && pid < ncolors) ? colors[pid] : 0xffffffu;
        const float vals[kFrameChannels] = {1.0f, 0.0f, 0.0f, 0.0f, float(A.z), float(pq.x), float(pq.y),
                                            float((col >> 16) & 0xff), float((col >> 8) & 0xff), float(col & 0xff)};
        const float mp = float(particle_mass * A.w);
        Real wx[3], wy[3];
        bspline(A.x, wx);
        bspline(A.y, wy);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const float w = float(wx[a] * wy[b]);
                const int X = cx + a - 1, Y = cy + b - 1;
                float add[kFrameChannels];
#pragma unroll
                for (int c = 0; c < kFrameChannels; c++) add[c] = w * vals[c];
                add[1] = w * mp;
                add[2] = w * mp * float(v.x);
                add[3] = w * mp * float(v.y);
                if (on) {
                    const int li = (X - x0) * th + (Y - y0);
#pragma unroll
                    for (int c = 0; c < kFrameChannels; c++) atomicAdd(&tile[c][li], add[c]);
                } else {
                    const size_t node = (size_t)X * gy + Y;
#pragma unroll
                    for (int c = 0; c < kFrameChannels; c++) atomicAdd(&F.ch[c][node], add[c]);
                }
            }
        atomicAdd(&F.count[(size_t)cx * gy + cy], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nt; k += 256) {
        const int lx = k / th, ly = k - lx * th;
        const size_t node = (size_t)(x0 + lx) * gy + (y0 + ly);
#pragma unroll
        for (int c = 0; c < kFrameChannels; c++)
            if (tile[c][k] != 0.0f) atomicAdd(&F.ch[c][node], tile[c][k]);
    }
}

static __device__ __forceinline__ uint8_t clamp_u8(float v) { return (uint8_t)fminf(fmaxf(v, 0.0f), 255.0f); }

static __global__ void __launch_bounds__(256) k_frame_finish(FrameOut F, const uint8_t *__restrict__ status,
                                                      const double2 *__restrict__ force, double force_div,
                                                      long long G)
{
    __shared__ float rf[2 * ICEMPM_MAX_REGIONS];
    for (int k = threadIdx.x; k < 2 * ICEMPM_MAX_REGIONS; k += 256) rf[k] = 0.0f;
    __syncthreads();
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i < G) {
        float c[kFrameChannels];
#pragma unroll
        for (int k = 0; k < kFrameChannels; k++) c[k] = F.ch[k][i];
        const float density = c[0], mass = c[1];
        if (density > 0.0f) {
            const float coeff = 1.0f / density;
            c[2] /= mass;
            c[3] /= mass;
            c[7] *= coeff; c[8] *= coeff; c[9] *= coeff;
            c[4] = c[4] * coeff - 1.0f;
            c[5] *= coeff;
            c[6] *= coeff;
        }
        const uint8_t mask = density > 0.1f ? 1 : 0;
        const uint8_t st = status[i];
        if (!mask || st != 100) {
            c[0] = 0.0f; c[1] = 0.0f; c[2] = c[3] = c[4] = c[5] = c[6] = 0.0f;
        }
        const float alpha = fminf(fmaxf(density, 0.0f), 1.0f);
#pragma unroll
        for (int k = 0; k < 3; k++)
            F.rgb[3 * i + k] = (uint8_t)(alpha * (float)clamp_u8(c[7 + k]) + (1.0f - alpha) * water_rgb(k));
#pragma unroll
        for (int k = 0; k < kFrameChannels; k++) F.ch[k][i] = c[k];
        F.mask[i] = mask;
        F.count8[i] = (uint8_t)F.count[i];
        const int region = st >= 100 ? st - 99 : st;
        if (region < ICEMPM_MAX_REGIONS) {
            const double2 f = force[i];
            if (f.x != 0.0) atomicAdd(&rf[2 * region], (float)(f.x / force_div));
            if (f.y != 0.0) atomicAdd(&rf[2 * region + 1], (float)(f.y / force_div));
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 2 * ICEMPM_MAX_REGIONS; k += 256)
        if (rf[k] != 0.0f) atomicAdd(&F.region_force[k], rf[k]);
}

}  // namespace icempm
