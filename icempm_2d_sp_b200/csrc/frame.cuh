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
// k_frame_scatter: four entries of the locality order per thread (one cell,
// as the sort arranged them), their node terms summed in registers column by
// column and merged with the vertically adjacent lanes' overlapping nodes;
// each node's sums go straight to the global accumulators with three 16-byte
// vector reductions (`red.global.add.v4.f32`): a node's eleven channels (the
// ten above and the point count of its cell) are interleaved in three float4.
// k_frame_finish: one node per thread; region sums reduced in shared memory.
#pragma once
#include "engine.cuh"

namespace icempm {

constexpr int kFrameChannels = 10;   // density, mass, m vx, m vy, Jp_inv, P, Q, r, g, b
// water colour (ColorMap::rgb_water, gui/colormap.h:36)
__host__ __device__ constexpr float water_rgb(int k) { return k == 0 ? 21.0f : (k == 1 ? 31.0f : 47.0f); }

struct FrameOut {
    float4 *acc;                 // 3 per node: the ten channels and the cell's point count, interleaved
    float *ch[kFrameChannels];   // G each: the finished channels
    uint8_t *rgb, *mask, *count8;
    float *region_force;         // 2 * ICEMPM_MAX_REGIONS
};

// Channel values of one point: density weight, mass, m vx, m vy, Jp_inv, P, Q, r, g, b.
template <class Real>
__device__ __forceinline__ void frame_values(const Pts<Real> &P, int i, Real particle_mass,
                                             const uint32_t *__restrict__ colors, uint32_t ncolors,
                                             float vals[kFrameChannels], float &x, float &y)
{
    const V4<Real> A = P.A[i];
    const V2<Real> v = P.V[i], pq = P.PQ[i];
    const uint32_t pid = P.pid[i];
    const uint32_t col = (colors && pid < ncolors) ? colors[pid] : 0xffffffu;
    const float mp = float(particle_mass * A.w);
    vals[0] = 1.0f; vals[1] = mp; vals[2] = mp * float(v.x); vals[3] = mp * float(v.y);
    vals[4] = float(A.z); vals[5] = float(pq.x); vals[6] = float(pq.y);
    vals[7] = float((col >> 16) & 0xff); vals[8] = float((col >> 8) & 0xff); vals[9] = float(col & 0xff);
    x = float(A.x); y = float(A.y);
}

__device__ __forceinline__ void red_add_v4(float4 *a, float x, float y, float z, float w)
{
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(a), "f"(x), "f"(y), "f"(z),
                 "f"(w)
                 : "memory");
}

// Adds node (X, Y)'s channel sums and `count` points to the accumulators.
__device__ __forceinline__ void frame_node_add(const FrameOut &F, int gy, int X, int Y, const float add[kFrameChannels],
                                               float count)
{
    float4 *a = F.acc + 3 * ((size_t)X * gy + Y);
    red_add_v4(a, add[0], add[1], add[2], add[3]);
    red_add_v4(a + 1, add[4], add[5], add[6], add[7]);
    red_add_v4(a + 2, add[8], add[9], count, 0.0f);
}

// A CTA takes 1024 entries of the locality order: 8 warps x 128, thread
// (warp w, lane l) the entries w*128 + 32j + l, j = 0..3, which the sort put
// in one cell.  When a thread's enabled points do share a cell, their node
// terms are summed in registers first, one column of three nodes at a time;
// lanes whose cells are vertically adjacent in one column (lane l+1 one cell
// above lane l, the usual case in the locality order) overlap in two of those
// nodes, so each lane adds its upper neighbour's lowest node and its lower
// neighbour's highest node into its centre node (warp shuffles) and writes a
// corner node only where no neighbour took it: three reductions per node for
// up to four points, and in a full column one node per column instead of
// three.  A thread whose points span cells adds each point on its own.
template <class Real>
__global__ void __launch_bounds__(256, 2) k_frame_scatter(Pts<Real> P, int n, int gx, int gy, Real particle_mass,
                                                       const uint32_t *__restrict__ colors, uint32_t ncolors,
                                                       FrameOut F)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int e0 = blockIdx.x * 1024 + w * 128 + lane;
    bool act[4];
    int cxs[4], cys[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int i = e0 + 32 * j;
        act[j] = false; cxs[j] = 0; cys[j] = 0;
        if (i < n) {
            const uint2 key = P.K[i];
            const int cx = (int)(key.x & 0xffff), cy = (int)(key.x >> 16);
            act[j] = !(key.y & kDisabled) && cx >= 1 && cx <= gx - 2 && cy >= 1 && cy <= gy - 2;
            cxs[j] = cx; cys[j] = cy;
        }
    }
    // the thread's enabled points: one cell?
    int first = -1, nact = 0;
    bool one_cell = true;
#pragma unroll
    for (int j = 0; j < 4; j++)
        if (act[j]) {
            if (first < 0) first = j;
            else if (cxs[j] != cxs[first] || cys[j] != cys[first]) one_cell = false;
            nact++;
        }
    const bool mine = nact > 0 && one_cell;
    int cx = 0, cy = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) if (j == first) { cx = cxs[j]; cy = cys[j]; }
    const uint32_t key = mine ? (((uint32_t)cx << 16) | (uint32_t)cy) : 0xffffffffu;
    const uint32_t key_up = __shfl_down_sync(FULL, key, 1);   // lane l+1
    const uint32_t key_dn = __shfl_up_sync(FULL, key, 1);     // lane l-1
    const bool above = mine && lane < 31 && key_up == key + 1u;
    const bool below = mine && lane > 0 && key_dn == key - 1u;

    // every lane takes part in the column loop (the shuffles); lanes without
    // a one-cell patch carry zeros and write nothing
    {
        float vals[4][kFrameChannels], wx[4][3], wy[4][3];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float x = 0.0f, y = 0.0f;
            if (mine && act[j]) {
                frame_values(P, e0 + 32 * j, particle_mass, colors, ncolors, vals[j], x, y);
                bspline(x, wx[j]);
                bspline(y, wy[j]);
            } else {
#pragma unroll
                for (int c = 0; c < kFrameChannels; c++) vals[j][c] = 0.0f;
#pragma unroll
                for (int k = 0; k < 3; k++) { wx[j][k] = 0.0f; wy[j][k] = 0.0f; }
            }
        }
#pragma unroll 1
        for (int a = 0; a < 3; a++) {
            float add[3][kFrameChannels + 1];   // nodes (a, 0..2): the ten channels and the point count
#pragma unroll
            for (int b = 0; b < 3; b++) {
#pragma unroll
                for (int c = 0; c < kFrameChannels; c++) add[b][c] = 0.0f;
                add[b][kFrameChannels] = (a == 1 && b == 1) ? float(nact) : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float wa = a == 0 ? wx[j][0] : (a == 1 ? wx[j][1] : wx[j][2]);   // registers, not a stack array
#pragma unroll
                for (int b = 0; b < 3; b++) {
                    const float wgt = wa * wy[j][b];
#pragma unroll
                    for (int c = 0; c < kFrameChannels; c++) add[b][c] += wgt * vals[j][c];
                }
            }
#pragma unroll
            for (int c = 0; c <= kFrameChannels; c++) {
                const float up = __shfl_down_sync(FULL, add[0][c], 1), dn = __shfl_up_sync(FULL, add[2][c], 1);
                if (above) add[1][c] += up;
                if (below) add[1][c] += dn;
            }
            if (mine) {
                frame_node_add(F, gy, cx + a - 1, cy, add[1], add[1][kFrameChannels]);
                // one pass for the edge node each lane still owns (in a column
                // run of cells only the run's ends own one), a second where a
                // lane owns both (a cell without vertical neighbours)
                if (!below || !above) {
                    float e[kFrameChannels + 1];
#pragma unroll
                    for (int c = 0; c <= kFrameChannels; c++) e[c] = !below ? add[0][c] : add[2][c];
                    frame_node_add(F, gy, cx + a - 1, cy + (!below ? -1 : 1), e, e[kFrameChannels]);
                }
                if (!below && !above) frame_node_add(F, gy, cx + a - 1, cy + 1, add[2], add[2][kFrameChannels]);
            }
        }
    }
    if (nact > 0 && !one_cell) {
#pragma unroll 1
        for (int j = 0; j < 4; j++) {
            if (!act[j]) continue;
            float vals[kFrameChannels], x, y, wx[3], wy[3];
            frame_values(P, e0 + 32 * j, particle_mass, colors, ncolors, vals, x, y);
            bspline(x, wx);
            bspline(y, wy);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    const float wgt = wx[a] * wy[b];
                    float add[kFrameChannels];
#pragma unroll
                    for (int c = 0; c < kFrameChannels; c++) add[c] = wgt * vals[c];
                    frame_node_add(F, gy, cxs[j] + a - 1, cys[j] + b - 1, add, (a == 1 && b == 1) ? 1.0f : 0.0f);
                }
        }
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
        const float4 a0 = F.acc[3 * i], a1 = F.acc[3 * i + 1], a2 = F.acc[3 * i + 2];
        float c[kFrameChannels] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y};
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
        F.count8[i] = (uint8_t)(uint32_t)a2.z;   // the reference keeps the low 8 bits
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
