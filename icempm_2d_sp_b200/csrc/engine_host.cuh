// engine_host.cuh -- host side of one variant of the step: device memory,
// host<->device conversion, the step loop (CUDA graphs), locality sorting and
// compaction.  Instantiated once per variant in engine_<variant>.cu.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

#include "transfer.cuh"
#include "frame.cuh"
#include "forcing.cuh"
#include "engine_iface.h"

namespace icempm {

#define ICEMPM_CUDA(call)                                                              \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

static inline double pow2_floor(double x) { return std::ldexp(1.0, (int)std::floor(std::log2(x))); }

template <class Real, class Acc> class BatchT;

template <class Real, class Acc>
class EngineT final : public Engine {
    friend class BatchT<Real, Acc>;

public:
    // fused kernel: threads per CTA and points per thread (a chunk of BT*PPT
    // points per CTA iteration; FP64 state halves the chunk to fit two stages)
    static constexpr int BT = sizeof(Real) == 8 ? 128 : ICEMPM_FUSED_BT;
    static constexpr int PPT = sizeof(Real) == 8 ? 2 : ICEMPM_FUSED_PPT;
    static constexpr int CH = BT * PPT;
    static constexpr int CAP = ICEMPM_FUSED_CAP;     // nodes in the fused kernel's shared scatter tile (0: none)
    static constexpr int CAP_P2G = 512;              // nodes in the priming scatter's shared tile
    static constexpr int BT_P2G = 256;   // threads per CTA of the priming scatter
    static constexpr int GRAPH_STEPS = 32;
    static constexpr size_t PAD = 2048;  // point arrays are padded to whole chunks
    static constexpr int STAGES = ICEMPM_FUSED_STAGES;
    using FusedSmem = ChunkSmem<Real, Acc, BT, PPT, CAP, STAGES>;

    EngineT() = default;
    ~EngineT() override { release(); }

    int init(const icempm_simparams_t &p, const uint8_t *status, const double *cur, uint32_t capacity,
             const icempm_options_t &o) override
    {
        prms_ = p; opts_ = o;
        gx_ = p.GridXTotal; gy_ = p.GridYTotal;
        if (gx_ < 5 || gy_ < 5 || gx_ > 65535 || gy_ > 65535) return fail(ICEMPM_E_ARG, "grid size out of range");
        if (!(p.cellsize > 0) || !(p.InitialTimeStep > 0)) return fail(ICEMPM_E_ARG, "cellsize and InitialTimeStep must be > 0");
        G_ = (size_t)gx_ * gy_;
        cap_ = std::max<uint32_t>(capacity, 1);
        ICEMPM_CUDA(cudaSetDevice(o.device));
        ICEMPM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        ICEMPM_CUDA(cudaEventCreate(&ev0_));
        ICEMPM_CUDA(cudaEventCreate(&ev1_));
        ICEMPM_CUDA(cudaEventCreate(&evs_[0]));
        ICEMPM_CUDA(cudaEventCreate(&evs_[1]));
        ICEMPM_CUDA(cudaEventCreate(&evs_[2]));
        // points, two parities for the sort gather
        // room for the cell padding of the locality order (a quarter more), in
        // whole chunks (the bulk copies read whole chunks)
        const size_t nc = ((size_t)cap_ + cap_ / 4 + 4 * PAD + PAD - 1) / PAD * PAD;
        nc_ = nc;
        const size_t per = nc * (3 * sizeof(V4<Real>) + 2 * sizeof(V2<Real>) + sizeof(uint2) + 2 * sizeof(uint32_t) + sizeof(double));
        ICEMPM_CUDA(cudaMalloc(&pts_mem_, 2 * per));
        for (int par = 0; par < 2; par++) {
            char *b = (char *)pts_mem_ + par * per;
            auto take = [&](size_t bytes) { char *r = b; b += bytes; return r; };
            Pts<Real> &P = pts_[par];
            P.A = (V4<Real> *)take(nc * sizeof(V4<Real>));
            P.H = (V4<Real> *)take(nc * sizeof(V4<Real>));
            P.C = (V4<Real> *)take(nc * sizeof(V4<Real>));
            P.V = (V2<Real> *)take(nc * sizeof(V2<Real>));
            P.PQ = (V2<Real> *)take(nc * sizeof(V2<Real>));
            P.K = (uint2 *)take(nc * sizeof(uint2));
            P.thick64 = (double *)take(nc * sizeof(double));
            P.slot = (uint32_t *)take(nc * sizeof(uint32_t));
            P.pid = (uint32_t *)take(nc * sizeof(uint32_t));
        }
        // grid
        Gp_ = (G_ + 31) / 32 * 32;   // channel stride: every channel starts 256-byte aligned
        ICEMPM_CUDA(cudaMalloc(&acc_, 3 * Gp_ * sizeof(Acc)));
        ICEMPM_CUDA(cudaMalloc(&vel_, G_ * sizeof(V2<Real>)));
        ICEMPM_CUDA(cudaMalloc(&cur_, G_ * sizeof(V2<Real>)));
        ICEMPM_CUDA(cudaMalloc(&frc_, G_ * sizeof(V4<Real>)));
        ICEMPM_CUDA(cudaMalloc(&status_, G_));
        ICEMPM_CUDA(cudaMalloc(&force_, G_ * sizeof(double2)));
        ICEMPM_CUDA(cudaMalloc(&st_, sizeof(DevStatus)));
        ICEMPM_CUDA(cudaMemsetAsync(acc_, 0, 3 * Gp_ * sizeof(Acc), stream_));
        ICEMPM_CUDA(cudaMemsetAsync(vel_, 0, G_ * sizeof(V2<Real>), stream_));
        ICEMPM_CUDA(cudaMemsetAsync(force_, 0, G_ * sizeof(double2), stream_));
        ICEMPM_CUDA(cudaMemsetAsync(st_, 0, sizeof(DevStatus), stream_));
        ICEMPM_CUDA(cudaMemcpyAsync(status_, status, G_, cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        int rc = set_current(cur);
        if (rc) return rc;
        // sort buffers
        ICEMPM_CUDA(cudaMalloc(&keys_[0], nc * sizeof(uint64_t)));
        ICEMPM_CUDA(cudaMalloc(&keys_[1], nc * sizeof(uint64_t)));
        ICEMPM_CUDA(cudaMalloc(&vals_[0], nc * sizeof(uint32_t)));
        ICEMPM_CUDA(cudaMalloc(&vals_[1], nc * sizeof(uint32_t)));
        ICEMPM_CUDA(cudaMalloc(&runs_, nc * sizeof(uint32_t)));
        ICEMPM_CUDA(cudaMalloc(&aux_, 8 * sizeof(int)));
        size_t t32 = 0, t64 = 0;
        ICEMPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t32, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                                    (uint32_t *)nullptr, (uint32_t *)nullptr, (int)nc, 0, 32, stream_));
        ICEMPM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, t64, (uint64_t *)nullptr, (uint64_t *)nullptr,
                                                    (uint32_t *)nullptr, (uint32_t *)nullptr, (int)nc, 0, 64, stream_));
        size_t ts1 = 0, ts2 = 0;
        ICEMPM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, ts1, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)nc, stream_));
        ICEMPM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, ts2, (uint32_t *)nullptr, (uint32_t *)nullptr, (int)nc, stream_));
        sort_tmp_bytes_ = std::max(std::max(t32, t64), std::max(ts1, ts2));
        ICEMPM_CUDA(cudaMalloc(&sort_tmp_, sort_tmp_bytes_));
        // a CTA of the fused kernel handles BT*PPT points, ~BT*PPT/4 cells at
        // 4 points per cell: one column strip of BT*PPT/4 cells, so that a
        // warp's 32 cells are 32 consecutive cells of one column (its
        // reductions then form one contiguous run of nodes per node row and
        // channel; fused kernel 0.500 ms with 8x16-cell tiles, 0.489 with 2x64,
        // 0.485 with 1x128 on the 23M-point scene)
        tile_.tx = 1; tile_.ty = BT * PPT / 4;
        tile_.ntiles_y = (gy_ + tile_.ty - 1) / tile_.ty;
        // persistent grid of the fused kernel: as many CTAs as fit on the device
        auto kern = k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_PLAIN>;
        ICEMPM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FusedSmem)));
        ICEMPM_CUDA(cudaFuncSetAttribute(k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_HARVEST>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FusedSmem)));
        if constexpr (sizeof(Real) == 4) {
            auto lk = k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_LEARNED>;
            const int lb = (int)fused_smem_bytes<FusedSmem, BT, FUSED_LEARNED>();
            ICEMPM_CUDA(cudaFuncSetAttribute(lk, cudaFuncAttributeMaxDynamicSharedMemorySize, lb));
            int lper = 0, lsms = 0;
            ICEMPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lper, lk, BT, lb));
            ICEMPM_CUDA(cudaDeviceGetAttribute(&lsms, cudaDevAttrMultiProcessorCount, o.device));
            learned_ctas_ = lper * lsms;
        }
        int per_sm = 0, sms = 0;
        ICEMPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, sizeof(FusedSmem)));
        ICEMPM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o.device));
        if (per_sm < 1) return fail(ICEMPM_E_UNSUPPORTED, "fused kernel does not fit on one SM");
        fused_ctas_ = per_sm * sms;
        return set_params(p, 1.0);
    }

    int set_params(const icempm_simparams_t &p, double max_thickness) override
    {
        prms_ = p;
        if (max_thickness > 0) max_thick_ = max_thickness;
        KParams<Real> &k = kp_;
        k.gx = gx_; k.gy = gy_;
        k.update_every = p.UpdateEveryNthStep;
        k.ext = opts_.forcing == ICEMPM_FORCING_EXTENDED; k.wind_kind = opts_.wind_kind;   // wind lives in frc_
        k.h = Real(p.cellsize); k.h_inv = Real(p.cellsize_inv);
        k.dt = Real(p.InitialTimeStep);
        k.dt_h_inv = Real(p.InitialTimeStep * p.cellsize_inv);
        k.four_h_inv = Real(4.0 * p.cellsize_inv);
        k.vmax2_01 = Real(p.vmax * p.vmax * 0.1);
        k.particle_mass = Real(p.ParticleMass);
        k.dt_vol_Dpinv = Real(p.dt_vol_Dpinv);
        k.dt_d = p.InitialTimeStep;
        k.kL = p.waterDragEffectiveLinear * p.InitialTimeStep;
        k.kQ = p.waterDragEffectiveQuadratic * p.InitialTimeStep;
        const double mref = std::max(p.ParticleMass * max_thick_, 1e-30);
        k.scale_m = pow2_floor(std::ldexp(1.0, 62) / (4096.0 * mref));
        k.scale_p = k.scale_m / 16.0;
        k.inv_scale_m = 1.0 / k.scale_m; k.inv_scale_p = 1.0 / k.scale_p;
        // one term may use 2^56 of the 2^63 range: 64 worst-case terms fit a node
        k.lim_m = (float)(std::ldexp(1.0, 56) / k.scale_m);
        k.lim_p = (float)(std::ldexp(1.0, 56) / k.scale_p);
        {   // broadcast pairs (the fixed-point scales are powers of two: exact in Real)
            using PT = P2<Real>;
            const auto pair = [](Real v) { PT r; r.x = v; r.y = v; return r; };
            constexpr bool FIXED = AccOps<Acc>::fixed;
            const Real sp = FIXED ? Real(k.scale_p) : Real(1);
            k.dt_h_inv2 = pair(k.dt_h_inv); k.neg_four_h_inv2 = pair(-k.four_h_inv); k.neg_h2 = pair(-k.h);
            k.one2 = pair(Real(1)); k.half2 = pair(Real(0.5));
            k.sp2 = pair(sp); k.hsp2 = pair(k.h * sp);
            k.sm_r = FIXED ? Real(k.scale_m) : Real(1);
        }
        k.ext_impulse = Real(p.InitialTimeStep * p.ParticleVolume);
        k.ext_impulse2.x = k.ext_impulse; k.ext_impulse2.y = k.ext_impulse;
        k.rho_w_cd = Real(opts_.water_density * opts_.water_drag_coeff);
        const Material m = material_of(p);
        k.mat = mat_of<Real>(m);
        k.harvest = harvest_;
        k.harvest_stride = harvest_stride_;
        k.tx_extra = tx_extra_;
        k.wait_ns = wait_ns_;
        primed_ = false;
        invalidate_graphs();
        return 0;
    }

    // Tests of the barrier-timeout path: each chunk's barrier expects
    // `extra_bytes` more than its copies deliver, and a wait gives up after
    // `wait_us` (0, 0 restores the production setting: exact bytes, 1 s).
    int set_barrier_test(uint32_t extra_bytes, uint32_t wait_us) override
    {
        tx_extra_ = extra_bytes;
        wait_ns_ = wait_us ? 1000ull * wait_us : kWaitLimitNs;
        kp_.tx_extra = tx_extra_;
        kp_.wait_ns = wait_ns_;
        invalidate_graphs();
        return 0;
    }

    // Wind at a world position for the extended forcing: uniform, or a
    // Rankine vortex (solid-body inside the radius, 1/r outside).
    void wind(double x, double y, double &ux, double &uy) const
    {
        ux = 0; uy = 0;
        if (opts_.wind_kind == ICEMPM_WIND_UNIFORM) { ux = opts_.wind_u; uy = opts_.wind_v; }
        else if (opts_.wind_kind == ICEMPM_WIND_RANKINE) {
            const double dx = x - opts_.wind_cx, dy = y - opts_.wind_cy;
            const double r = std::sqrt(dx * dx + dy * dy);
            if (r > 0) {
                const double sp = (r < opts_.wind_radius) ? opts_.wind_vmax * r / opts_.wind_radius
                                                          : opts_.wind_vmax * opts_.wind_radius / r;
                ux = -dy / r * sp; uy = dx / r * sp;
            }
        }
    }

    // Current per node, and for the extended forcing the node table
    // {current, wind stress rho_a Ca |U| U} read by the point impulses.
    int set_current(const double *cur) override
    {
        std::vector<V2<Real>> h(G_);
        std::vector<V4<Real>> f(G_);
        const double ca = opts_.air_density * opts_.air_drag_coeff;
        for (size_t i = 0; i < G_; i++) {
            const double cx = cur ? cur[i] : 0.0, cy = cur ? cur[G_ + i] : 0.0;
            h[i].x = Real(cx); h[i].y = Real(cy);
            double ux, uy;
            wind((double)(i / gy_) * prms_.cellsize, (double)(i % gy_) * prms_.cellsize, ux, uy);
            const double um = std::sqrt(ux * ux + uy * uy);
            f[i].x = Real(cx); f[i].y = Real(cy);
            f[i].z = Real(ca * um * ux); f[i].w = Real(ca * um * uy);
        }
        ICEMPM_CUDA(cudaMemcpyAsync(cur_, h.data(), G_ * sizeof(V2<Real>), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaMemcpyAsync(frc_, f.data(), G_ * sizeof(V4<Real>), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        // the extended forcing enters the P2G: a P2G already done for the next step is stale
        if (opts_.forcing == ICEMPM_FORCING_EXTENDED) primed_ = false;
        return 0;
    }

    // ---- time-varying forcing (forcing.cuh) ----
    int set_flow_frames(const double *a, const double *b) override
    {
        if (!a && b) return fail(ICEMPM_E_ARG, "current frame b given without frame a");
        if (!a) { cudaFree(flow_ab_); flow_ab_ = nullptr; return 0; }
        if (!b) b = a;
        if (!flow_ab_) ICEMPM_CUDA(cudaMalloc(&flow_ab_, 4 * G_ * sizeof(double)));
        ICEMPM_CUDA(cudaMemcpyAsync(flow_ab_, a, 2 * G_ * sizeof(double), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaMemcpyAsync(flow_ab_ + 2 * G_, b, 2 * G_ * sizeof(double), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return 0;
    }
    int set_wind_frames(const float *w, int rows, int cols, double cell, double x0, double y0) override
    {
        if (!w) { cudaFree((void *)wind_.w); wind_ = WindGrid{}; wind_cap_ = 0; return 0; }
        if (rows < 1 || cols < 1 || (long long)rows * cols > (1LL << 28))
            return fail(ICEMPM_E_ARG, "wind grid rows and cols must be in 1..2^28 samples");
        if (!(cell > 0) || !std::isfinite(cell) || !std::isfinite(x0) || !std::isfinite(y0))
            return fail(ICEMPM_E_ARG, "wind grid spacing must be finite and > 0, origin finite");
        const size_t ns = (size_t)rows * cols;
        if (ns > wind_cap_) {
            cudaFree((void *)wind_.w);
            wind_.w = nullptr;
            ICEMPM_CUDA(cudaMalloc((void **)&wind_.w, ns * sizeof(float4)));
            wind_cap_ = ns;
        }
        ICEMPM_CUDA(cudaMemcpyAsync((void *)wind_.w, w, ns * sizeof(float4), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        wind_.rows = rows; wind_.cols = cols; wind_.cell = cell; wind_.x0 = x0; wind_.y0 = y0;
        return 0;
    }
    int set_forcing_time(double tc, double tw) override
    {
        if (!flow_ab_ && !wind_.w) return fail(ICEMPM_E_STATE, "no current or wind frames set");
        if (!(tc >= 0 && tc <= 1) || !(tw >= 0 && tw <= 1))
            return fail(ICEMPM_E_ARG, "interpolation weights must be in [0, 1]");
        const unsigned nb = (unsigned)((G_ + 255) / 256);
        k_blend_forcing<Real><<<nb, 256, 0, stream_>>>((long long)G_, gy_, prms_.cellsize, flow_ab_,
                                                      flow_ab_ ? flow_ab_ + 2 * G_ : nullptr, tc, wind_, tw,
                                                      opts_.air_density * opts_.air_drag_coeff, cur_, frc_);
        ICEMPM_CUDA(cudaGetLastError());
        launches_++;
        if (opts_.forcing == ICEMPM_FORCING_EXTENDED) primed_ = false;
        return 0;
    }
    int get_forcing(double *cur, double *stress) override
    {
        std::vector<V4<Real>> f(G_);
        ICEMPM_CUDA(cudaMemcpyAsync(f.data(), frc_, G_ * sizeof(V4<Real>), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        for (size_t i = 0; i < G_; i++) {
            if (cur) { cur[i] = (double)f[i].x; cur[G_ + i] = (double)f[i].y; }
            if (stress) { stress[i] = (double)f[i].z; stress[G_ + i] = (double)f[i].w; }
        }
        return 0;
    }

    int ensure_stage()
    {
        if (stage_) return 0;
        ICEMPM_CUDA(cudaMalloc(&stage_, (size_t)ICEMPM_N_PTS_ARRAYS * cap_ * sizeof(double)));
        return 0;
    }

    int upload(const double *hssoa, uint32_t host_cap, uint32_t n, int32_t disabled) override
    {
        if (n > cap_) return fail(ICEMPM_E_CAPACITY, "point count exceeds the context capacity");
        if (n > host_cap) return fail(ICEMPM_E_ARG, "size exceeds the host buffer capacity");
        int rc = ensure_stage();
        if (rc) return rc;
        rc = stage_free();
        if (rc) return rc;
        if (n > 0) {
            ICEMPM_CUDA(cudaMemcpy2DAsync(stage_, (size_t)n * sizeof(double), hssoa, (size_t)host_cap * sizeof(double),
                                          (size_t)n * sizeof(double), ICEMPM_N_PTS_ARRAYS, cudaMemcpyHostToDevice, stream_));
            k_upload<Real><<<(n + 255) / 256, 256, 0, stream_>>>(stage_, n, (int)n, pts_[par_]);
            ICEMPM_CUDA(cudaGetLastError());
            launches_++;
        }
        n_ = n;
        n_real_ = n;
        double mt = 0;
        for (uint32_t i = 0; i < n; i++) mt = std::max(mt, std::fabs(hssoa[(size_t)18 * host_cap + i]));
        set_params(prms_, mt > 0 ? mt : 1.0);
        DevStatus s{};
        s.disabled = disabled;
        ICEMPM_CUDA(cudaMemcpyAsync(&st_->disabled, &s.disabled, sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        steps_since_sort_ = 0;
        if (n_ > 0) {
            rc = locality_sort();
            if (rc) return rc;
        }
        return 0;
    }

    int download(double *hssoa, uint32_t host_cap, uint32_t *size) override
    {
        int rc = download_async(hssoa, host_cap, size);
        if (rc) return rc;
        rc = download_wait();
        if (rc) return rc;
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return 0;
    }

    // The state is converted into the staging buffer on the compute stream;
    // the device-to-host copy runs on the copy stream, so sub-steps enqueued
    // afterwards overlap it.  A later upload or download first waits (on the
    // device) for the copy that still reads the staging buffer.
    int download_async(double *hssoa, uint32_t host_cap, uint32_t *size) override
    {
        if (n_real_ > host_cap) return fail(ICEMPM_E_CAPACITY, "host buffer capacity is smaller than the point count");
        int rc = ensure_stage();
        if (rc) return rc;
        if (!copy_stream_) {
            ICEMPM_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
            ICEMPM_CUDA(cudaEventCreateWithFlags(&ev_staged_, cudaEventDisableTiming));
            ICEMPM_CUDA(cudaEventCreateWithFlags(&ev_copied_, cudaEventDisableTiming));
        }
        rc = stage_free();
        if (rc) return rc;
        if (n_ > 0) {
            k_download<Real><<<(n_ + 255) / 256, 256, 0, stream_>>>(pts_[par_], (int)n_, stage_, n_real_);
            ICEMPM_CUDA(cudaGetLastError());
            launches_++;
            ICEMPM_CUDA(cudaEventRecord(ev_staged_, stream_));
            ICEMPM_CUDA(cudaStreamWaitEvent(copy_stream_, ev_staged_, 0));
            ICEMPM_CUDA(cudaMemcpy2DAsync(hssoa, (size_t)host_cap * sizeof(double), stage_, (size_t)n_real_ * sizeof(double),
                                          (size_t)n_real_ * sizeof(double), ICEMPM_N_PTS_ARRAYS, cudaMemcpyDeviceToHost,
                                          copy_stream_));
            ICEMPM_CUDA(cudaEventRecord(ev_copied_, copy_stream_));
            copy_pending_ = true;
        }
        if (size) *size = n_real_;
        return 0;
    }
    int download_wait() override
    {
        if (copy_pending_) {
            ICEMPM_CUDA(cudaEventSynchronize(ev_copied_));
            copy_pending_ = false;
        }
        return 0;
    }
    // the compute stream waits for a copy that still reads the staging buffer
    int stage_free()
    {
        if (copy_pending_) ICEMPM_CUDA(cudaStreamWaitEvent(stream_, ev_copied_, 0));
        return 0;
    }

    int update_constants(const icempm_simparams_t &p) override
    {
        const uint32_t zero = 0;
        ICEMPM_CUDA(cudaMemcpyAsync(&st_->err, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return set_params(p, -1.0);
    }

    // ---------------------------------------------------------------- step
    void launch_update()
    {
        constexpr int NPT = ICEMPM_UPDATE_NPT;
        const unsigned nb = (unsigned)(((G_ + NPT - 1) / NPT + 255) / 256);
        if (opts_.forcing == ICEMPM_FORCING_EXTENDED)
            k_grid_update<Real, Acc, true, NPT><<<nb, 256, 0, stream_>>>(kp_, grid(), st_, (long long)G_);
        else
            k_grid_update<Real, Acc, false, NPT><<<nb, 256, 0, stream_>>>(kp_, grid(), st_, (long long)G_);
        launches_++;
    }

    void launch_fused()
    {
        const int nchunks = (int)(((size_t)n_ + CH - 1) / CH);
        const unsigned nb = (unsigned)(ICEMPM_FUSED_PERSIST ? std::min(nchunks, fused_ctas_) : nchunks);
        bool learned = false;
        if constexpr (sizeof(Real) == 4) {
            if (kp_.mlp && learned_ctas_ > 0) {
                const unsigned lnb = (unsigned)(ICEMPM_FUSED_PERSIST ? std::min(nchunks, learned_ctas_) : nchunks);
                k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_LEARNED>
                    <<<lnb, BT, fused_smem_bytes<FusedSmem, BT, FUSED_LEARNED>(), stream_>>>(kp_, pts_[par_], grid(), st_,
                                                                                          (int)n_, nchunks);
                learned = true;
            }
        }
        if (learned) {
        } else if (kp_.harvest)
            k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_HARVEST>
                <<<nb, BT, sizeof(FusedSmem), stream_>>>(kp_, pts_[par_], grid(), st_, (int)n_, nchunks);
        else
            k_g2p_p2g<Real, Acc, BT, PPT, CAP, STAGES, FUSED_PLAIN>
                <<<nb, BT, sizeof(FusedSmem), stream_>>>(kp_, pts_[par_], grid(), st_, (int)n_, nchunks);
        launches_++;
    }
    // The plain FP32 baseline (ICEMPM_VARIANT_TEXTBOOK): three plain kernels
    // per sub-step instead of the fused one (k_textbook_p2g / k_textbook_g2p).
    bool textbook() const { return std::is_same<Acc, float>::value && opts_.variant == ICEMPM_VARIANT_TEXTBOOK; }

    void launch_textbook(bool prime_only)
    {
        if constexpr (std::is_same<Acc, float>::value) {
            const unsigned nb = (unsigned)((n_ + 255) / 256);
            if (!prime_only) {
                k_textbook_g2p<Real><<<nb, 256, 0, stream_>>>(kp_, pts_[par_], grid(), st_, (int)n_);
                launches_++;
            }
            k_textbook_p2g<Real><<<nb, 256, 0, stream_>>>(kp_, pts_[par_], grid(), st_, (int)n_, prime_only ? 0 : 1);
            launches_++;
        }
    }

    int prime()
    {
        ICEMPM_CUDA(cudaMemsetAsync(acc_, 0, 3 * Gp_ * sizeof(Acc), stream_));
        ICEMPM_CUDA(cudaMemsetAsync(&st_->err_pending, 0, sizeof(uint32_t), stream_));
        if (n_ > 0 && textbook()) {
            launch_textbook(true);
            ICEMPM_CUDA(cudaGetLastError());
        } else if (n_ > 0) {
            const unsigned nb = (n_ + BT_P2G - 1) / BT_P2G;
            k_p2g<Real, Acc, BT_P2G, CAP_P2G><<<nb, BT_P2G, 0, stream_>>>(kp_, pts_[par_], grid(), st_, (int)n_);
            launches_++;
            ICEMPM_CUDA(cudaGetLastError());
        }
        primed_ = true;
        return 0;
    }

    int run_chunk_direct(int k)
    {
        for (int s = 0; s < k; s++) {
            launch_update();
            if (n_ > 0) launch_step_points();
        }
        ICEMPM_CUDA(cudaGetLastError());
        return 0;
    }

    void launch_step_points()
    {
        if (textbook()) launch_textbook(false);
        else launch_fused();
    }

    int run_chunk_graph()
    {
        if (!graph_exec_ || graph_n_ != n_ || graph_par_ != par_) {
            invalidate_graphs();
            cudaGraph_t g;
            ICEMPM_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = launches_;
            for (int s = 0; s < GRAPH_STEPS; s++) {
                launch_update();
                if (n_ > 0) launch_step_points();
            }
            graph_launches_ = launches_ - before;
            launches_ = before;
            cudaError_t e = cudaStreamEndCapture(stream_, &g);
            if (e != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&graph_exec_, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) { graph_exec_ = nullptr; return fail(ICEMPM_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)); }
            graph_n_ = n_; graph_par_ = par_;
        }
        ICEMPM_CUDA(cudaGraphLaunch(graph_exec_, stream_));
        launches_ += graph_launches_;
        return 0;
    }

    int step(int nsteps, int first_step) override
    {
        if (nsteps < 0) return fail(ICEMPM_E_ARG, "nsteps < 0");
        ICEMPM_CUDA(cudaEventRecord(ev0_, stream_));
        k_set_step<<<1, 1, 0, stream_>>>(st_, first_step, 1, nsteps);
        launches_++;
        int rc = 0;
        if (!primed_) { rc = prime(); if (rc) return rc; }
        float sort_ms = 0;
        int remaining = nsteps;
        while (remaining > 0) {
            if (opts_.sort_every > 0 && steps_since_sort_ >= opts_.sort_every && n_ > 0) {
                ICEMPM_CUDA(cudaEventRecord(evs_[0], stream_));
                rc = locality_sort();
                if (rc) return rc;
                ICEMPM_CUDA(cudaEventRecord(evs_[1], stream_));
                ICEMPM_CUDA(cudaEventSynchronize(evs_[1]));
                float ms = 0;
                cudaEventElapsedTime(&ms, evs_[0], evs_[1]);
                sort_ms += ms;
            }
            int chunk = remaining;
            if (opts_.sort_every > 0) chunk = std::min(chunk, std::max(1, opts_.sort_every - steps_since_sort_));
            if (opts_.use_graphs && chunk >= GRAPH_STEPS) {
                chunk = GRAPH_STEPS;
                rc = run_chunk_graph();
            } else {
                rc = run_chunk_direct(chunk);
            }
            if (rc) return rc;
            remaining -= chunk;
            steps_since_sort_ += chunk;
        }
        ICEMPM_CUDA(cudaEventRecord(ev1_, stream_));
        last_sort_ms_ = sort_ms;
        timed_ = true;
        return 0;
    }

    // Device time between the event pair around the last icempm_step or
    // icempm_phase_times call, and the locality-sort time inside it.
    // Sort cadence on the live scene, which therefore advances (step indices
    // from first_step): trial_steps sub-steps in the current order, one
    // locality sort (timed), trial_steps sub-steps in the sorted order; a
    // cadence k in {100, 400} is kept when sorted ms/step + sort ms / k beats
    // the current order's ms/step, else 0 (sort only at upload and
    // compaction).  The choice becomes the context's sort_every.
    int tune_sort(int trial_steps, int first_step, int32_t *sort_every) override
    {
        if (trial_steps <= 0) return fail(ICEMPM_E_ARG, "trial_steps must be > 0");
        opts_.sort_every = 0;
        int rc = step(trial_steps, first_step);
        if (rc) return rc;
        float ms[4];
        rc = timings(ms);
        if (rc) return rc;
        const float unsorted = ms[0] / (float)trial_steps;
        ICEMPM_CUDA(cudaEventRecord(evs_[0], stream_));
        rc = locality_sort();
        if (rc) return rc;
        ICEMPM_CUDA(cudaEventRecord(evs_[1], stream_));
        ICEMPM_CUDA(cudaEventSynchronize(evs_[1]));
        float sort_ms = 0;
        ICEMPM_CUDA(cudaEventElapsedTime(&sort_ms, evs_[0], evs_[1]));
        rc = step(trial_steps, first_step + trial_steps);
        if (rc) return rc;
        rc = timings(ms);
        if (rc) return rc;
        const float sorted = ms[0] / (float)trial_steps;
        float best = unsorted;
        int k_best = 0;
        for (int k : {100, 400}) {
            const float est = sorted + sort_ms / (float)k;
            if (est < best) { best = est; k_best = k; }
        }
        opts_.sort_every = k_best;
        steps_since_sort_ = trial_steps;
        if (sort_every) *sort_every = k_best;
        return 0;
    }

    int timings(float ms[4]) override
    {
        ms[0] = ms[1] = ms[2] = ms[3] = 0;
        if (timed_) {
            ICEMPM_CUDA(cudaEventSynchronize(ev1_));
            ICEMPM_CUDA(cudaEventElapsedTime(&ms[0], ev0_, ev1_));
        }
        ms[3] = last_sort_ms_;
        return 0;
    }

    int phase_times(int nsteps, float *update_ms, float *fused_ms) override
    {
        // time nsteps steps launched directly, accumulating per-kernel event pairs
        if (!primed_) { int rc = prime(); if (rc) return rc; }
        k_set_step<<<1, 1, 0, stream_>>>(st_, -1, 0, nsteps);
        launches_++;
        std::vector<cudaEvent_t> ev(3 * nsteps);
        for (auto &e : ev) ICEMPM_CUDA(cudaEventCreate(&e));
        ICEMPM_CUDA(cudaEventRecord(ev0_, stream_));
        for (int s = 0; s < nsteps; s++) {
            cudaEventRecord(ev[3 * s], stream_);
            launch_update();
            cudaEventRecord(ev[3 * s + 1], stream_);
            if (n_ > 0) launch_step_points();
            cudaEventRecord(ev[3 * s + 2], stream_);
        }
        ICEMPM_CUDA(cudaEventRecord(ev1_, stream_));
        ICEMPM_CUDA(cudaGetLastError());
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        timed_ = true;
        last_sort_ms_ = 0;
        float u = 0, f = 0;
        for (int s = 0; s < nsteps; s++) {
            float a = 0, b = 0;
            cudaEventElapsedTime(&a, ev[3 * s], ev[3 * s + 1]);
            cudaEventElapsedTime(&b, ev[3 * s + 1], ev[3 * s + 2]);
            u += a; f += b;
        }
        for (auto &e : ev) cudaEventDestroy(e);
        *update_ms = u; *fused_ms = f;
        steps_since_sort_ += nsteps;
        return 0;
    }

    int status(uint32_t *err, int32_t *dis) override
    {
        DevStatus s;
        ICEMPM_CUDA(cudaMemcpyAsync(&s, st_, sizeof(s), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        if (err) *err = s.err;
        if (dis) *dis = s.disabled;
        return 0;
    }

    int clear_forces() override
    {
        ICEMPM_CUDA(cudaMemsetAsync(force_, 0, G_ * sizeof(double2), stream_));
        return 0;
    }

    // Forces divided by elapsed * dt on the device, into the reference's
    // [fx block, fy block] layout, then one copy into the caller's buffer.
    int forces(double *fxfy, int elapsed) override
    {
        if (!force_out_) ICEMPM_CUDA(cudaMalloc(&force_out_, 2 * G_ * sizeof(double)));
        const double div = (double)elapsed * prms_.InitialTimeStep;
        const unsigned nb = (unsigned)((G_ + 255) / 256);
        k_forces_out<<<nb, 256, 0, stream_>>>(force_, (long long)G_, div, force_out_);
        ICEMPM_CUDA(cudaGetLastError());
        launches_++;
        ICEMPM_CUDA(cudaMemcpyAsync(fxfy, force_out_, 2 * G_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return 0;
    }

    // Sort by the tiled locality key into the other parity, in the fused
    // kernel's interleaved order (host slots unchanged).  Each cell's run of
    // enabled points is padded to a multiple of four with placeholders when
    // the padded order fits the arrays; the placeholders of an earlier padding
    // are dropped first (they sort last).
    int locality_sort()
    {
        if (n_ == 0) return 0;
        const unsigned nb = (n_ + 255) / 256;
        uint32_t *k32in = (uint32_t *)keys_[0], *k32out = (uint32_t *)keys_[1];
        k_keys_tiled<<<nb, 256, 0, stream_>>>(pts_[par_].K, pts_[par_].slot, (int)n_, tile_, k32in, vals_[0]);
        launches_++;
        size_t tb = sort_tmp_bytes_;
        ICEMPM_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp_, tb, k32in, k32out, vals_[0], vals_[1], (int)n_, 0, 32, stream_));
        launches_ += 4;
        k_key_bounds<<<(n_ + 256) / 256, 256, 0, stream_>>>(k32out, (int)n_, aux_);
        launches_++;
        int bounds[2] = {0, 0};
        ICEMPM_CUDA(cudaMemcpyAsync(bounds, aux_, sizeof(bounds), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        const uint32_t n_en = (uint32_t)bounds[0], n_real = (uint32_t)bounds[1];
        // run bookkeeping in the free halves of the key buffers and vals_[0]
        uint32_t *flags = k32in, *run_id = k32in + nc_, *begin = k32out + nc_, *padded = vals_[0], *pstart = runs_;
        uint32_t n_pad = n_real, n_pad_en = n_en;
        int runs = 0;
        if (n_en > 0) {
            const unsigned nbe = (n_en + 255) / 256;
            k_run_flags<<<nbe, 256, 0, stream_>>>(k32out, (int)n_en, flags);
            tb = sort_tmp_bytes_;
            ICEMPM_CUDA(cub::DeviceScan::InclusiveSum(sort_tmp_, tb, flags, run_id, (int)n_en, stream_));
            k_run_begin<<<nbe, 256, 0, stream_>>>(run_id, (int)n_en, begin);
            launches_ += 3;
            uint32_t r = 0;
            ICEMPM_CUDA(cudaMemcpyAsync(&r, run_id + n_en - 1, sizeof(r), cudaMemcpyDeviceToHost, stream_));
            ICEMPM_CUDA(cudaStreamSynchronize(stream_));
            runs = (int)r;
            k_run_padded<<<(runs + 255) / 256, 256, 0, stream_>>>(begin, runs, (int)n_en, padded);
            tb = sort_tmp_bytes_;
            ICEMPM_CUDA(cub::DeviceScan::ExclusiveSum(sort_tmp_, tb, padded, pstart, runs, stream_));
            launches_ += 2;
            uint32_t last[2] = {0, 0};
            ICEMPM_CUDA(cudaMemcpyAsync(&last[0], pstart + runs - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
            ICEMPM_CUDA(cudaMemcpyAsync(&last[1], padded + runs - 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
            ICEMPM_CUDA(cudaStreamSynchronize(stream_));
            n_pad_en = last[0] + last[1];
            n_pad = n_pad_en + (n_real - n_en);
            if ((size_t)n_pad > nc_) {   // does not fit: unpadded order
                n_pad = n_real; n_pad_en = n_en; runs = 0;
            }
        }
        if (runs > 0) {
            k_gather_padded<Real><<<(n_real + 255) / 256, 256, 0, stream_>>>(
                pts_[par_], pts_[1 - par_], vals_[1], (int)n_real, n_en, n_pad_en, n_pad, run_id, begin, pstart, PPT);
            k_fill_placeholders<Real><<<(runs + 255) / 256, 256, 0, stream_>>>(pts_[1 - par_], runs, n_en, n_pad, begin,
                                                                              pstart, padded, PPT);
            launches_ += 2;
        } else if (n_real > 0) {
            k_gather<Real><<<(n_real + 255) / 256, 256, 0, stream_>>>(pts_[par_], pts_[1 - par_], vals_[1],
                                                                     (int)n_real, 0, PPT);
            launches_++;
        }
        ICEMPM_CUDA(cudaGetLastError());
        par_ = 1 - par_;
        n_ = n_pad;
        n_real_ = n_real;
        steps_since_sort_ = 0;
        invalidate_graphs();
        return 0;
    }

    // RemoveDisabledAndSort (host_side_soa.cpp:36-47) on the device.
    int sort_compact() override
    {
        if (n_ > 0) {
            const unsigned nb = (n_ + 255) / 256;
            k_keys_reference<<<nb, 256, 0, stream_>>>(pts_[par_].K, pts_[par_].slot, (int)n_, gy_, keys_[0], vals_[0]);
            launches_++;
            size_t tb = sort_tmp_bytes_;
            ICEMPM_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp_, tb, keys_[0], keys_[1], vals_[0], vals_[1], (int)n_, 0, 64, stream_));
            launches_ += 4;
            k_gather<Real><<<nb, 256, 0, stream_>>>(pts_[par_], pts_[1 - par_], vals_[1], (int)n_, 1, 0);
            k_count_active<<<nb, 256, 0, stream_>>>(keys_[1], (int)n_, st_);
            launches_ += 2;
            ICEMPM_CUDA(cudaGetLastError());
            par_ = 1 - par_;
            DevStatus s;
            ICEMPM_CUDA(cudaMemcpyAsync(&s, st_, sizeof(s), cudaMemcpyDeviceToHost, stream_));
            ICEMPM_CUDA(cudaStreamSynchronize(stream_));
            n_ = (uint32_t)s.n_active;
            n_real_ = n_;
        }
        const int32_t zero = 0;
        ICEMPM_CUDA(cudaMemcpyAsync(&st_->disabled, &zero, sizeof(zero), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        primed_ = false;
        invalidate_graphs();
        return locality_sort();
    }

    // Return-map pairs of the following steps (see HarvestBuf), at most
    // `capacity` records, points with (index + step) % stride == 0.
    int harvest_begin(uint32_t capacity, int stride) override
    {
        if (capacity == 0 || stride < 1) return fail(ICEMPM_E_ARG, "capacity must be > 0 and stride >= 1");
        int rc = harvest_free();
        if (rc) return rc;
        ICEMPM_CUDA(cudaMalloc(&harvest_rec_, 2 * (size_t)capacity * sizeof(float4)));
        ICEMPM_CUDA(cudaMalloc(&harvest_, sizeof(HarvestBuf)));
        HarvestBuf h{0u, capacity, harvest_rec_};
        ICEMPM_CUDA(cudaMemcpyAsync(harvest_, &h, sizeof(h), cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        harvest_stride_ = stride;
        kp_.harvest = harvest_;
        kp_.harvest_stride = stride;
        invalidate_graphs();
        return 0;
    }

    // Copies the records (8 floats each) out, reports how many were offered
    // (*count may exceed the capacity), and stops recording.
    int harvest_end(float *records, uint32_t host_cap, uint32_t *count) override
    {
        if (!harvest_) return fail(ICEMPM_E_STATE, "no harvest in progress");
        HarvestBuf h{};
        ICEMPM_CUDA(cudaMemcpyAsync(&h, harvest_, sizeof(h), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        const uint32_t m = std::min(std::min(h.count, h.cap), host_cap);
        if (records && m)
            ICEMPM_CUDA(cudaMemcpy(records, harvest_rec_, 2 * (size_t)m * sizeof(float4), cudaMemcpyDeviceToHost));
        if (count) *count = h.count;
        return harvest_free();
    }

    // Saved-frame grid arrays (frame.cuh) into the caller's host buffers.
    int prepare_frame(const uint32_t *colors, uint32_t ncolors, int elapsed, icempm_frame_t *out) override
    {
        if (elapsed <= 0) return fail(ICEMPM_E_ARG, "elapsed_steps must be > 0");
        if (!frame_mem_) {
            const size_t bytes = G_ * (3 * sizeof(float4) + kFrameChannels * sizeof(float) + 5) +
                                 2 * ICEMPM_MAX_REGIONS * sizeof(float) + 256;
            ICEMPM_CUDA(cudaMalloc(&frame_mem_, bytes));
            char *b = (char *)frame_mem_;
            frame_.acc = (float4 *)b; b += G_ * 3 * sizeof(float4);
            frame_.region_force = (float *)b; b += 2 * ICEMPM_MAX_REGIONS * sizeof(float);
            for (int c = 0; c < kFrameChannels; c++) { frame_.ch[c] = (float *)b; b += G_ * sizeof(float); }
            frame_.rgb = (uint8_t *)b; b += 3 * G_;
            frame_.mask = (uint8_t *)b; b += G_;
            frame_.count8 = (uint8_t *)b;
        }
        if (colors && ncolors) {
            if (ncolors > colors_cap_) {
                cudaFree(colors_);
                colors_ = nullptr;
                ICEMPM_CUDA(cudaMalloc(&colors_, (size_t)ncolors * sizeof(uint32_t)));
                colors_cap_ = ncolors;
            }
            ICEMPM_CUDA(cudaMemcpyAsync(colors_, colors, (size_t)ncolors * sizeof(uint32_t), cudaMemcpyHostToDevice,
                                        stream_));
        }
        const size_t zero_bytes = G_ * 3 * sizeof(float4) + 2 * ICEMPM_MAX_REGIONS * sizeof(float);
        ICEMPM_CUDA(cudaMemsetAsync(frame_mem_, 0, zero_bytes, stream_));
        if (n_ > 0) {
            k_frame_scatter<Real><<<(n_ + 1023) / 1024, 256, 0, stream_>>>(
                pts_[par_], (int)n_, gx_, gy_, Real(prms_.ParticleMass), (colors && ncolors) ? colors_ : nullptr,
                (colors && ncolors) ? ncolors : 0u, frame_);
            launches_++;
        }
        k_frame_finish<<<(unsigned)((G_ + 255) / 256), 256, 0, stream_>>>(
            frame_, status_, force_, (double)elapsed * prms_.InitialTimeStep, (long long)G_);
        launches_++;
        ICEMPM_CUDA(cudaGetLastError());
        float *const dst[kFrameChannels] = {out->point_density, out->mass, out->vx, out->vy, out->Jpinv,
                                            out->P, out->Q, out->r, out->g, out->b};
        for (int c = 0; c < kFrameChannels; c++)
            if (dst[c]) ICEMPM_CUDA(cudaMemcpyAsync(dst[c], frame_.ch[c], G_ * sizeof(float), cudaMemcpyDeviceToHost, stream_));
        if (out->rgb) ICEMPM_CUDA(cudaMemcpyAsync(out->rgb, frame_.rgb, 3 * G_, cudaMemcpyDeviceToHost, stream_));
        if (out->mass_mask) ICEMPM_CUDA(cudaMemcpyAsync(out->mass_mask, frame_.mask, G_, cudaMemcpyDeviceToHost, stream_));
        if (out->count) ICEMPM_CUDA(cudaMemcpyAsync(out->count, frame_.count8, G_, cudaMemcpyDeviceToHost, stream_));
        if (out->forces_per_region)
            ICEMPM_CUDA(cudaMemcpyAsync(out->forces_per_region, frame_.region_force,
                                        2 * ICEMPM_MAX_REGIONS * sizeof(float), cudaMemcpyDeviceToHost, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return 0;
    }

    uint32_t count() const override { return n_real_; }
    int device() const { return opts_.device; }
    cudaStream_t stream() const override { return stream_; }
    uint64_t launches() const override { return launches_; }
    double fixed_scale_m() const override { return kp_.scale_m; }
    double fixed_scale_p() const override { return kp_.scale_p; }

private:
    // The learned return map on the step path (FP32 state only): the FP32
    // parameters and normalisation (device pointers) are packed for the
    // fused kernel, whose projections onto the yield surface then go to the
    // network, with the exact map as fallback above `tol`.  Null params: off.
    int set_learned_map(const float *d_params, const float *d_norm, float tol) override
    {
        if (sizeof(Real) != 4 || textbook())
            return fail(ICEMPM_E_UNSUPPORTED, "the learned return map needs the fused FP32-state variants");
        if (!d_params) {
            kp_.mlp = nullptr;
            invalidate_graphs();
            return 0;
        }
        if (!d_norm || !(tol > 0.0f)) return fail(ICEMPM_E_ARG, "norm must be given and tol > 0");
        if (learned_ctas_ < 1) return fail(ICEMPM_E_UNSUPPORTED, "the learned fused kernel does not fit on one SM");
        if (!mlp_packed_) ICEMPM_CUDA(cudaMalloc(&mlp_packed_, mlp_packed_bytes()));
        if (!mlp_counts_) ICEMPM_CUDA(cudaMalloc(&mlp_counts_, 2 * sizeof(unsigned long long)));
        int rc = mlp_pack(d_params, d_norm, mlp_packed_, stream_);
        if (rc) return rc;
        ICEMPM_CUDA(cudaMemsetAsync(mlp_counts_, 0, 2 * sizeof(unsigned long long), stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        kp_.mlp = static_cast<const mlp::Packed *>(mlp_packed_);
        kp_.mlp_tol = tol;
        kp_.mlp_counts = mlp_counts_;
        invalidate_graphs();
        return 0;
    }

    int learned_counts(uint64_t *kept, uint64_t *fallbacks) override
    {
        unsigned long long h[2] = {0, 0};
        if (mlp_counts_) {
            ICEMPM_CUDA(cudaMemcpyAsync(h, mlp_counts_, sizeof(h), cudaMemcpyDeviceToHost, stream_));
            ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        }
        if (kept) *kept = h[0];
        if (fallbacks) *fallbacks = h[1];
        return 0;
    }

    int harvest_free()
    {
        if (stream_) ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        cudaFree(harvest_);
        cudaFree(harvest_rec_);
        harvest_ = nullptr;
        harvest_rec_ = nullptr;
        kp_.harvest = nullptr;
        invalidate_graphs();
        return 0;
    }
    Grid<Real, Acc> grid() const
    {
        Grid<Real, Acc> g;
        g.acc.m = acc_; g.acc.px = acc_ + Gp_; g.acc.py = acc_ + 2 * Gp_; g.vel = vel_; g.cur = cur_; g.frc = frc_; g.status = status_; g.force = force_;
        return g;
    }
    void invalidate_graphs()
    {
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    }
    void release()
    {
        if (copy_stream_) cudaStreamSynchronize(copy_stream_);
        if (stream_) cudaStreamSynchronize(stream_);
        invalidate_graphs();
        cudaFree(pts_mem_); cudaFree(acc_); cudaFree(vel_); cudaFree(cur_); cudaFree(frc_); cudaFree(status_);
        cudaFree(force_); cudaFree(st_); cudaFree(stage_); cudaFree(keys_[0]); cudaFree(keys_[1]);
        cudaFree(vals_[0]); cudaFree(vals_[1]); cudaFree(sort_tmp_); cudaFree(harvest_); cudaFree(harvest_rec_); cudaFree(mlp_packed_); cudaFree(mlp_counts_); cudaFree(frame_mem_); cudaFree(colors_); cudaFree(runs_); cudaFree(aux_);
        cudaFree(flow_ab_); cudaFree((void *)wind_.w);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        for (auto &e : evs_) if (e) cudaEventDestroy(e);
        if (stream_) cudaStreamDestroy(stream_);
        stream_ = nullptr;
        if (ev_staged_) cudaEventDestroy(ev_staged_);
        if (ev_copied_) cudaEventDestroy(ev_copied_);
        if (copy_stream_) cudaStreamDestroy(copy_stream_);
        copy_stream_ = nullptr;
        cudaFree(force_out_);
    }

    icempm_simparams_t prms_{};
    icempm_options_t opts_{};
    int gx_ = 0, gy_ = 0;
    size_t G_ = 0;
    uint32_t cap_ = 0;
    uint32_t n_ = 0;        // entries of the point arrays the kernels walk (points + placeholders)
    uint32_t n_real_ = 0;   // points (host slots)
    size_t nc_ = 0;         // allocated entries per point array
    double max_thick_ = 1.0;
    void *frame_mem_ = nullptr;       // saved-frame grid arrays (allocated on first use)
    FrameOut frame_{};
    uint32_t *colors_ = nullptr;
    uint32_t colors_cap_ = 0;
    HarvestBuf *harvest_ = nullptr;   // device record of return-map pairs (null: off)
    float4 *harvest_rec_ = nullptr;
    int harvest_stride_ = 1;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr, evs_[3] = {nullptr, nullptr, nullptr};
    void *pts_mem_ = nullptr;
    Pts<Real> pts_[2]{};
    int par_ = 0;
    Acc *acc_ = nullptr;   // mass, x- and y-momentum arrays of G_ each, Gp_ apart
    size_t Gp_ = 0;
    V2<Real> *vel_ = nullptr, *cur_ = nullptr;
    V4<Real> *frc_ = nullptr;
    double *flow_ab_ = nullptr;   // current frames a, b (2 G_ doubles each), null: static current
    WindGrid wind_{};             // wind frames, null samples: static wind
    size_t wind_cap_ = 0;
    uint8_t *status_ = nullptr;
    double2 *force_ = nullptr;
    DevStatus *st_ = nullptr;
    double *stage_ = nullptr;
    double *force_out_ = nullptr;          // boundary forces / (elapsed dt), fx block then fy block
    cudaStream_t copy_stream_ = nullptr;   // device-to-host copies of icempm_download_points_async
    cudaEvent_t ev_staged_ = nullptr, ev_copied_ = nullptr;
    bool copy_pending_ = false;
    uint64_t *keys_[2] = {nullptr, nullptr};
    uint32_t *vals_[2] = {nullptr, nullptr};
    uint32_t *runs_ = nullptr;   // padded run starts of the locality order
    int *aux_ = nullptr;         // small device results read back by the host
    void *sort_tmp_ = nullptr;
    size_t sort_tmp_bytes_ = 0;
    TileKey tile_{8, 8, 1};
    KParams<Real> kp_{};
    void *mlp_packed_ = nullptr;                  // the learned map's packed network
    unsigned long long *mlp_counts_ = nullptr;    // its answers kept / exact fallbacks
    int learned_ctas_ = 0;                        // persistent grid of the learned instance
    uint32_t tx_extra_ = 0;
    unsigned long long wait_ns_ = kWaitLimitNs;
    bool primed_ = false, timed_ = false;
    int fused_ctas_ = 1;
    int steps_since_sort_ = 0;
    float last_sort_ms_ = 0;
    cudaGraphExec_t graph_exec_ = nullptr;
    uint32_t graph_n_ = 0;
    int graph_par_ = -1;
    uint64_t graph_launches_ = 0;
    uint64_t launches_ = 0;
};

}  // namespace icempm
