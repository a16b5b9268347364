// batch.cuh -- ensembles: many independent scenes advanced by one launch of
// each kernel per sub-step (k_grid_update_batch, k_g2p_p2g_batch), captured
// in CUDA graphs.  Each scene stays an ordinary context (upload, download,
// status, sort and compaction go through it); the batch holds a device table
// of the scenes' descriptors and its own sub-step counter.  Instantiated once
// per variant beside EngineT.
#pragma once
#include <algorithm>
#include <vector>

#include "engine_host.cuh"

namespace icempm {

template <class Real, class Acc>
class BatchT final : public Batch {
    using E = EngineT<Real, Acc>;
    static constexpr int BT = E::BT, PPT = E::PPT, CH = E::CH;
    // shapes of the batched fused kernel the tuner chooses from: tile nodes
    // (0: no shared tile, node sums straight to the global accumulators) x stages
    static constexpr int NSHAPES = 4;
    static constexpr int SHAPE_TILE[NSHAPES] = {0, 0, 512, 1024};
    static constexpr int SHAPE_STAGES[NSHAPES] = {2, 1, 1, 1};

    template <int CAPX, int ST> using Smem = ChunkSmem<Real, Acc, BT, PPT, CAPX, ST>;

public:
    ~BatchT() override { release(); }

    int init(std::vector<E *> eng)
    {
        eng_ = std::move(eng);
        device_ = eng_[0]->device();
        ICEMPM_CUDA(cudaSetDevice(device_));
        ICEMPM_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        ICEMPM_CUDA(cudaEventCreate(&ev0_));
        ICEMPM_CUDA(cudaEventCreate(&ev1_));
        ICEMPM_CUDA(cudaMalloc(&bst_, sizeof(DevStatus)));
        ICEMPM_CUDA(cudaMemsetAsync(bst_, 0, sizeof(DevStatus), stream_));
        ICEMPM_CUDA(cudaMalloc(&d_scenes_, eng_.size() * sizeof(SceneDesc<Real, Acc>)));
        int sms = 0;
        ICEMPM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
        int rc = setup_shape<0, 2>(0, sms);
        if (!rc) rc = setup_shape<0, 1>(1, sms);
        if (!rc) rc = setup_shape<512, 1>(2, sms);
        if (!rc) rc = setup_shape<1024, 1>(3, sms);
        if (rc) return rc;
        if (ctas_[0] < 1) return fail(ICEMPM_E_UNSUPPORTED, "batched fused kernel does not fit on one SM");
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        return 0;
    }

    int step(int nsteps, int first_step) override
    {
        if (nsteps < 0) return fail(ICEMPM_E_ARG, "nsteps < 0");
        ICEMPM_CUDA(cudaSetDevice(device_));
        int rc = prepare();
        if (rc) return rc;
        // capture and instantiate the graph before the timed region starts
        if (tune_.graph_steps > 0 && nsteps >= tune_.graph_steps) {
            rc = build_graph();
            if (rc) return rc;
        }
        ICEMPM_CUDA(cudaEventRecord(ev0_, stream_));
        k_set_step<<<1, 1, 0, stream_>>>(bst_, first_step, 1, nsteps);
        launches_++;
        int remaining = nsteps;
        while (remaining > 0) {
            if (tune_.sort_every > 0 && since_sort_ >= tune_.sort_every) {
                rc = sort_all();
                if (rc) return rc;
            }
            int chunk = remaining;
            if (tune_.sort_every > 0) chunk = std::min(chunk, std::max(1, tune_.sort_every - since_sort_));
            if (tune_.graph_steps > 0 && chunk >= tune_.graph_steps) {
                chunk = tune_.graph_steps;
                rc = run_graph();
            } else {
                for (int s = 0; s < chunk; s++) launch_step();
                ICEMPM_CUDA(cudaGetLastError());
            }
            if (rc) return rc;
            remaining -= chunk;
            since_sort_ += chunk;
        }
        ICEMPM_CUDA(cudaEventRecord(ev1_, stream_));
        ICEMPM_CUDA(cudaEventSynchronize(ev1_));   // the scenes' own streams may use the results next
        timed_ = true;
        return 0;
    }

    int timings(float ms[4]) override
    {
        ms[0] = ms[1] = ms[2] = ms[3] = 0;
        if (timed_) ICEMPM_CUDA(cudaEventElapsedTime(&ms[0], ev0_, ev1_));
        return 0;
    }

    // Chooses the kernel shape (tile nodes x stages) and the sort cadence on
    // the live scenes, which therefore advance (step indices continue from
    // first_step).  Each shape is timed over `trial_steps` sub-steps in CUDA
    // graphs of 50; then all scenes are sorted once (timed) and the best
    // shape is timed again, so a cadence k costs its sort amortised over k
    // sub-steps and earns the sorted order's speed: cadence k is kept when
    // sorted_per_step + sort_ms / k beats the unsorted time.
    int autotune(int trial_steps, int first_step, icempm_batch_tuning_t *out) override
    {
        if (trial_steps <= 0) return fail(ICEMPM_E_ARG, "trial_steps must be > 0");
        icempm_batch_tuning_t t = tune_;
        t.sort_every = 0;
        t.graph_steps = 50;
        int step_idx = first_step, best_shape = -1;
        float best_ms = 1e30f;
        for (int shape = 0; shape < NSHAPES; shape++) {
            if (ctas_[shape] < 1) continue;
            t.tile_nodes = SHAPE_TILE[shape];
            t.stages = SHAPE_STAGES[shape];
            int rc = set_tuning(&t);
            if (!rc) rc = step(trial_steps, step_idx);
            if (rc) return rc;
            step_idx += trial_steps;
            float ms[4];
            timings(ms);
            const float per = ms[0] / (float)trial_steps;
            if (per < best_ms) { best_ms = per; best_shape = shape; }
        }
        t.tile_nodes = SHAPE_TILE[best_shape];
        t.stages = SHAPE_STAGES[best_shape];
        int rc = set_tuning(&t);
        if (rc) return rc;
        // sorted order: time one sort of every scene, then the best shape again
        ICEMPM_CUDA(cudaEventRecord(ev0_, stream_));
        rc = sort_all();
        if (rc) return rc;
        ICEMPM_CUDA(cudaEventRecord(ev1_, stream_));
        ICEMPM_CUDA(cudaEventSynchronize(ev1_));
        float sort_ms = 0;
        ICEMPM_CUDA(cudaEventElapsedTime(&sort_ms, ev0_, ev1_));
        rc = step(trial_steps, step_idx);
        if (rc) return rc;
        float ms[4];
        timings(ms);
        const float sorted_per = ms[0] / (float)trial_steps;
        const int cadences[2] = {100, 400};
        float chosen = best_ms;
        for (int k : cadences) {
            const float est = sorted_per + sort_ms / (float)k;
            if (est < chosen) { chosen = est; t.sort_every = k; }
        }
        t.ms_per_step = chosen;
        rc = set_tuning(&t);
        if (rc) return rc;
        if (out) *out = tune_;
        return 0;
    }

    int set_tuning(const icempm_batch_tuning_t *t) override
    {
        int shape = -1;
        for (int s = 0; s < NSHAPES; s++)
            if (SHAPE_TILE[s] == t->tile_nodes && SHAPE_STAGES[s] == t->stages) shape = s;
        if (shape < 0) return fail(ICEMPM_E_UNSUPPORTED, "tile_nodes/stages: 0/2, 0/1, 512/1 or 1024/1");
        if (ctas_[shape] < 1) return fail(ICEMPM_E_UNSUPPORTED, "that kernel shape does not fit on this device");
        if (t->sort_every < 0 || t->graph_steps < 0) return fail(ICEMPM_E_ARG, "negative cadence");
        if (shape != shape_ || t->graph_steps != tune_.graph_steps) invalidate_graph();
        shape_ = shape;
        tune_ = *t;
        return 0;
    }

    int get_tuning(icempm_batch_tuning_t *t) const override
    {
        *t = tune_;
        return 0;
    }

    uint64_t launches() const override { return launches_; }

private:
    template <int CAPX, int ST> int setup_shape(int shape, int sms)
    {
        auto kern = k_g2p_p2g_batch<Real, Acc, BT, PPT, CAPX, ST>;
        const int bytes = (int)sizeof(Smem<CAPX, ST>);
        ICEMPM_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        int per_sm = 0;
        ICEMPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT, bytes));
        ctas_[shape] = per_sm * sms;
        return 0;
    }

    // every scene primed and idle on its own stream; descriptor tables current
    int prepare()
    {
        for (E *e : eng_) {
            if (!e->primed_) { int rc = e->prime(); if (rc) return rc; }
            ICEMPM_CUDA(cudaStreamSynchronize(e->stream_));
        }
        return build_tables();
    }

    int build_tables()
    {
        std::vector<SceneDesc<Real, Acc>> d(eng_.size());
        chunk_scene_.clear();
        block_scene_.clear();
        for (size_t i = 0; i < eng_.size(); i++) {
            E *e = eng_[i];
            SceneDesc<Real, Acc> &s = d[i];
            s.kp = e->kp_;
            s.kp.tx_extra = 0;                  // the batch kernel waits for the exact bytes, 1 s at most
            s.kp.wait_ns = kWaitLimitNs;
            s.P = e->pts_[e->par_];
            s.G = e->grid();
            s.st = e->st_;
            s.n = (int)e->n_;
            s.chunk0 = (int)chunk_scene_.size();
            s.nnodes = (long long)e->G_;
            s.block0 = (int)block_scene_.size();
            s.ext = e->opts_.forcing == ICEMPM_FORCING_EXTENDED;
            const size_t nch = ((size_t)e->n_ + CH - 1) / CH;
            chunk_scene_.insert(chunk_scene_.end(), nch, (int)i);
            constexpr size_t BN = 256 * ICEMPM_UPDATE_NPT;   // nodes per block of the batch grid update
            block_scene_.insert(block_scene_.end(), (e->G_ + BN - 1) / BN, (int)i);
        }
        if (chunk_scene_.size() > (size_t)INT32_MAX || block_scene_.size() > (size_t)INT32_MAX)
            return fail(ICEMPM_E_CAPACITY, "batch too large");
        const int nchunks = (int)chunk_scene_.size(), nblocks = (int)block_scene_.size();
        if (nchunks > chunk_cap_) {
            cudaFree(d_chunk_scene_);
            d_chunk_scene_ = nullptr;
            ICEMPM_CUDA(cudaMalloc(&d_chunk_scene_, std::max(nchunks, 1) * sizeof(int)));
            chunk_cap_ = nchunks;
        }
        if (nblocks > block_cap_) {
            cudaFree(d_block_scene_);
            d_block_scene_ = nullptr;
            ICEMPM_CUDA(cudaMalloc(&d_block_scene_, std::max(nblocks, 1) * sizeof(int)));
            block_cap_ = nblocks;
        }
        if (nchunks != nchunks_ || nblocks != nblocks_) invalidate_graph();
        nchunks_ = nchunks;
        nblocks_ = nblocks;
        ICEMPM_CUDA(cudaMemcpyAsync(d_scenes_, d.data(), d.size() * sizeof(d[0]), cudaMemcpyHostToDevice, stream_));
        if (nchunks)
            ICEMPM_CUDA(cudaMemcpyAsync(d_chunk_scene_, chunk_scene_.data(), nchunks * sizeof(int),
                                        cudaMemcpyHostToDevice, stream_));
        if (nblocks)
            ICEMPM_CUDA(cudaMemcpyAsync(d_block_scene_, block_scene_.data(), nblocks * sizeof(int),
                                        cudaMemcpyHostToDevice, stream_));
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));   // the host vectors are pageable and reused
        return 0;
    }

    int sort_all()
    {
        ICEMPM_CUDA(cudaStreamSynchronize(stream_));
        for (E *e : eng_) {
            int rc = e->locality_sort();
            if (rc) return rc;
            ICEMPM_CUDA(cudaStreamSynchronize(e->stream_));
        }
        since_sort_ = 0;
        return build_tables();
    }

    template <int CAPX, int ST> void launch_fused()
    {
        const unsigned nb = (unsigned)std::min(nchunks_, ctas_[shape_]);
        k_g2p_p2g_batch<Real, Acc, BT, PPT, CAPX, ST>
            <<<nb, BT, sizeof(Smem<CAPX, ST>), stream_>>>(d_scenes_, d_chunk_scene_, nchunks_, bst_);
    }

    void launch_step()
    {
        if (nblocks_ > 0)
            k_grid_update_batch<Real, Acc, ICEMPM_UPDATE_NPT><<<nblocks_, 256, 0, stream_>>>(d_scenes_, d_block_scene_, bst_);
        if (nchunks_ > 0) {
            if (shape_ == 0) launch_fused<0, 2>();
            else if (shape_ == 1) launch_fused<0, 1>();
            else if (shape_ == 2) launch_fused<512, 1>();
            else launch_fused<1024, 1>();
        }
        launches_ += 2;
    }

    int build_graph()
    {
        if (!graph_exec_) {
            cudaGraph_t g;
            ICEMPM_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = launches_;
            for (int s = 0; s < tune_.graph_steps; s++) launch_step();
            graph_launches_ = launches_ - before;
            launches_ = before;
            cudaError_t e = cudaStreamEndCapture(stream_, &g);
            if (e != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&graph_exec_, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                graph_exec_ = nullptr;
                return fail(ICEMPM_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
            }
        }
        return 0;
    }

    int run_graph()
    {
        int rc = build_graph();
        if (rc) return rc;
        ICEMPM_CUDA(cudaGraphLaunch(graph_exec_, stream_));
        launches_ += graph_launches_;
        return 0;
    }

    void invalidate_graph()
    {
        if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    }

    void release()
    {
        if (stream_) cudaStreamSynchronize(stream_);
        invalidate_graph();
        cudaFree(bst_); cudaFree(d_scenes_); cudaFree(d_chunk_scene_); cudaFree(d_block_scene_);
        if (ev0_) cudaEventDestroy(ev0_);
        if (ev1_) cudaEventDestroy(ev1_);
        if (stream_) cudaStreamDestroy(stream_);
        stream_ = nullptr;
    }

    std::vector<E *> eng_;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    DevStatus *bst_ = nullptr;
    SceneDesc<Real, Acc> *d_scenes_ = nullptr;
    int *d_chunk_scene_ = nullptr, *d_block_scene_ = nullptr;
    int chunk_cap_ = 0, block_cap_ = 0, nchunks_ = -1, nblocks_ = -1;
    std::vector<int> chunk_scene_, block_scene_;
    int ctas_[NSHAPES] = {0, 0, 0};
    int shape_ = 0;
    icempm_batch_tuning_t tune_{0, 2, 0, 50, 0.0f, {0, 0, 0}};
    int since_sort_ = 0;
    bool timed_ = false;
    cudaGraphExec_t graph_exec_ = nullptr;
    uint64_t graph_launches_ = 0, launches_ = 0;
};

template <class Real, class Acc>
Batch *make_batch_t(Engine *const *engines, int count)
{
    std::vector<EngineT<Real, Acc> *> v;
    for (int i = 0; i < count; i++) {
        auto *e = dynamic_cast<EngineT<Real, Acc> *>(engines[i]);
        if (!e) { fail(ICEMPM_E_ARG, "all contexts of a batch must use the same variant"); return nullptr; }
        if (!v.empty() && e->device() != v[0]->device()) {
            fail(ICEMPM_E_ARG, "all contexts of a batch must be on the same device");
            return nullptr;
        }
        v.push_back(e);
    }
    auto *b = new BatchT<Real, Acc>();
    if (b->init(std::move(v))) { delete b; return nullptr; }
    return b;
}

}  // namespace icempm
