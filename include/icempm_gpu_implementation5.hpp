// icempm_gpu_implementation5.hpp -- header-only C++ shim with the public shape
// of the reference's GPU_Implementation5 / GPU_Partition / HostSideSOA
// (simulation/gpu_implementation5.h:23-68, gpu_partition.h:63-134,
// hssoa/host_side_soa.h:51-74), implemented over the C ABI of icempm.h, so that
// code written against the reference's GPU driver -- icy::Model::Step
// (model.cpp:7-78), SnapshotManager::SplitIntoPartitionsAndTransferToDevice
// (snapshotmanager.cpp:295-306) -- keeps its calls.
//
// Per sub-step the reference calls reset_grid(), p2g(), update_nodes(t),
// g2p(recordPQ), record_timings(); here g2p() advances the device by one
// sub-step (icempm_step) and the other three only record their arguments.
// The step index of each sub-step is counted from SimulationStep at the last
// transfer_to_device()/update_constants(), as Model::Step numbers them.
// step_frame(n) runs n sub-steps in one call (CUDA graphs) for callers that
// can batch.
//
// Errors: CUDA/API failures throw std::runtime_error with icempm_last_error(),
// as the reference throws on CUDA errors; device error bits land in
// error_code after transfer_from_device(), as in the reference.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "icempm.h"

namespace icempm_shim {

using SimParams = icempm_simparams_t;

inline void check(int rc, const char *what)
{
    if (rc < 0) throw std::runtime_error(std::string(what) + ": " + icempm_last_error());
}

// HostSideSOA (host_side_soa.h:51-74): 19 f64 rows with pitch = capacity.
struct HostSideSOA {
    std::vector<double> storage;
    double *host_buffer = nullptr;
    unsigned capacity = 0;
    unsigned size = 0;

    void Allocate(int pts_capacity)
    {
        capacity = (unsigned)pts_capacity;
        size = 0;
        storage.assign((size_t)capacity * ICEMPM_N_PTS_ARRAYS, 0.0);
        host_buffer = storage.data();
    }
    double *getPointerToLine(int idxLine) { return host_buffer + (size_t)capacity * idxLine; }

    static uint32_t u32(const double *slot) { uint32_t v; std::memcpy(&v, slot, 4); return v; }

    // RemoveDisabledAndSort (host_side_soa.cpp:36-47) on the host; ties keep
    // their order.
    void RemoveDisabledAndSort(int GridY)
    {
        std::vector<uint32_t> idx;
        idx.reserve(size);
        for (unsigned i = 0; i < size; i++)
            if (!(u32(&host_buffer[i + (size_t)capacity * ICEMPM_IDX_UTILITY]) & ICEMPM_STATUS_DISABLED)) idx.push_back(i);
        auto key = [&](uint32_t i) {
            const uint32_t c = u32(&host_buffer[i + (size_t)capacity * ICEMPM_IDX_CELL]);
            return (uint64_t)(c & 0xffff) * (uint64_t)GridY + (c >> 16);
        };
        std::stable_sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) { return key(a) < key(b); });
        std::vector<double> row(idx.size());
        for (int r = 0; r < ICEMPM_N_PTS_ARRAYS; r++) {
            double *line = getPointerToLine(r);
            for (size_t k = 0; k < idx.size(); k++) row[k] = line[idx[k]];
            std::copy(row.begin(), row.end(), line);
        }
        size = (unsigned)idx.size();
    }
};

// The fields of GPU_Partition that Model::Step reads (gpu_partition.h:92-121).
struct GPU_Partition {
    int PartitionID = 0, Device = 0;
    size_t nPts_partition = 0, GridX_partition = 0, GridX_offset = 0, nPtsPitch = 0;
    uint32_t error_code = 0;
    int disabled_points_count = 0;
    float timing_10_P2GAndHalo = 0, timing_20_acceptHalo = 0, timing_30_updateGrid = 0, timing_40_G2P = 0;
    float timing_60_ptsSent = 0, timing_70_ptsAccepted = 0, timing_stepTotal = 0;

    void reset_timings()
    {
        timing_10_P2GAndHalo = timing_20_acceptHalo = timing_30_updateGrid = timing_40_G2P = 0;
        timing_60_ptsSent = timing_70_ptsAccepted = timing_stepTotal = 0;
    }
    void normalize_timings(int cycles)
    {
        const float c = 1000.f / (float)cycles;
        timing_10_P2GAndHalo *= c; timing_20_acceptHalo *= c; timing_30_updateGrid *= c; timing_40_G2P *= c;
        timing_60_ptsSent *= c; timing_70_ptsAccepted *= c; timing_stepTotal *= c;
    }
};

class GPU_Implementation5 {
public:
    GPU_Implementation5() = default;
    ~GPU_Implementation5() { icempm_destroy(ctx_); }
    GPU_Implementation5(const GPU_Implementation5 &) = delete;
    GPU_Implementation5 &operator=(const GPU_Implementation5 &) = delete;

    const SimParams *prms = nullptr;       // the reference reads model->prms
    std::vector<GPU_Partition> partitions;
    HostSideSOA hssoa;
    uint32_t error_code = 0;
    std::vector<uint32_t> point_colors_rgb;
    std::vector<uint8_t> grid_status_buffer;
    std::vector<uint8_t> original_image_colors_rgb;
    std::vector<double> grid_boundary_normals, grid_boundary_forces;
    std::vector<double> current_flow_data;   // WindAndCurrentInterpolator::current_flow_data layout
    std::function<void()> transfer_completion_callback;
    icempm_options_t options = default_options();

    static icempm_options_t default_options() { icempm_options_t o; icempm_default_options(&o); return o; }

    void allocate_host_arrays_grid()
    {
        const size_t g = (size_t)prms->GridXTotal * prms->GridYTotal;
        grid_status_buffer.assign(g, 100);
        grid_boundary_normals.assign(2 * g, 0.0);
        grid_boundary_forces.assign(2 * g, 0.0);
        original_image_colors_rgb.assign(3 * (size_t)prms->InitializationImageSizeX * prms->InitializationImageSizeY, 0);
    }
    void allocate_host_arrays_points()
    {
        hssoa.Allocate(prms->nPtsInitial);
        point_colors_rgb.assign(prms->nPtsInitial, 0);
    }
    // GPU_Implementation5::initialize (gpu_implementation5.cpp:94-128): one partition.
    void initialize()
    {
        partitions.assign(1, GPU_Partition());
        partitions.front().Device = options.device;
    }
    void split_hssoa_into_partitions()
    {
        GPU_Partition &p = partitions.front();
        p.nPts_partition = hssoa.size;
        p.GridX_partition = prms->GridXTotal;
        p.disabled_points_count = 0;
    }
    void allocate_device_arrays()
    {
        icempm_destroy(ctx_);
        ctx_ = nullptr;
        const double *cur = current_flow_data.empty() ? nullptr : current_flow_data.data();
        check(icempm_create(prms, grid_status_buffer.data(), cur, (uint32_t)std::max<int>(prms->nPtsInitial, 1),
                            &options, &ctx_), "icempm_create");
        partitions.front().nPtsPitch = (size_t)std::max<int>(prms->nPtsInitial, 1);
    }
    void transfer_to_device()
    {
        check(icempm_upload_points(ctx_, hssoa.host_buffer, hssoa.capacity, hssoa.size,
                                   partitions.front().disabled_points_count), "icempm_upload_points");
        next_step_ = prms->SimulationStep;
    }
    void transfer_wind_and_current_data_to_device()
    {
        check(icempm_set_current(ctx_, current_flow_data.empty() ? nullptr : current_flow_data.data()),
              "icempm_set_current");
    }
    void update_constants()
    {
        error_code = 0;
        check(icempm_update_constants(ctx_, prms), "icempm_update_constants");
        next_step_ = prms->SimulationStep;
    }
    void reset_timings() { partitions.front().reset_timings(); }
    void clear_force_accumulator() { check(icempm_clear_force_accumulator(ctx_), "icempm_clear_force_accumulator"); }
    void reset_grid() {}
    void p2g() {}
    void update_nodes(float simulation_time, float /*windSpeed*/ = 0, float /*windAngle*/ = 0) { (void)simulation_time; }
    void g2p(const bool /*recordPQ*/, const bool /*enablePointTransfer*/ = false, int /*applyGlensLaw*/ = 0)
    {
        step_frame(1);
    }
    // n sub-steps from the current step index in one call
    void step_frame(int n)
    {
        check(icempm_step(ctx_, n, next_step_), "icempm_step");
        next_step_ += n;
        steps_since_timing_ += n;
    }
    void record_timings(const bool /*enablePointTransfer*/ = false) {}

    // GPU_Implementation5::transfer_from_device (gpu_implementation5.cpp:188-224)
    void transfer_from_device(const int elapsed_cycles)
    {
        GPU_Partition &p = partitions.front();
        uint32_t n = 0;
        check(icempm_point_count(ctx_, &n), "icempm_point_count");
        if (n > hssoa.capacity) throw std::runtime_error("transfer_from_device capacity exceeded");
        check(icempm_download_points(ctx_, hssoa.host_buffer, hssoa.capacity, &n), "icempm_download_points");
        hssoa.size = n;
        p.nPts_partition = n;
        uint32_t err = 0;
        int32_t dis = 0;
        check(icempm_get_status(ctx_, &err, &dis), "icempm_get_status");
        p.error_code = err;
        p.disabled_points_count = dis;
        if (err) error_code = err;
        check(icempm_get_boundary_forces(ctx_, grid_boundary_forces.data(), elapsed_cycles), "icempm_get_boundary_forces");
        float ms[4];
        check(icempm_timings(ctx_, ms), "icempm_timings");
        p.timing_stepTotal += ms[0];
        p.timing_30_updateGrid += ms[1];
        p.timing_40_G2P += ms[2];
        if (transfer_completion_callback) transfer_completion_callback();
    }
    void synchronize()
    {
        uint32_t e;
        int32_t d;
        if (ctx_) check(icempm_get_status(ctx_, &e, &d), "icempm_get_status");
    }
    // device-side RemoveDisabledAndSort + download (replaces the host sort and
    // re-upload of model.cpp:63-72 when the caller does not need them on the host)
    void compact_on_device()
    {
        check(icempm_sort_compact(ctx_), "icempm_sort_compact");
        uint32_t n = 0;
        check(icempm_download_points(ctx_, hssoa.host_buffer, hssoa.capacity, &n), "icempm_download_points");
        hssoa.size = n;
        partitions.front().nPts_partition = n;
        partitions.front().disabled_points_count = 0;
    }
    icempm_t *context() { return ctx_; }

private:
    icempm_t *ctx_ = nullptr;
    int32_t next_step_ = 0;
    int steps_since_timing_ = 0;
};

}  // namespace icempm_shim
