// shim_driver.cpp -- runs the reference's frame loop (icy::Model::Step,
// simulation/model.cpp:7-78) through the GPU_Implementation5 shim over the C
// ABI, for the tests.  Usage: shim_driver <scene.bin> <out.bin> <frames>
//   scene.bin: SimParams (328 B), u32 n, u32 capacity, u8 status[G],
//              f64 current[2G], f64 hssoa[19*capacity]
//   out.bin:   f64 hssoa[19*capacity], u32 size, u32 error_code, i32 disabled
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "icempm_gpu_implementation5.hpp"

using icempm_shim::GPU_Implementation5;

int main(int argc, char **argv)
{
    if (argc < 4) { std::cerr << "usage: shim_driver scene.bin out.bin frames\n"; return 2; }
    std::ifstream in(argv[1], std::ios::binary);
    icempm_simparams_t prms;
    uint32_t n = 0, cap = 0;
    in.read(reinterpret_cast<char *>(&prms), sizeof(prms));
    in.read(reinterpret_cast<char *>(&n), 4);
    in.read(reinterpret_cast<char *>(&cap), 4);
    const size_t G = (size_t)prms.GridXTotal * prms.GridYTotal;
    GPU_Implementation5 gpu;
    gpu.prms = &prms;
    prms.nPtsInitial = (int)cap;
    gpu.initialize();
    gpu.allocate_host_arrays_grid();
    gpu.allocate_host_arrays_points();
    in.read(reinterpret_cast<char *>(gpu.grid_status_buffer.data()), (std::streamsize)G);
    gpu.current_flow_data.resize(2 * G);
    in.read(reinterpret_cast<char *>(gpu.current_flow_data.data()), (std::streamsize)(2 * G * sizeof(double)));
    in.read(reinterpret_cast<char *>(gpu.hssoa.host_buffer), (std::streamsize)((size_t)19 * cap * sizeof(double)));
    if (!in) { std::cerr << "short scene file\n"; return 2; }
    gpu.hssoa.size = n;
    const int frames = std::atoi(argv[3]);
    try {
        // SnapshotManager::SplitIntoPartitionsAndTransferToDevice + Model::Prepare
        gpu.split_hssoa_into_partitions();
        gpu.allocate_device_arrays();
        gpu.transfer_to_device();
        gpu.update_constants();
        gpu.transfer_wind_and_current_data_to_device();
        for (int f = 0; f < frames; f++) {
            gpu.reset_timings();
            gpu.clear_force_accumulator();
            double simulation_time = 0;
            int count_unupdated_steps = 0;
            do {
                const int step = prms.SimulationStep + count_unupdated_steps;
                simulation_time = prms.InitialTimeStep * step;
                gpu.reset_grid();
                gpu.p2g();
                gpu.update_nodes((float)simulation_time, 0, 0);
                const bool isCycleStart = step % prms.UpdateEveryNthStep == 0;
                gpu.g2p(isCycleStart, false, false);
                gpu.record_timings(false);
                count_unupdated_steps++;
            } while ((prms.SimulationStep + count_unupdated_steps) % prms.UpdateEveryNthStep != 0);
            gpu.transfer_from_device(count_unupdated_steps);
            prms.SimulationTime = simulation_time;
            prms.SimulationStep += count_unupdated_steps;
            auto &p = gpu.partitions.front();
            const float disabled_proportion = (float)p.disabled_points_count / p.nPts_partition;
            if (disabled_proportion > ICEMPM_DISABLED_PTS_PROPORTION_THRESHOLD) {
                gpu.hssoa.RemoveDisabledAndSort(prms.GridYTotal);
                gpu.split_hssoa_into_partitions();
                gpu.transfer_to_device();
            }
            if (gpu.error_code) break;
        }
    } catch (const std::exception &e) {
        std::cerr << "shim_driver: " << e.what() << "\n";
        return 1;
    }
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char *>(gpu.hssoa.host_buffer), (std::streamsize)((size_t)19 * cap * sizeof(double)));
    const uint32_t size = gpu.hssoa.size, err = gpu.error_code;
    const int32_t dis = gpu.partitions.front().disabled_points_count;
    out.write(reinterpret_cast<const char *>(&size), 4);
    out.write(reinterpret_cast<const char *>(&err), 4);
    out.write(reinterpret_cast<const char *>(&dis), 4);
    return 0;
}
