/* Device harness around the reference's own CUDA step (igorg520b/iceMPM_2d_sp):
 *   simulation/kernels.cuh, helper_math.cuh, givens.cuh, parameters_sim.h
 * compiled unmodified for sm_100a, where they lie, by
 * oracle/refbuild/build_ref_gpu.py, with the stand-in headers in stubs/
 * (a host+device 2x2 Eigen subset, spdlog/HDF5 no-ops).  This file replaces
 * GPU_Partition (simulation/gpu_partition.cpp), which needs HDF5 and the
 * wind interpolator to compile, with the few calls the sub-step makes:
 *   allocate            gpu_partition.cpp:259-293  (cudaMallocPitch, 19 point rows, 9 grid rows)
 *   update_constants    gpu_partition.cpp:140-170  (cudaMemcpyToSymbol of gprms and the partition symbols)
 *   reset_grid          gpu_partition.cpp:300-308  (memset of grid rows 0-2 each sub-step)
 *   p2g / update_nodes / g2p  gpu_partition.cpp:322-365 (tpb_P2G / tpb_Upd / tpb_G2P blocks)
 * with the sub-step loop of Model::Step (simulation/model.cpp:18-39):
 * simulation time passed as float, recordPQ when step % UpdateEveryNthStep == 0.
 * One scene at a time (the reference keeps its state in __constant__ /
 * __device__ symbols).  TEST AND MEASUREMENT INFRASTRUCTURE ONLY: it measures
 * the reference's GPU step and pins parity against it; the product never
 * links it. */
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>

#include <cuda_runtime.h>

#include "parameters_sim.h"
#include "helper_math.cuh"

/* prototypes of the kernel helpers, same signatures as gpu_partition.h:28-59 */
__device__ void svd2x2(const PointMatrix2r &mA, PointMatrix2r &mU, PointVector2r &mS, PointMatrix2r &mV);
__device__ void Wolper_Drucker_Prager(const t_PointReal &initial_strength, const t_PointReal &p_tr,
                                      const t_PointReal &q_tr, const t_PointReal &Je_tr,
                                      const PointMatrix2r &U, const PointMatrix2r &V,
                                      const PointVector2r &vSigmaSquared, const PointVector2r &v_s_hat_tr,
                                      PointMatrix2r &Fe, t_PointReal &Jp_inv);
__device__ void CheckIfPointIsInsideFailureSurface(uint32_t &utility_data, const uint16_t &grain,
                                                   const t_PointReal &p, const t_PointReal &q,
                                                   const t_PointReal &strength);
__device__ void ComputeSVD(const PointMatrix2r &Fe, PointMatrix2r &U, PointVector2r &vSigma, PointMatrix2r &V,
                           PointVector2r &vSigmaSquared, PointVector2r &v_s_hat_tr,
                           const t_PointReal &kappa, const t_PointReal &mu, const t_PointReal &Je_tr);
__device__ void ComputePQ(t_PointReal &Je_tr, t_PointReal &p_tr, t_PointReal &q_tr,
                          const double &kappa, const double &mu, const PointMatrix2r &F);
__device__ void GetParametersForGrain(uint32_t utility_data, t_PointReal &pmin, t_PointReal &pmax,
                                      t_PointReal &qmax, t_PointReal &beta, t_PointReal &mSq,
                                      t_PointReal &pmin2);
__device__ PointMatrix2r KirchhoffStress_Wolper(const PointMatrix2r &F);
__device__ PointVector2r dev_d(PointVector2r Adiag);
__device__ PointMatrix2r dev(PointMatrix2r A);
__device__ void CalculateWeightCoeffs(const PointVector2r &pos, PointArray2r ww[3]);

#include "kernels.cuh"

namespace {

struct RefScene {
    SimParams prms{};
    double *pts = nullptr;      // 19 rows, pitch pts_pitch (elements)
    double *grid = nullptr;     // 9 rows, pitch grid_pitch (elements)
    uint8_t *status = nullptr;
    size_t pts_pitch = 0, grid_pitch = 0, capacity = 0, n = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

RefScene *g_scene = nullptr;
std::string g_err;

int fail(const char *what, cudaError_t e)
{
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return -2;
}

#define REF_CHECK(call, what)                       \
    do {                                            \
        cudaError_t e_ = (call);                    \
        if (e_ != cudaSuccess) return fail(what, e_); \
    } while (0)

/* GPU_Partition::update_constants (gpu_partition.cpp:140-170) */
int upload_symbols(RefScene &s)
{
    const uint32_t zero = 0;
    const int izero = 0;
    const size_t gx = (size_t)s.prms.GridXTotal;
    REF_CHECK(cudaMemcpyToSymbol(gpu_error_indicator, &zero, sizeof(zero)), "gpu_error_indicator");
    REF_CHECK(cudaMemcpyToSymbol(gpu_disabled_points_count, &izero, sizeof(izero)), "gpu_disabled_points_count");
    REF_CHECK(cudaMemcpyToSymbol(gprms, &s.prms, sizeof(SimParams)), "gprms");
    REF_CHECK(cudaMemcpyToSymbol(partition_buffer_pts, &s.pts, sizeof(double *)), "partition_buffer_pts");
    REF_CHECK(cudaMemcpyToSymbol(partition_buffer_grid, &s.grid, sizeof(double *)), "partition_buffer_grid");
    REF_CHECK(cudaMemcpyToSymbol(partition_gridX, &gx, sizeof(size_t)), "partition_gridX");
    REF_CHECK(cudaMemcpyToSymbol(partition_pitch_grid, &s.grid_pitch, sizeof(size_t)), "partition_pitch_grid");
    REF_CHECK(cudaMemcpyToSymbol(partition_count_pts, &s.n, sizeof(size_t)), "partition_count_pts");
    REF_CHECK(cudaMemcpyToSymbol(partition_pitch_pts, &s.pts_pitch, sizeof(size_t)), "partition_pitch_pts");
    REF_CHECK(cudaMemcpyToSymbol(partition_grid_status, &s.status, sizeof(uint8_t *)), "partition_grid_status");
    return 0;
}

}  // namespace

extern "C" {

const char *ref_gpu_last_error(void) { return g_err.c_str(); }

int ref_gpu_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

void ref_gpu_destroy(void)
{
    if (!g_scene) return;
    RefScene &s = *g_scene;
    if (s.stream) cudaStreamSynchronize(s.stream);
    cudaFree(s.pts);
    cudaFree(s.grid);
    cudaFree(s.status);
    if (s.ev0) cudaEventDestroy(s.ev0);
    if (s.ev1) cudaEventDestroy(s.ev1);
    if (s.stream) cudaStreamDestroy(s.stream);
    delete g_scene;
    g_scene = nullptr;
}

/* Allocates the scene (gpu_partition.cpp:259-293) and uploads the grid
 * status and the 9 grid rows (host pitch grid_host_pitch elements; rows 5-6
 * carry the current field the way transfer_wind_and_current_data_to_device
 * leaves them). */
int ref_gpu_create(const SimParams *prms, const uint8_t *grid_status, const double *grid, size_t grid_host_pitch,
                   size_t capacity)
{
    ref_gpu_destroy();
    if (!prms || !grid_status || !grid || capacity == 0) {
        g_err = "null argument or zero capacity";
        return -1;
    }
    g_scene = new RefScene();
    RefScene &s = *g_scene;
    s.prms = *prms;
    s.capacity = capacity;
    const size_t gx = (size_t)prms->GridXTotal, gy = (size_t)prms->GridYTotal, G = gx * gy;
    if (grid_host_pitch < G) {
        g_err = "grid host pitch below GridXTotal*GridYTotal";
        return -1;
    }
    REF_CHECK(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking), "stream");
    REF_CHECK(cudaEventCreate(&s.ev0), "event");
    REF_CHECK(cudaEventCreate(&s.ev1), "event");
    size_t pitch = 0;
    REF_CHECK(cudaMallocPitch((void **)&s.grid, &pitch, sizeof(double) * G, SimParams::nGridArrays), "grid");
    s.grid_pitch = pitch / sizeof(double);
    REF_CHECK(cudaMalloc((void **)&s.status, G), "grid status");
    REF_CHECK(cudaMallocPitch((void **)&s.pts, &pitch, sizeof(double) * capacity, SimParams::nPtsArrays), "points");
    s.pts_pitch = pitch / sizeof(double);
    REF_CHECK(cudaMemset2D(s.grid, s.grid_pitch * sizeof(double), 0, s.grid_pitch * sizeof(double),
                           SimParams::nGridArrays), "grid clear");
    REF_CHECK(cudaMemcpy2D(s.grid, s.grid_pitch * sizeof(double), grid, grid_host_pitch * sizeof(double),
                           G * sizeof(double), SimParams::nGridArrays, cudaMemcpyHostToDevice), "grid upload");
    REF_CHECK(cudaMemcpy(s.status, grid_status, G, cudaMemcpyHostToDevice), "grid status upload");
    return upload_symbols(s);
}

/* transfer_to_device (gpu_partition.cpp:81-137): n points from a host HSSOA
 * whose rows are host_pitch doubles apart; resets the error word and the
 * disabled-point counter. */
int ref_gpu_upload(const double *soa, size_t host_pitch, size_t n)
{
    if (!g_scene) { g_err = "no scene"; return -4; }
    RefScene &s = *g_scene;
    if (n > s.capacity || host_pitch < n) { g_err = "n exceeds capacity or host pitch"; return -5; }
    s.n = n;
    if (n)
        REF_CHECK(cudaMemcpy2D(s.pts, s.pts_pitch * sizeof(double), soa, host_pitch * sizeof(double),
                               n * sizeof(double), SimParams::nPtsArrays, cudaMemcpyHostToDevice), "points upload");
    return upload_symbols(s);
}

/* nsteps sub-steps starting at first_step: reset_grid, p2g, update_nodes, g2p
 * with the reference's launch shapes, enqueued back to back on one stream.
 * *ms (optional) = device time between events around the loop. */
int ref_gpu_run(int nsteps, int first_step, float *ms)
{
    if (!g_scene) { g_err = "no scene"; return -4; }
    RefScene &s = *g_scene;
    const SimParams &p = s.prms;
    const int n = (int)s.n;
    const int nNodes = p.GridYTotal * p.GridXTotal;
    const int bP2G = (n + p.tpb_P2G - 1) / p.tpb_P2G;
    const int bUpd = (nNodes + p.tpb_Upd - 1) / p.tpb_Upd;
    const int bG2P = (n + p.tpb_G2P - 1) / p.tpb_G2P;
    REF_CHECK(cudaEventRecord(s.ev0, s.stream), "event record");
    for (int k = 0; k < nsteps; k++) {
        const int step = first_step + k;
        const float simulation_time = (float)(p.InitialTimeStep * step);
        REF_CHECK(cudaMemsetAsync(s.grid, 0, s.grid_pitch * 3 * sizeof(double), s.stream), "reset_grid");
        if (bP2G > 0) partition_kernel_p2g<<<bP2G, p.tpb_P2G, 0, s.stream>>>();
        REF_CHECK(cudaGetLastError(), "p2g kernel");
        partition_kernel_update_nodes<<<bUpd, p.tpb_Upd, 0, s.stream>>>(simulation_time);
        REF_CHECK(cudaGetLastError(), "update_nodes");
        const bool recordPQ = step % p.UpdateEveryNthStep == 0;
        if (bG2P > 0) partition_kernel_g2p<<<bG2P, p.tpb_G2P, 0, s.stream>>>(recordPQ);
        REF_CHECK(cudaGetLastError(), "g2p kernel");
    }
    REF_CHECK(cudaEventRecord(s.ev1, s.stream), "event record");
    REF_CHECK(cudaEventSynchronize(s.ev1), "step loop");
    if (ms) REF_CHECK(cudaEventElapsedTime(ms, s.ev0, s.ev1), "elapsed time");
    return 0;
}

/* transfer_from_device (gpu_partition.cpp:17-59): the points, the error word,
 * the disabled count and (optionally) the 9 grid rows. */
int ref_gpu_download(double *soa, size_t host_pitch, double *grid, size_t grid_host_pitch, uint32_t *err,
                     int *disabled)
{
    if (!g_scene) { g_err = "no scene"; return -4; }
    RefScene &s = *g_scene;
    REF_CHECK(cudaStreamSynchronize(s.stream), "sync");
    if (soa && s.n)
        REF_CHECK(cudaMemcpy2D(soa, host_pitch * sizeof(double), s.pts, s.pts_pitch * sizeof(double),
                               s.n * sizeof(double), SimParams::nPtsArrays, cudaMemcpyDeviceToHost), "points download");
    if (grid) {
        const size_t G = (size_t)s.prms.GridXTotal * s.prms.GridYTotal;
        REF_CHECK(cudaMemcpy2D(grid, grid_host_pitch * sizeof(double), s.grid, s.grid_pitch * sizeof(double),
                               G * sizeof(double), SimParams::nGridArrays, cudaMemcpyDeviceToHost), "grid download");
    }
    if (err) REF_CHECK(cudaMemcpyFromSymbol(err, gpu_error_indicator, sizeof(uint32_t)), "error word");
    if (disabled) REF_CHECK(cudaMemcpyFromSymbol(disabled, gpu_disabled_points_count, sizeof(int)), "disabled count");
    return 0;
}

}  /* extern "C" */
