/* Host harness around the reference's own sources (igorg520b/iceMPM_2d_sp):
 *   simulation/parameters_sim.h, helper_math.cuh, givens.cuh, kernels.cuh,
 *   parameters_sim.cpp, hssoa/host_side_soa.cpp, hssoa/proxypoint2d.cpp
 * compiled unmodified, where they lie, by oracle/refbuild/build_ref.py, with
 * the stand-in headers in stubs/.  The three __global__ kernels run as plain
 * functions, once per (block, thread).  ref_run_steps runs P2G serially in
 * index order, so its "atomics" are applied in point-index order (the golden
 * fixtures); ref_run_steps_parallel runs P2G's blocks in parallel with real
 * atomic adds, as the GPU does (the timed host baseline).  The grid update
 * and G2P always run their blocks in parallel.  TEST INFRASTRUCTURE ONLY: it
 * pins the oracle restatement (oracle/icempm_oracle.c) to the reference code
 * and times the reference's own step on the host cores. */
#include <cstddef>
#include <cstdint>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "parameters_sim.h"
#include "helper_math.cuh"

thread_local ref_dim3 blockIdx, threadIdx, blockDim;
bool ref_atomics_on = false;

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
#include "host_side_soa.h"

/* Serial launch: blocks and threads in index order (used for P2G, whose
 * floating-point atomics are emulated as plain adds). */
template <class K> static void emulate_launch(size_t nthreads, int tpb, K kernel)
{
    const size_t nblocks = (nthreads + tpb - 1) / tpb;
    blockDim.x = tpb;
    for (size_t b = 0; b < nblocks; b++) {
        blockIdx.x = (unsigned)b;
        for (int t = 0; t < tpb; t++) { threadIdx.x = t; kernel(); }
    }
}

/* Parallel launch over blocks with OpenMP, for the grid update and G2P: their
 * threads write disjoint data; the only shared writes are the disabled-point
 * counter (atomic in the stub) and the error word, which these kernels touch
 * only on NaN or out-of-cell errors. */
template <class K> static void emulate_launch_parallel(size_t nthreads, int tpb, K kernel)
{
    const long long nblocks = (long long)((nthreads + tpb - 1) / tpb);
#pragma omp parallel for schedule(static)
    for (long long b = 0; b < nblocks; b++) {
        blockDim.x = tpb;
        blockIdx.x = (unsigned)b;
        for (int t = 0; t < tpb; t++) { threadIdx.x = t; kernel(); }
    }
}

extern "C" {

void ref_params_reset(SimParams *p) { p->Reset(); }
void ref_compute_helpers(SimParams *p) { p->ComputeHelperVariables(); }

/* Byte offsets of the SimParams fields in declaration order; returns sizeof. */
int ref_simparams_layout(long long *off, int n)
{
#define O(f) offsetof(SimParams, f)
    const long long v[] = {
        O(tpb_P2G), O(tpb_Upd), O(tpb_G2P), O(nPartitions), O(nPtsInitial), O(SimulationStartUnixTime),
        O(InitialTimeStep), O(SimulationEndTime), O(AnimationFramePeriod), O(SimulationStep),
        O(SimulationTime), O(SaveSnapshots), O(SnapshotPeriod), O(GridXTotal), O(GridYTotal),
        O(ModeledRegionOffsetX), O(ModeledRegionOffsetY), O(InitializationImageSizeX),
        O(InitializationImageSizeY), O(DimensionHorizontal), O(windDragCoeff_airDensity),
        O(UseWindData), O(UseCurrentData), O(sea_water_density), O(waterDragEffectiveLinear),
        O(waterDragEffectiveQuadratic), O(IceDensity), O(PoissonsRatio), O(YoungsModulus),
        O(IceCompressiveStrength), O(IceTensileStrength), O(IceShearStrength), O(IceTensileStrength2),
        O(DP_phi), O(DP_threshold_p), O(RidgeFormationCoeff), O(cellsize), O(ParticleVolume),
        O(ParticleViewSize), O(dt_vol_Dpinv), O(vmax), O(lambda), O(mu), O(kappa), O(ParticleMass),
        O(cellsize_inv), O(Dp_inv), O(UpdateEveryNthStep)};
#undef O
    const int m = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < m; i++) off[i] = v[i];
    return (int)sizeof(SimParams);
}

void ref_svd2x2(const double *F, double *U, double *S, double *V)
{
    PointMatrix2r mA, mU, mV;
    PointVector2r mS;
    mA(0, 0) = F[0]; mA(0, 1) = F[1]; mA(1, 0) = F[2]; mA(1, 1) = F[3];
    svd2x2(mA, mU, mS, mV);
    U[0] = mU(0, 0); U[1] = mU(0, 1); U[2] = mU(1, 0); U[3] = mU(1, 1);
    V[0] = mV(0, 0); V[1] = mV(0, 1); V[2] = mV(1, 0); V[3] = mV(1, 1);
    S[0] = mS[0]; S[1] = mS[1];
}

/* The sub-step loop of Model::Step (model.cpp:18-39) over GPU_Partition's
 * reset_grid / p2g / update_nodes / g2p (gpu_partition.cpp:300-365) with the
 * reference kernels.  parallel_p2g: P2G's blocks over OpenMP threads with
 * atomic adds (summation order then varies run to run, as on the GPU).
 * Returns gpu_error_indicator; adds to *disabled. */
static uint32_t run_steps(const SimParams *prms, double *soa, size_t pitch, size_t n, double *grid, size_t gpitch,
                          uint8_t *status, int nsteps, int first_step, int *disabled, bool parallel_p2g)
{
    gprms = *prms;
    partition_buffer_pts = soa;
    partition_buffer_grid = grid;
    partition_gridX = (size_t)prms->GridXTotal;
    partition_pitch_grid = gpitch;
    partition_count_pts = n;
    partition_pitch_pts = pitch;
    partition_grid_status = status;
    gpu_error_indicator = 0;
    gpu_disabled_points_count = 0;
    ref_atomics_on = parallel_p2g;
    const size_t nNodes = (size_t)prms->GridXTotal * prms->GridYTotal;
    for (int k = 0; k < nsteps; k++) {
        const int step = first_step + k;
        const float simulation_time = (float)(prms->InitialTimeStep * step);
        std::memset(grid, 0, gpitch * 3 * sizeof(double));
        if (parallel_p2g) emulate_launch_parallel(n, prms->tpb_P2G, [] { partition_kernel_p2g(); });
        else emulate_launch(n, prms->tpb_P2G, [] { partition_kernel_p2g(); });
        emulate_launch_parallel(nNodes, prms->tpb_Upd, [&] { partition_kernel_update_nodes(simulation_time); });
        const bool isCycleStart = step % prms->UpdateEveryNthStep == 0;
        emulate_launch_parallel(n, prms->tpb_G2P, [&] { partition_kernel_g2p(isCycleStart); });
    }
    ref_atomics_on = false;
    if (disabled) *disabled += gpu_disabled_points_count;
    return gpu_error_indicator;
}

uint32_t ref_run_steps(const SimParams *prms, double *soa, size_t pitch, size_t n, double *grid,
                       size_t gpitch, uint8_t *status, int nsteps, int first_step, int *disabled)
{
    return run_steps(prms, soa, pitch, n, grid, gpitch, status, nsteps, first_step, disabled, false);
}

uint32_t ref_run_steps_parallel(const SimParams *prms, double *soa, size_t pitch, size_t n, double *grid,
                                size_t gpitch, uint8_t *status, int nsteps, int first_step, int *disabled)
{
    return run_steps(prms, soa, pitch, n, grid, gpitch, status, nsteps, first_step, disabled, true);
}

/* HostSideSOA::RemoveDisabledAndSort on a caller-owned buffer. */
unsigned ref_remove_disabled_and_sort(double *soa, unsigned capacity, unsigned size, int gridY)
{
    HostSideSOA h;
    h.host_buffer = soa;
    h.capacity = capacity;
    h.size = size;
    h.RemoveDisabledAndSort(gridY);
    unsigned r = h.size;
    h.host_buffer = nullptr;  /* the buffer stays the caller's */
    return r;
}

int ref_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  /* extern "C" */
