/* Host harness around the reference's SnapshotManager::PrepareFrameArrays and
 * SnapshotManager::CalculateWeightCoeffs (simulation/data_manager/
 * snapshotmanager.cpp:611-765 of igorg520b/iceMPM_2d_sp).  Those two member
 * functions are read from the reference checkout where it lies and compiled
 * unmodified (oracle/refbuild/build_ref.py extracts them into
 * oracle/_ref/frame_extract.inc at build time; the rest of the file needs HDF5,
 * OpenJPEG, stb and the whole Model).  The class itself comes from the
 * reference's own snapshotmanager.h and gui/colormap.h; icy::Model is a
 * stand-in with the members the function reads (model.h, gpu_implementation5.h:
 * prms, gpu.hssoa, gpu.point_colors_rgb, gpu.grid_status_buffer,
 * gpu.grid_boundary_forces).  TEST INFRASTRUCTURE ONLY: it produces the
 * golden frames that pin the frame rasteriser and its CPU restatement. */
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <vector>

#include "parameters_sim.h"
#include "host_side_soa.h"

namespace icy {
class Model {
public:
    SimParams prms;
    struct Gpu {
        HostSideSOA hssoa;
        std::vector<uint32_t> point_colors_rgb;
        std::vector<uint8_t> grid_status_buffer;
        std::vector<t_GridReal> grid_boundary_forces;
    } gpu;
};
}  // namespace icy

/* The harness reads the private per-cell counts after the call. */
#define private public
#include "snapshotmanager.h"
#undef private

icy::SnapshotManager::SnapshotManager() {}
icy::SnapshotManager::~SnapshotManager() {}

#include "frame_extract.inc"

extern "C" {

/* Runs the reference's PrepareFrameArrays on a caller-owned HSSOA (19 rows of
 * `pitch` doubles, `n` points), point colours (indexed by point id), grid
 * status and boundary forces (2 x gx*gy, fx rows then fy rows).  Writes the
 * ten float channels (gx*gy each), rgb (3 per node), mass_mask and count
 * (gx*gy each), and forces_per_region (MAX_REGIONS x 2 floats).  Returns
 * MAX_REGIONS. */
int ref_prepare_frame(const SimParams *prms, double *soa, unsigned pitch, unsigned n, const uint32_t *colors,
                      unsigned ncolors, const uint8_t *status, const double *forces, float *density,
                      float *mass, float *vx, float *vy, float *Jpinv, float *P, float *Q, float *r, float *g,
                      float *b, uint8_t *rgb, uint8_t *mass_mask, uint8_t *count, float *forces_per_region)
{
    icy::Model model;
    model.prms = *prms;
    const size_t G = (size_t)prms->GridXTotal * prms->GridYTotal;
    model.gpu.hssoa.host_buffer = soa;
    model.gpu.hssoa.capacity = pitch;
    model.gpu.hssoa.size = n;
    model.gpu.point_colors_rgb.assign(colors, colors + ncolors);
    model.gpu.grid_status_buffer.assign(status, status + G);
    model.gpu.grid_boundary_forces.assign(forces, forces + 2 * G);
    icy::SnapshotManager sm;
    sm.model = &model;
    sm.PrepareFrameArrays();
    std::copy(sm.vis_point_density.begin(), sm.vis_point_density.end(), density);
    std::copy(sm.vis_mass.begin(), sm.vis_mass.end(), mass);
    std::copy(sm.vis_vx.begin(), sm.vis_vx.end(), vx);
    std::copy(sm.vis_vy.begin(), sm.vis_vy.end(), vy);
    std::copy(sm.vis_Jpinv.begin(), sm.vis_Jpinv.end(), Jpinv);
    std::copy(sm.vis_P.begin(), sm.vis_P.end(), P);
    std::copy(sm.vis_Q.begin(), sm.vis_Q.end(), Q);
    std::copy(sm.vis_r.begin(), sm.vis_r.end(), r);
    std::copy(sm.vis_g.begin(), sm.vis_g.end(), g);
    std::copy(sm.vis_b.begin(), sm.vis_b.end(), b);
    std::copy(sm.rgb.begin(), sm.rgb.end(), rgb);
    std::copy(sm.mass_mask.begin(), sm.mass_mask.end(), mass_mask);
    std::copy(sm.count.begin(), sm.count.end(), count);
    for (int k = 0; k < SimParams::MAX_REGIONS; k++) {
        forces_per_region[2 * k] = sm.forces_per_region[k].x();
        forces_per_region[2 * k + 1] = sm.forces_per_region[k].y();
    }
    model.gpu.hssoa.host_buffer = nullptr;   /* the buffer stays the caller's */
    return SimParams::MAX_REGIONS;
}

}  /* extern "C" */
