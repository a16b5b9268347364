// engine_iface.h -- variant-independent interface between the C ABI (capi.cu)
// and the per-variant engines (engine_<variant>.cu).
#pragma once
#include <cstdint>
#include <string>
#include <cuda_runtime.h>
#include "icempm.h"

namespace icempm {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const std::string &msg);

// The learned return map's network packed for the in-kernel evaluation
// (surrogate.cu): FP32 parameters and normalisation (device pointers) into
// a device buffer of mlp_packed_bytes().
int mlp_pack(const float *d_params, const float *d_norm, void *d_packed, cudaStream_t stream);
size_t mlp_packed_bytes();

class Engine {
public:
    virtual ~Engine() {}
    virtual int init(const icempm_simparams_t &p, const uint8_t *status, const double *cur, uint32_t capacity,
                     const icempm_options_t &o) = 0;
    virtual int set_params(const icempm_simparams_t &p, double max_thickness) = 0;
    virtual int set_current(const double *cur) = 0;
    virtual int upload(const double *hssoa, uint32_t host_cap, uint32_t n, int32_t disabled) = 0;
    virtual int download(double *hssoa, uint32_t host_cap, uint32_t *size) = 0;
    virtual int download_async(double *hssoa, uint32_t host_cap, uint32_t *size) = 0;
    virtual int download_wait() = 0;
    virtual int update_constants(const icempm_simparams_t &p) = 0;
    virtual int step(int nsteps, int first_step) = 0;
    virtual int timings(float ms[4]) = 0;
    virtual int phase_times(int nsteps, float *update_ms, float *fused_ms) = 0;
    virtual int status(uint32_t *err, int32_t *dis) = 0;
    virtual int clear_forces() = 0;
    virtual int forces(double *fxfy, int elapsed) = 0;
    virtual int sort_compact() = 0;
    virtual uint32_t count() const = 0;
    virtual cudaStream_t stream() const = 0;
    virtual uint64_t launches() const = 0;
    virtual double fixed_scale_m() const = 0;
    virtual double fixed_scale_p() const = 0;
    virtual int harvest_begin(uint32_t capacity, int stride) = 0;
    virtual int harvest_end(float *records, uint32_t host_cap, uint32_t *count) = 0;
    virtual int prepare_frame(const uint32_t *colors, uint32_t ncolors, int elapsed, icempm_frame_t *out) = 0;
    virtual int set_flow_frames(const double *a, const double *b) = 0;
    virtual int set_wind_frames(const float *w, int rows, int cols, double cell, double x0, double y0) = 0;
    virtual int set_forcing_time(double tc, double tw) = 0;
    virtual int get_forcing(double *cur, double *stress) = 0;
    virtual int set_barrier_test(uint32_t extra_bytes, uint32_t wait_us) = 0;
    virtual int set_learned_map(const float *d_params, const float *d_norm, float tol) = 0;
    virtual int learned_counts(uint64_t *kept, uint64_t *fallbacks) = 0;
    virtual int tune_sort(int trial_steps, int first_step, int32_t *sort_every) = 0;
};

// Ensemble of contexts of one variant stepped together (batch.cuh).
class Batch {
public:
    virtual ~Batch() {}
    virtual int step(int nsteps, int first_step) = 0;
    virtual int timings(float ms[4]) = 0;
    virtual int autotune(int trial_steps, int first_step, icempm_batch_tuning_t *out) = 0;
    virtual int set_tuning(const icempm_batch_tuning_t *t) = 0;
    virtual int get_tuning(icempm_batch_tuning_t *t) const = 0;
    virtual uint64_t launches() const = 0;
};

Engine *make_engine_fixed();
Engine *make_engine_fp32();
Engine *make_engine_fp64();
// nullptr (with the message recorded) when the contexts do not fit one batch
Batch *make_batch_fixed(Engine *const *engines, int count);
Batch *make_batch_fp32(Engine *const *engines, int count);
Batch *make_batch_fp64(Engine *const *engines, int count);

}  // namespace icempm
