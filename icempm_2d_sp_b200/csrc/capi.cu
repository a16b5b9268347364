// capi.cu -- the extern "C" boundary declared in include/icempm.h.
// Each entry point validates its arguments, forwards to the variant engine and
// turns failures into negative return codes with a per-thread message; no C++
// exception crosses the boundary.
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine_iface.h"

namespace icempm {
static thread_local std::string g_last_error;
int fail(int code, const std::string &msg)
{
    g_last_error = msg;
    return code;
}
}  // namespace icempm

using icempm::fail;

struct icempm_context {
    icempm::Engine *eng = nullptr;
    icempm_simparams_t prms{};
    icempm_options_t opts{};
};

struct icempm_batch {
    icempm::Batch *b = nullptr;
};

#define ICEMPM_GUARD_BATCH(bt) \
    if (!(bt) || !(bt)->b) return fail(ICEMPM_E_ARG, "null batch")

#define ICEMPM_GUARD_CTX(ctx) \
    if (!(ctx) || !(ctx)->eng) return fail(ICEMPM_E_ARG, "null context")

#define ICEMPM_TRY(expr)                                                   \
    try {                                                                  \
        return (expr);                                                     \
    } catch (const std::bad_alloc &) {                                     \
        return fail(ICEMPM_E_NOMEM, "host allocation failed");             \
    } catch (const std::exception &e) {                                    \
        return fail(ICEMPM_E_STATE, e.what());                             \
    } catch (...) {                                                        \
        return fail(ICEMPM_E_STATE, "unknown exception");                  \
    }

extern "C" {

void icempm_default_options(icempm_options_t *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->variant = ICEMPM_VARIANT_FIXED;
    o->forcing = ICEMPM_FORCING_COMPAT;
    o->sort_every = 0;
    o->use_graphs = 1;
    o->block_threads = 128;
    o->warp_reduce = 1;
    o->device = 0;
    o->water_density = 1025.0;
    o->water_drag_coeff = 5.5e-3;
    o->air_density = 1.3;
    o->air_drag_coeff = 1.2e-3;
    o->wind_kind = ICEMPM_WIND_NONE;
}

int icempm_create(const icempm_simparams_t *prms, const uint8_t *grid_status, const double *current_vxvy,
                  uint32_t capacity, const icempm_options_t *opts, icempm_t **out)
{
    if (!out) return fail(ICEMPM_E_ARG, "out is null");
    *out = nullptr;
    if (!prms || !grid_status) return fail(ICEMPM_E_ARG, "prms and grid_status are required");
    icempm_options_t o;
    if (opts) o = *opts; else icempm_default_options(&o);
    if (o.block_threads != 0 && o.block_threads != 128)
        return fail(ICEMPM_E_UNSUPPORTED, "block_threads must be 0 or 128");
    if (o.forcing != ICEMPM_FORCING_COMPAT && o.forcing != ICEMPM_FORCING_EXTENDED)
        return fail(ICEMPM_E_ARG, "unknown forcing");
    icempm::Engine *e = nullptr;
    switch (o.variant) {
    case ICEMPM_VARIANT_FIXED: e = icempm::make_engine_fixed(); break;
    case ICEMPM_VARIANT_FP32: e = icempm::make_engine_fp32(); break;
    case ICEMPM_VARIANT_FP64: e = icempm::make_engine_fp64(); break;
    case ICEMPM_VARIANT_TEXTBOOK: e = icempm::make_engine_fp32(); break;   // FP32 engine, textbook step
    default: return fail(ICEMPM_E_ARG, "unknown variant");
    }
    icempm_context *c = new (std::nothrow) icempm_context;
    if (!c) { delete e; return fail(ICEMPM_E_NOMEM, "context allocation failed"); }
    c->eng = e;
    c->prms = *prms;
    c->opts = o;
    int rc;
    try {
        rc = e->init(*prms, grid_status, current_vxvy, capacity, o);
    } catch (...) {
        rc = fail(ICEMPM_E_STATE, "exception during init");
    }
    if (rc) { delete e; delete c; return rc; }
    *out = c;
    icempm::g_last_error.clear();
    return ICEMPM_OK;
}

int icempm_destroy(icempm_t *ctx)
{
    if (!ctx) return ICEMPM_OK;
    delete ctx->eng;
    delete ctx;
    return ICEMPM_OK;
}

int icempm_upload_points(icempm_t *ctx, const double *hssoa, uint32_t capacity, uint32_t size, int32_t disabled_count)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!hssoa && size) return fail(ICEMPM_E_ARG, "hssoa is null");
    ICEMPM_TRY(ctx->eng->upload(hssoa, capacity, size, disabled_count));
}

int icempm_update_constants(icempm_t *ctx, const icempm_simparams_t *prms)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!prms) return fail(ICEMPM_E_ARG, "prms is null");
    if (prms->GridXTotal != ctx->prms.GridXTotal || prms->GridYTotal != ctx->prms.GridYTotal)
        return fail(ICEMPM_E_ARG, "grid size cannot change after create");
    ctx->prms = *prms;
    ICEMPM_TRY(ctx->eng->update_constants(*prms));
}

int icempm_set_current(icempm_t *ctx, const double *current_vxvy)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_current(current_vxvy));
}

int icempm_set_flow_frames(icempm_t *ctx, const double *current_a, const double *current_b)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_flow_frames(current_a, current_b));
}

int icempm_set_wind_frames(icempm_t *ctx, const float *wind, int32_t rows, int32_t cols, double cell, double x0,
                           double y0)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_wind_frames(wind, rows, cols, cell, x0, y0));
}

int icempm_set_forcing_time(icempm_t *ctx, double tc, double tw)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_forcing_time(tc, tw));
}

int icempm_get_forcing(icempm_t *ctx, double *current_vxvy, double *wind_stress_xy)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->get_forcing(current_vxvy, wind_stress_xy));
}

int icempm_step(icempm_t *ctx, int32_t nsteps, int32_t first_step)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->step(nsteps, first_step));
}

int icempm_download_points(icempm_t *ctx, double *hssoa, uint32_t capacity, uint32_t *size)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!hssoa) return fail(ICEMPM_E_ARG, "hssoa is null");
    ICEMPM_TRY(ctx->eng->download(hssoa, capacity, size));
}

int icempm_download_points_async(icempm_t *ctx, double *hssoa, uint32_t capacity, uint32_t *size)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!hssoa) return fail(ICEMPM_E_ARG, "hssoa is null");
    ICEMPM_TRY(ctx->eng->download_async(hssoa, capacity, size));
}

int icempm_download_wait(icempm_t *ctx)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->download_wait());
}

int icempm_get_status(icempm_t *ctx, uint32_t *error_bits, int32_t *disabled_count)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->status(error_bits, disabled_count));
}

int icempm_clear_force_accumulator(icempm_t *ctx)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->clear_forces());
}

int icempm_get_boundary_forces(icempm_t *ctx, double *fxfy, int32_t elapsed_steps)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!fxfy) return fail(ICEMPM_E_ARG, "fxfy is null");
    if (elapsed_steps <= 0) return fail(ICEMPM_E_ARG, "elapsed_steps must be > 0");
    ICEMPM_TRY(ctx->eng->forces(fxfy, elapsed_steps));
}

int icempm_sort_compact(icempm_t *ctx)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->sort_compact());
}

int icempm_timings(icempm_t *ctx, float ms[4])
{
    ICEMPM_GUARD_CTX(ctx);
    if (!ms) return fail(ICEMPM_E_ARG, "ms is null");
    ICEMPM_TRY(ctx->eng->timings(ms));
}

int icempm_phase_times(icempm_t *ctx, int32_t nsteps, float *update_ms, float *fused_ms)
{
    ICEMPM_GUARD_CTX(ctx);
    if (nsteps <= 0 || !update_ms || !fused_ms) return fail(ICEMPM_E_ARG, "bad arguments");
    ICEMPM_TRY(ctx->eng->phase_times(nsteps, update_ms, fused_ms));
}

int icempm_point_count(icempm_t *ctx, uint32_t *n)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!n) return fail(ICEMPM_E_ARG, "n is null");
    *n = ctx->eng->count();
    return ICEMPM_OK;
}

int icempm_get_stream(icempm_t *ctx, void **stream)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!stream) return fail(ICEMPM_E_ARG, "stream is null");
    *stream = (void *)ctx->eng->stream();
    return ICEMPM_OK;
}

int icempm_launch_count(icempm_t *ctx, uint64_t *count)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!count) return fail(ICEMPM_E_ARG, "count is null");
    *count = ctx->eng->launches();
    return ICEMPM_OK;
}

int icempm_fixed_point_scales(icempm_t *ctx, double *scale_mass, double *scale_momentum)
{
    ICEMPM_GUARD_CTX(ctx);
    if (scale_mass) *scale_mass = ctx->eng->fixed_scale_m();
    if (scale_momentum) *scale_momentum = ctx->eng->fixed_scale_p();
    return ICEMPM_OK;
}

int icempm_host_register(void *ptr, size_t bytes)
{
    if (!ptr || !bytes) return fail(ICEMPM_E_ARG, "null or empty range");
    cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
    if (e != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string("cudaHostRegister: ") + cudaGetErrorString(e));
    return ICEMPM_OK;
}

int icempm_host_unregister(void *ptr)
{
    cudaError_t e = cudaHostUnregister(ptr);
    if (e != cudaSuccess) return fail(ICEMPM_E_CUDA, std::string("cudaHostUnregister: ") + cudaGetErrorString(e));
    return ICEMPM_OK;
}

int icempm_device_count(int *count)
{
    if (!count) return fail(ICEMPM_E_ARG, "count is null");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) { *count = 0; return fail(ICEMPM_E_CUDA, cudaGetErrorString(e)); }
    return ICEMPM_OK;
}

int icempm_prepare_frame(icempm_t *ctx, const uint32_t *point_colors_rgb, uint32_t ncolors, int32_t elapsed_steps,
                         icempm_frame_t *out)
{
    ICEMPM_GUARD_CTX(ctx);
    if (!out) return fail(ICEMPM_E_ARG, "out is null");
    ICEMPM_TRY(ctx->eng->prepare_frame(point_colors_rgb, ncolors, elapsed_steps, out));
}

int icempm_harvest_begin(icempm_t *ctx, uint32_t capacity, int32_t stride)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->harvest_begin(capacity, stride));
}

int icempm_harvest_end(icempm_t *ctx, float *records, uint32_t capacity, uint32_t *count)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->harvest_end(records, capacity, count));
}

int icempm_set_learned_map(icempm_t *ctx, const float *d_params, const float *d_norm, float tol)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_learned_map(d_params, d_norm, tol));
}

int icempm_learned_map_counts(icempm_t *ctx, uint64_t *kept, uint64_t *fallbacks)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->learned_counts(kept, fallbacks));
}

int icempm_tune_sort_cadence(icempm_t *ctx, int32_t trial_steps, int32_t first_step, int32_t *sort_every)
{
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->tune_sort(trial_steps, first_step, sort_every));
}

int icempm_debug_barrier_timeout(icempm_t *ctx, uint32_t extra_bytes, uint32_t wait_limit_us)
{
    if (extra_bytes % 16u != 0) return fail(ICEMPM_E_ARG, "extra_bytes must be a multiple of 16");
    ICEMPM_GUARD_CTX(ctx);
    ICEMPM_TRY(ctx->eng->set_barrier_test(extra_bytes, wait_limit_us));
}

int icempm_batch_create(icempm_t *const *contexts, int32_t count, icempm_batch_t **out)
{
    if (!out) return fail(ICEMPM_E_ARG, "out is null");
    *out = nullptr;
    if (!contexts || count < 1) return fail(ICEMPM_E_ARG, "at least one context is required");
    std::vector<icempm::Engine *> eng((size_t)count);
    for (int i = 0; i < count; i++) {
        if (!contexts[i] || !contexts[i]->eng) return fail(ICEMPM_E_ARG, "null context in the batch");
        if (contexts[i]->opts.variant != contexts[0]->opts.variant)
            return fail(ICEMPM_E_ARG, "all contexts of a batch must use the same variant");
        eng[i] = contexts[i]->eng;
    }
    icempm::Batch *b = nullptr;
    try {
        switch (contexts[0]->opts.variant) {
        case ICEMPM_VARIANT_FIXED: b = icempm::make_batch_fixed(eng.data(), count); break;
        case ICEMPM_VARIANT_FP32: b = icempm::make_batch_fp32(eng.data(), count); break;
        case ICEMPM_VARIANT_FP64: b = icempm::make_batch_fp64(eng.data(), count); break;
        default: return fail(ICEMPM_E_ARG, "batches take the fixed, fp32 or fp64 variant");
        }
    } catch (const std::bad_alloc &) {
        return fail(ICEMPM_E_NOMEM, "host allocation failed");
    }
    if (!b) return ICEMPM_E_STATE;
    icempm_batch *bt = new (std::nothrow) icempm_batch;
    if (!bt) { delete b; return fail(ICEMPM_E_NOMEM, "batch allocation failed"); }
    bt->b = b;
    *out = bt;
    return ICEMPM_OK;
}

int icempm_batch_destroy(icempm_batch_t *batch)
{
    if (!batch) return ICEMPM_OK;
    delete batch->b;
    delete batch;
    return ICEMPM_OK;
}

int icempm_batch_step(icempm_batch_t *batch, int32_t nsteps, int32_t first_step)
{
    ICEMPM_GUARD_BATCH(batch);
    ICEMPM_TRY(batch->b->step(nsteps, first_step));
}

int icempm_batch_autotune(icempm_batch_t *batch, int32_t trial_steps, int32_t first_step, icempm_batch_tuning_t *out)
{
    ICEMPM_GUARD_BATCH(batch);
    ICEMPM_TRY(batch->b->autotune(trial_steps, first_step, out));
}

int icempm_batch_set_tuning(icempm_batch_t *batch, const icempm_batch_tuning_t *tuning)
{
    ICEMPM_GUARD_BATCH(batch);
    if (!tuning) return fail(ICEMPM_E_ARG, "tuning is null");
    ICEMPM_TRY(batch->b->set_tuning(tuning));
}

int icempm_batch_get_tuning(icempm_batch_t *batch, icempm_batch_tuning_t *tuning)
{
    ICEMPM_GUARD_BATCH(batch);
    if (!tuning) return fail(ICEMPM_E_ARG, "tuning is null");
    ICEMPM_TRY(batch->b->get_tuning(tuning));
}

int icempm_batch_timings(icempm_batch_t *batch, float ms[4])
{
    ICEMPM_GUARD_BATCH(batch);
    if (!ms) return fail(ICEMPM_E_ARG, "ms is null");
    ICEMPM_TRY(batch->b->timings(ms));
}

int icempm_batch_launch_count(icempm_batch_t *batch, uint64_t *count)
{
    ICEMPM_GUARD_BATCH(batch);
    if (!count) return fail(ICEMPM_E_ARG, "count is null");
    *count = batch->b->launches();
    return ICEMPM_OK;
}

const char *icempm_last_error(void) { return icempm::g_last_error.c_str(); }

}  // extern "C"
