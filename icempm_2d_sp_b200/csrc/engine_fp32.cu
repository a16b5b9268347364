// FP32 point state, FP32 atomics.
#include "batch.cuh"
namespace icempm { Engine *make_engine_fp32() { return new EngineT<float, float>(); } }
namespace icempm { Batch *make_batch_fp32(Engine *const *e, int n) { return make_batch_t<float, float>(e, n); } }
