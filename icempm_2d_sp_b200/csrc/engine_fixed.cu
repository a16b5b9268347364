// FP32 point state, int64 fixed-point P2G accumulation (deterministic).
#include "batch.cuh"
namespace icempm { Engine *make_engine_fixed() { return new EngineT<float, long long>(); } }
namespace icempm { Batch *make_batch_fixed(Engine *const *e, int n) { return make_batch_t<float, long long>(e, n); } }
