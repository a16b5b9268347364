// FP64 point state and arithmetic, FP64 atomics.
#include "batch.cuh"
namespace icempm { Engine *make_engine_fp64() { return new EngineT<double, double>(); } }
namespace icempm { Batch *make_batch_fp64(Engine *const *e, int n) { return make_batch_t<double, double>(e, n); } }
