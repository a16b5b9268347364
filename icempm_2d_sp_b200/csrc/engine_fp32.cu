// FP32 point state, FP32 atomics.
#include "engine_host.cuh"
namespace icempm { Engine *make_engine_fp32() { return new EngineT<float, float>(); } }
