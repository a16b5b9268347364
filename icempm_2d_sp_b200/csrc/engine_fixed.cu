// FP32 point state, int64 fixed-point P2G accumulation (deterministic).
#include "engine_host.cuh"
namespace icempm { Engine *make_engine_fixed() { return new EngineT<float, long long>(); } }
