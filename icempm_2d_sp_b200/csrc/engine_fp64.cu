// FP64 point state and arithmetic, FP64 atomics.
#include "engine_host.cuh"
namespace icempm { Engine *make_engine_fp64() { return new EngineT<double, double>(); } }
