// vlsg_engine32.cu -- the FP32 engine.  Compiled with fused multiply-add:
// its results are compared with the FP64 path within a tolerance, not bit
// for bit.
#include "vlsg_engine.cuh"

namespace vlsg {
EngineBase *makeEngineF32() { return new Engine<float>(); }
} // namespace vlsg
