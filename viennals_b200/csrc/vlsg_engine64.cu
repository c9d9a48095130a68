// vlsg_engine64.cu -- the FP64 engine.  Compiled without contraction of
// multiplies and adds (-fmad=false), with IEEE division and square root, so
// every rule rounds as the reference's Advect<double,3> does.
#include "vlsg_engine.cuh"

namespace vlsg {
EngineBase *makeEngineF64() { return new Engine<double>(); }
} // namespace vlsg
