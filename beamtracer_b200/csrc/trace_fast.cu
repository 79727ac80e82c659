// The trajectory tracer of trace.cu compiled with contracted multiply-adds (--fmad=true):
// the same step, each a * b + c one fused multiply-add rounded once, so the trajectories
// agree with the exact build (and the oracle) to rounding, not bit for bit, with a shorter
// chain of dependent FP64 instructions a step.  Its entry points end in _fast.
#define BT_TRACE_FAST 1
#include "trace.cu"
