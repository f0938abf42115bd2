// Fused basis-column evaluation engine (passes of up to four gates per HBM round trip).
#pragma once

#include "engine.h"

namespace rqc {

// Same contract as evaluate() (engine.h); maxk = gates fused per pass (1..4).
int evaluate_fused(Runtime& rt, const CircuitSpec& c, const TargetSpec& t, int mode, int precision, int maxk,
                   double2* d_out);

}  // namespace rqc
