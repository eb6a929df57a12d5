/* FP32 (IEEE, no fast-math) build of the CPU oracle (test infrastructure only; see rmg_oracle.h). */
#include "rmg_oracle.h"
#define REAL float
#define P ora32_
#include "rmg_oracle_impl.h"
