/* FP64 build of the CPU oracle (test infrastructure only; see rmg_oracle.h). */
#include "rmg_oracle.h"
#define REAL double
#define P ora64_
#include "rmg_oracle_impl.h"
