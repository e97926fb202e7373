/* Host-only stand-in for <cuda.h>; see cuda_runtime.h in this folder. */
#include "cuda_runtime.h"
