/* stand-in, test infrastructure only (see hip_runtime.h) */
#include "hip_runtime.h"
