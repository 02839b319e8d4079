// cuda_texture_types.h -- host stand-in (TEST INFRASTRUCTURE): everything lives in cuda_runtime.h.
#include "cuda_runtime.h"
