// curand_kernel.h -- HOST STAND-IN (TEST INFRASTRUCTURE: the reference-pinned oracle under
// oracle/_ref).  The reference seeds one XORWOW state per pixel with clock64()
// (`curand_init(clock64(), p.y, p.x, &state)`, DPE.cu:1024-1037), so no two of its runs draw the
// same numbers.  Here the state is a Philox4x32-10 counter stream (Salmon, Moraes, Dror, Shaw,
// SC'11), the stream the oracle and the CUDA kernels use: draw n of pixel p = y * W + x is word 0
// of philox({n, p, 0x5EED, 0}, key = the harness's seed), and curand_uniform maps a word u to
// ((u >> 8) + 1) * 2^-24, in (0, 1] like curand_uniform.  The clock64() seed is ignored; W and the
// key come from the harness (ref_rng_configure).
#ifndef REFSHIM_CURAND_KERNEL_H_
#define REFSHIM_CURAND_KERNEL_H_

#include "cuda_runtime.h"

struct curandStateXORWOW {
  unsigned int pixel;
  unsigned int counter;
};
typedef struct curandStateXORWOW curandState;

void ref_rng_configure(int width, unsigned long long seed);
void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long offset, curandState *state);
unsigned int curand(curandState *state);
float curand_uniform(curandState *state);

#endif
