// pass-1 register-FFT kernels for transform length 384
#define NSIZE 384
#include "pass1_fast.inc"
