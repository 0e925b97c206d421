// pass-1 register-FFT kernels for transform length 72
#define NSIZE 72
#include "pass1_fast.inc"
