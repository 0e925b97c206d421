// pass-1 register-FFT kernels for transform length 288
#define NSIZE 288
#include "pass1_fast.inc"
