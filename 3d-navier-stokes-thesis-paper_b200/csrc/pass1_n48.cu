// pass-1 register-FFT kernels for transform length 48
#define NSIZE 48
#include "pass1_fast.inc"
