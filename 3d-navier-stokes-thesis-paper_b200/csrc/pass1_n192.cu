// pass-1 register-FFT kernels for transform length 192
#define NSIZE 192
#include "pass1_fast.inc"
