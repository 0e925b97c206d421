// pass-1 register-FFT kernels for transform length 24
#define NSIZE 24
#include "pass1_fast.inc"
