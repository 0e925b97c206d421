// pass-1 register-FFT kernels for transform length 576
#define NSIZE 576
#include "pass1_fast.inc"
