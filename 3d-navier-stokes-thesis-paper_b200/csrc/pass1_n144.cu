// pass-1 register-FFT kernels for transform length 144
#define NSIZE 144
#include "pass1_fast.inc"
