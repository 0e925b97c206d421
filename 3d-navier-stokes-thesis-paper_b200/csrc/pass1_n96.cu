// pass-1 register-FFT kernels for transform length 96
#define NSIZE 96
#include "pass1_fast.inc"
