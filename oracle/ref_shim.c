/* Test-infrastructure shim: compiles the reference's single-header library
 * (include/notorious_fft.h of NotoriousLOB/Notorious-FFT) into a shared object
 * under oracle/_ref/.  Nothing in this file is product code; only the tests,
 * smoke() and the CPU-baseline leg of bench.py load the result. */
#define NOTORIOUS_FFT_IMPLEMENTATION
#include "notorious_fft.h"
