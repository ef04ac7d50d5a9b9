/* cufftw.h (host stand-in): the reference includes this name; it only needs
 * the cuFFT API, see cufft.h.  TEST INFRASTRUCTURE ONLY. */
#include "cufft.h"
