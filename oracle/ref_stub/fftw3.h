/* Empty stand-in: the CPU device backend header includes <fftw3.h>, but the
 * short-range nonbonded path makes no FFT call. */
