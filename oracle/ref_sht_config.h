/* Build configuration for compiling the reference SHTns 3.5.2 CPU sources into
 * the oracle library (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
 * Written for this project from the option list of the reference's
 * sht_config.h.in: an OpenMP build with explicit SIMD, Ishioka's recurrence,
 * and the multi-threaded FFTW interface (provided here by oracle/fftw_shim.c). */
#define HAVE_COMPLEX_H 1
#define HAVE_MATH_H 1
#define HAVE_STDIO_H 1
#define HAVE_STDLIB_H 1
#define HAVE_STRING_H 1
#define HAVE_LIBM 1
#define HAVE_LIBFFTW3 1
#define HAVE_LIBFFTW3_OMP 1
#define SHTNS_ISHIOKA 1
#define SHT_VERBOSE 1
#define _GCC_VEC_ 1
#define PACKAGE_VERSION "3.5.2"
