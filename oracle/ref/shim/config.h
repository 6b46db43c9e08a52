/* Hand-written stand-in for the autoconf-generated config.h of the MAOS
 * reference build.  Test infrastructure only: it lets the reference CPU path
 * compile with a plain Makefile (oracle/ref/Makefile). */
#ifndef MAOSREF_SHIM_CONFIG_H
#define MAOSREF_SHIM_CONFIG_H
#define BIGENDIAN 0
#define SRCDIR "/nonexistent/maos-src"
#define BUILDDIR "/nonexistent/maos-build"
#define LDSUFFIX "so"
#define DEBUG 0
#define HAS_OPENMP 1
#define MAOS_DISABLE_SCHEDULER 1
#define USE_STATIC 0
#define HAS_FFTWF 1
#define BUILTIN_FFTW_THREADS 1
#define HAS_LWS 0
#define USE_CUDA 0
#define CUDA_DOUBLE 0
#define GIT_VERSION "reference-oracle-build"
#define PACKAGE_VERSION "1.0"
#define PACKAGE "maos"
#endif
