/*
 * Hand-written configuration header for compiling the reference libflame
 * sources directly with gcc (oracle/Makefile.ref), standing in for the file
 * that the reference's configure script would generate from
 * build/FLA_config.h.in.  The settings mirror a configure run with
 *   --enable-builtin-blas --enable-lapack2flame --enable-legacy-lapack
 *   --disable-ldim-alignment --enable-non-critical-code
 *   --enable-internal-error-checking=full --enable-portable-timer
 * and, when FLA_REF_SUPERMATRIX is defined by the Makefile,
 *   --enable-multithreading=openmp --enable-supermatrix.
 * Test infrastructure only: this configures the CPU oracle build.
 */
#ifndef FLA_CONFIG_H
#define FLA_CONFIG_H

#define FLA_ENABLE_BUILTIN_BLAS 1
#define FLA_ENABLE_LAPACK2FLAME 1
#define FLA_ENABLE_LEGACY_LAPACK 1
#define FLA_ENABLE_NON_CRITICAL_CODE 1
#define FLA_ENABLE_INTERNAL_ERROR_CHECKING 1
#define FLA_INTERNAL_ERROR_CHECKING_LEVEL 2
#define FLA_ENABLE_BLIS1_USE_OF_FLA_MALLOC 1
#define FLA_ENABLE_PORTABLE_TIMER 1
#define FLA_PORTABLE_TIMER_IS_CLOCK_GETTIME 1
#define FLA_MEMORY_ALIGNMENT_BOUNDARY 16
#define FLA_VECTOR_INTRINSIC_TYPE 0
#define FLA_DEFAULT_M_BLOCKSIZE 128
#define FLA_DEFAULT_K_BLOCKSIZE 128
#define FLA_DEFAULT_N_BLOCKSIZE 128
#define BLIS1_FROM_LIBFLAME 1

#ifdef FLA_REF_SUPERMATRIX
#define FLA_ENABLE_MULTITHREADING 1
#define FLA_MULTITHREADING_MODEL 1
#define FLA_ENABLE_SUPERMATRIX 1
#else
#define FLA_MULTITHREADING_MODEL 0
#endif

#define HAVE_ASSERT_H 1
#define HAVE_FCNTL_H 1
#define HAVE_INTTYPES_H 1
#define HAVE_LIBM 1
#define HAVE_MATH_H 1
#define HAVE_MEMORY_H 1
#define HAVE_SIGNAL_H 1
#define HAVE_STDINT_H 1
#define HAVE_STDLIB_H 1
#define HAVE_STRINGS_H 1
#define HAVE_STRING_H 1
#define HAVE_SYS_STAT_H 1
#define HAVE_SYS_TIME_H 1
#define HAVE_SYS_TYPES_H 1
#define HAVE_UNISTD_H 1
#define TIME_WITH_SYS_TIME 1
#define PROTOTYPES 1
#define STDC_HEADERS 1
#ifndef _GNU_SOURCE
#define _GNU_SOURCE 1
#endif

#endif
