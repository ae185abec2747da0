/* Hand-written configuration for building the reference library from its own
 * sources with the generic FP64-accumulating DFT backend (no FFTW3, no MPI,
 * no OpenCL).  This stands in for the header that the reference's autoconf
 * step would generate (configure.ac), which cannot run here.  It only selects
 * features; it contains no reference code. */
#ifndef FCB_REF_CONFIG_HPP
#define FCB_REF_CONFIG_HPP

#define OVXX_DFT_FFT 1
#define OVXX_TIMER_POSIX 1
#define OVXX_ALLOC_ALIGNMENT 32
#define OVXX_HAS_EXCEPTIONS 1
#define VSIP_HAS_EXCEPTIONS 1
#define HAVE_STD_ISFINITE 1
#define HAVE_STD_ISNAN 1
#define HAVE_STD_ISNORMAL 1
#define OVXX_DEFAULT_COMPLEX_STORAGE_SPLIT 0
#define VSIP_BIG_ENDIAN 0

#define SIZEOF_CHAR 1
#define SIZEOF_SHORT 2
#define SIZEOF_INT 4
#define SIZEOF_LONG 8
#define SIZEOF_LONG_LONG 8
#define SIZEOF_FLOAT 4
#define SIZEOF_DOUBLE 8
#define SIZEOF_LONG_DOUBLE 16

#endif
