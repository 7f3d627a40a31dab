/* Hand-written build configuration for compiling the reference library in the
 * oracle build (stands in for the header its CMake would configure).  Only the
 * platform facts of this image are set; every optional feature stays off. */
#include "hmat/config.h"
#define HAVE_STDINT_H 1
#define HAVE_UNISTD_H 1
#define HAVE_SYS_TYPES_H 1
#define HAVE_TIME_H 1
#define HAVE_SYS_RESOURCE_H 1
#define HAVE_LIBRT 1
#define HAVE_GOTO_GET_NUM_PROCS 1
#define HAVE_OPENBLAS_SET_NUM_THREADS 1
#if defined(HAVE_GOTO_GET_NUM_PROCS) && defined(HAVE_OPENBLAS_SET_NUM_THREADS)
#define OPENBLAS_DISABLE_THREADS
#endif
