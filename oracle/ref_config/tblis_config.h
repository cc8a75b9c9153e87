/* Hand-written configuration header for compiling the TBLIS reference sources
 * directly (without running its autotools build). It defines what the
 * reference's configure step would: index types (ptrdiff_t / char, the
 * reference defaults in configure.ac:91-123) and the host feature macros. */
#ifndef _TBLIS_CONFIG_H_ORACLE
#define _TBLIS_CONFIG_H_ORACLE
#include <stddef.h>
#define TBLIS_LEN_TYPE ptrdiff_t
#define TBLIS_STRIDE_TYPE ptrdiff_t
#define TBLIS_LABEL_TYPE char
#define TBLIS_RESTRICT __restrict__
#define TBLIS_HAVE_SYSCONF 1
#define TBLIS_HAVE__SC_NPROCESSORS_CONF 1
#define TBLIS_HAVE__SC_NPROCESSORS_ONLN 1
#define TBLIS_HAVE_LSCPU 1
#define TBLIS_TOPDIR "."
#endif
