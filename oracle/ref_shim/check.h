/* Test-infrastructure stand-in for the parent project's check.h (missing from
 * the reference tree; included at LinearBasis/gold/include/Data.h:13).  The
 * macros abort on a non-zero status, which is what the parent's versions do. */
#ifndef ORACLE_REF_CHECK_H
#define ORACLE_REF_CHECK_H
#include <cstdio>
#include <cstdlib>
#define MPI_ERR_CHECK(call) do { int e_ = (call); if (e_ != 0) { \
	fprintf(stderr, "MPI error %d at %s:%d\n", e_, __FILE__, __LINE__); abort(); } } while (0)
#define PTHREAD_ERR_CHECK(call) MPI_ERR_CHECK(call)
#endif
