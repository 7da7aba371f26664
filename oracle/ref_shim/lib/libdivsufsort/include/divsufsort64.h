/* Build shim: libdivsufsort is only needed by `hera index -g` (genome
 * FM-index, out of scope).  Declares the one type and function the reference
 * names; the stub aborts if the genome index path is ever taken. */
#ifndef HERA_SHIM_DIVSUFSORT64_H
#define HERA_SHIM_DIVSUFSORT64_H
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
typedef int64_t saidx64_t;
typedef int32_t saint_t;
static inline saint_t divsufsort64(const unsigned char *T, saidx64_t *SA, saidx64_t n)
{
	(void)T; (void)SA; (void)n;
	fprintf(stderr, "divsufsort64: genome index is not part of the oracle build\n");
	abort();
	return -1;
}
#endif
