// Host helpers of the drop-in classes, with the names and the error
// behaviour of the reference's common.hh (common.cc:1-60): a fatal error
// prints its message and exits with the given status.
#ifndef VDI_HOST_COMMON_HH
#define VDI_HOST_COMMON_HH

#include <cstdio>

void fatal_error(const char* p, int code);
FILE* safe_fopen(const char* filename, const char* mode);
void safe_fread(void* ptr, size_t size, size_t count, FILE* fp, const char* p);
/** Wall-clock seconds (the reference's wtime). */
double wtime();
/** Exits through fatal_error when a C-ABI call returned an error. */
void vdi_check(int status, const char* where);

#endif
