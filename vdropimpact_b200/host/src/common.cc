// Host helpers with the reference's error behaviour (common.cc:1-60).
#include "common.hh"

#include <chrono>
#include <cstdlib>

#include "vdi.h"

FILE* safe_fopen(const char* filename, const char* mode) {
    FILE* f = fopen(filename, mode);
    if (f == NULL) {
        fprintf(stderr, "Error opening file \"%s\"\n", filename);
        exit(1);
    }
    return f;
}

void safe_fread(void* ptr, size_t size, size_t count, FILE* fp, const char* p) {
    if (fread(ptr, size, count, fp) != count) {
        fprintf(stderr, "Can't read %s from file\n", p);
        exit(1);
    }
}

void fatal_error(const char* p, int code) {
    fprintf(stderr, "Error: %s\n", p);
    exit(code);
}

double wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void vdi_check(int status, const char* where) {
    if (status == VDI_OK) return;
    char msg[768];
    snprintf(msg, sizeof(msg), "%s: %s (%s)", where, vdi_status_string(status), vdi_last_error());
    fatal_error(msg, 1);
}
