/* Test helper (LD_PRELOAD): the reference's sample driver sample_binary_file.cu reads and
 * writes fixed paths under "/path/to/" (its placeholders for the user's files).  This shim
 * interposes fopen and redirects those paths to the directory named by CEEMDAN_PATH_DIR, so
 * the unmodified driver runs in a test's temporary directory.  Other paths are untouched. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

FILE* fopen(const char* path, const char* mode) {
    static FILE* (*real_fopen)(const char*, const char*) = NULL;
    if (!real_fopen) real_fopen = (FILE * (*)(const char*, const char*)) dlsym(RTLD_NEXT, "fopen");
    const char* prefix = "/path/to/";
    const char* dir = getenv("CEEMDAN_PATH_DIR");
    if (dir && path && strncmp(path, prefix, strlen(prefix)) == 0) {
        char buf[4096];
        snprintf(buf, sizeof(buf), "%s/%s", dir, path + strlen(prefix));
        return real_fopen(buf, mode);
    }
    return real_fopen(path, mode);
}
