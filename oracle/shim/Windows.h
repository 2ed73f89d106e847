/* Minimal stand-in for <Windows.h> so the reference's sources compile with
   gcc/nvcc on Linux.  Only the directory helpers used by the reference's VTU
   writer (inOut.cpp) are provided. */
#pragma once
#include <errno.h>
#include <sys/stat.h>
#define ERROR_ALREADY_EXISTS EEXIST
static inline int CreateDirectoryA(const char* path, void* unused)
{
    (void)unused;
    return mkdir(path, 0755) == 0;
}
static inline int GetLastError(void) { return errno; }
