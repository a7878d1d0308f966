/* Force-included when compiling the reference's Sim.cu on Linux: it calls the
 * MSVC-only fopen_s (Sim.cu:5029,5046). TEST INFRASTRUCTURE ONLY. */
#pragma once
#include <cerrno>
#include <cstdio>
static inline int fopen_s(FILE** f, const char* path, const char* mode) {
    *f = std::fopen(path, mode);
    return *f ? 0 : errno;
}
