// Portability shim force-included (-include) when compiling the reference renderer's C++
// sources on Linux for the oracle. It maps the two Windows-only CRT calls the reference uses
// (_wfopen in medium.cpp:131, integrator.cpp:37/59, image.cpp:217/300, import_pbrt.cpp:601;
// _fseeki64 in image.cpp:285) onto their POSIX equivalents. No reference source is edited.
#pragma once
#ifdef __cplusplus
#include <cstdio>
#include <cstdlib>
#include <cwchar>
#include <string>
#include <sys/types.h>
inline FILE *_wfopen(const wchar_t *path, const wchar_t *mode) {
    std::string p, m;
    for (const wchar_t *c = path; *c; ++c) p.push_back(char(*c));
    for (const wchar_t *c = mode; *c; ++c) m.push_back(char(*c));
    return std::fopen(p.c_str(), m.c_str());
}
inline int _fseeki64(FILE *f, long long off, int whence) { return fseeko(f, off_t(off), whence); }
#endif
