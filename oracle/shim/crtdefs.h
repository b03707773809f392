/* Oracle build shim (test infrastructure only).
 *
 * The reference's include/Image_Type.h:8 includes the MSVC header <crtdefs.h>.
 * On Linux this stand-in supplies the standard headers the reference relies on
 * implicitly and a `_splitpath_s` used by FilterIO::generate_OPath
 * (include/Filter.h:242), which is CLI-only and never called on the BM3D path. */
#ifndef ORACLE_SHIM_CRTDEFS_H_
#define ORACLE_SHIM_CRTDEFS_H_

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <cmath>
#include <string>
#include <vector>
#include <algorithm>
#include <type_traits>
#include <utility>
#include <iostream>

inline int _splitpath_s(const char *path, char *drive, size_t, char *dir, size_t,
                        char *fname, size_t, char *ext, size_t)
{
    /* Minimal POSIX split: no drive letters. */
    const char *slash = std::strrchr(path, '/');
    const char *base = slash ? slash + 1 : path;
    const char *dot = std::strrchr(base, '.');
    drive[0] = '\0';
    size_t dlen = static_cast<size_t>(base - path);
    std::memcpy(dir, path, dlen);
    dir[dlen] = '\0';
    size_t flen = dot ? static_cast<size_t>(dot - base) : std::strlen(base);
    std::memcpy(fname, base, flen);
    fname[flen] = '\0';
    std::strcpy(ext, dot ? dot : "");
    return 0;
}

#endif
