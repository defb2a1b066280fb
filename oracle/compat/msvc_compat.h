/* Test infrastructure only (oracle build): force-included when the reference's
 * MSVC-only headers are compiled with g++ on Linux.
 *
 * The reference (FEM/, MsFEM/, Library/) calls the MSVC "secure" CRT variants
 * (printf_s, fopen_s, sprintf_s with and without an explicit size, sscanf_s,
 * mbstowcs_s), CLK_TCK and CreateDirectory, and relies on MSVC resolving
 * abs(double) to the floating-point overload.  Under g++ without `using std::abs`
 * the call in Library/GeometryShape.h:1688 binds to C int abs(int) and every
 * tetrahedron volume truncates to zero, so this header pulls std::abs into the
 * global namespace before any reference header is seen.
 *
 * Standard headers are included here, before Library/Math.h defines its
 * function-like `max` macro (Library/Math.h:13-15), so libstdc++ is unaffected.
 */
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <cwchar>
#include <functional>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <vector>
#include <sys/stat.h>
#include <unistd.h>

using std::abs;

#define printf_s printf
#define fprintf_s fprintf
#define scanf_s scanf
#define fscanf_s fscanf
#define sscanf_s sscanf
#define CLK_TCK CLOCKS_PER_SEC

typedef const char* LPCTSTR;

static inline int fopen_s(FILE** f, const char* name, const char* mode)
{
    *f = std::fopen(name, mode);
    return *f ? 0 : 1;
}

/* The reference's headers pass a wide string cast to LPCTSTR (MsFEM/MsFEM.h:600-601,
 * MsFEM/MsFEM_Grid.h:4810-4811) and write into the directory right after: create it. */
static inline int CreateDirectory(LPCTSTR p, void*)
{
    if (!p) return 0;
    char buf[4096];
    if (p[0] != 0 && p[1] == 0) {
        const size_t k = std::wcstombs(buf, reinterpret_cast<const wchar_t*>(p), sizeof(buf) - 1);
        if (k == (size_t)-1) return 0;
        buf[k] = 0;
    } else {
        std::snprintf(buf, sizeof(buf), "%s", p);
    }
    return ::mkdir(buf, 0755) == 0;
}

static inline int mbstowcs_s(size_t* out_len, wchar_t* dst, size_t dst_len, const char* src, size_t)
{
    size_t k = std::mbstowcs(dst, src, dst_len);
    if (out_len) *out_len = k;
    return 0;
}

/* sprintf_s(buffer_array, fmt, ...) : size deduced from the array type */
template <size_t N, class... A>
static inline int sprintf_s(char (&buf)[N], const char* fmt, A... args)
{
    return std::snprintf(buf, N, fmt, args...);
}

/* sprintf_s(ptr, size, fmt, ...) */
static inline int sprintf_s(char* buf, size_t n, const char* fmt, ...)
{
    va_list v;
    va_start(v, fmt);
    int r = std::vsnprintf(buf, n, fmt, v);
    va_end(v);
    return r;
}
