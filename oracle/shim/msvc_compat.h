/*
 * Bounded-string helpers with the MSVC array-template signatures the
 * reference calls (strcpy_s/strcat_s/sprintf_s on char arrays, e.g.
 * main.cpp:15, airpore.cpp:472-477,681-685,940). Force-included when the
 * reference is compiled as the CPU oracle; not part of the product.
 */
#ifndef ORACLE_SHIM_MSVC_COMPAT_H
#define ORACLE_SHIM_MSVC_COMPAT_H
#ifdef __cplusplus
#include <cstddef>
#include <cstdio>
#include <cstring>

template <std::size_t N>
inline int strcpy_s(char (&dst)[N], const char *src)
{
    std::size_t n = std::strlen(src);
    if (n >= N) n = N - 1;
    std::memcpy(dst, src, n);
    dst[n] = '\0';
    return 0;
}

template <std::size_t N>
inline int strcat_s(char (&dst)[N], const char *src)
{
    std::size_t used = std::strlen(dst);
    std::size_t n = std::strlen(src);
    if (used + n >= N) n = N - 1 - used;
    std::memcpy(dst + used, src, n);
    dst[used + n] = '\0';
    return 0;
}

template <std::size_t N, typename... Args>
inline int sprintf_s(char (&dst)[N], const char *fmt, Args... args)
{
    return std::snprintf(dst, N, fmt, args...);
}
#endif
#endif
