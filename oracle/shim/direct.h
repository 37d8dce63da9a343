/* POSIX stand-in for the Windows <direct.h> used by the reference
 * (airpore.cpp:13,463,483). Oracle build only. */
#ifndef ORACLE_SHIM_DIRECT_H
#define ORACLE_SHIM_DIRECT_H
#include <sys/stat.h>
#include <sys/types.h>
inline int _mkdir(const char *path) { return mkdir(path, 0777); }
#endif
