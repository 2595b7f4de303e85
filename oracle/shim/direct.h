// POSIX stand-ins for the MSVC directory calls (oracle build of the reference only).
#pragma once
#include <sys/stat.h>
#include <unistd.h>
inline int _mkdir(const char* p) { return mkdir(p, 0755); }
inline int _chdir(const char* p) { return chdir(p); }
inline char* _getcwd(char* b, int n) { return getcwd(b, (size_t)n); }
