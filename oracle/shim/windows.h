// Minimal Win32 stand-ins so the reference's MSVC sources compile with g++ on
// Linux (oracle build of the reference only; nothing in the product uses this).
// Named shared memory is only used by the reference in primary-secondary mode (the
// normal field of each time layer): here a mapping name is a file of that name in
// the working directory, mapped read-only.
#pragma once
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fcntl.h>
#include <map>
#include <stdint.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

typedef void* HANDLE;
typedef const char* LPCTSTR;
typedef char* LPTSTR;
typedef void* PVOID;
typedef unsigned long DWORD;
#define INVALID_HANDLE_VALUE ((HANDLE)(-1))
#define FILE_MAP_READ 4
#define FILE_MAP_ALL_ACCESS 0xf001f
#define PAGE_READWRITE 4
#define CP_ACP 0
#define TRUE 1
#define FALSE 0
#define CopyMemory(d, s, n) memcpy((d), (s), (n))

// mapping handles are file descriptors + 1; views remember their sizes for munmap
inline std::map<const void*, size_t>& tdem_shim_views() {
  static std::map<const void*, size_t> v;
  return v;
}
inline HANDLE OpenFileMapping(int, int, const wchar_t* name) {
  char path[1024];
  size_t i = 0;
  for (; name && name[i] && i + 1 < sizeof path; ++i) path[i] = (char)name[i];
  path[i] = 0;
  const int fd = open(path, O_RDONLY);
  return fd < 0 ? nullptr : (HANDLE)(intptr_t)(fd + 1);
}
inline void* MapViewOfFile(HANDLE h, int, int, int, size_t n) {
  if (!h || !n) return nullptr;
  struct stat st;
  const int fd = (int)(intptr_t)h - 1;
  if (fstat(fd, &st) != 0 || (size_t)st.st_size < n) return nullptr;  // never map past the file
  void* p = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
  if (p == MAP_FAILED) return nullptr;
  tdem_shim_views()[p] = n;
  return p;
}
inline int UnmapViewOfFile(const void* p) {
  auto it = tdem_shim_views().find(p);
  if (it == tdem_shim_views().end()) return 0;
  munmap(const_cast<void*>(p), it->second);
  tdem_shim_views().erase(it);
  return 1;
}
inline int CloseHandle(HANDLE h) {
  if (h && h != INVALID_HANDLE_VALUE) close((int)(intptr_t)h - 1);
  return 1;
}
inline DWORD GetLastError() { return 0; }
inline int MultiByteToWideChar(int, int, const char* s, int, wchar_t* w, int n) {
  int i = 0;
  for (; s && s[i] && i + 1 < n; ++i) w[i] = (wchar_t)(unsigned char)s[i];
  if (w && n > 0) w[i] = 0;
  return i + 1;
}

typedef long long __time64_t;
inline __time64_t _time64(__time64_t* t) {
  __time64_t v = (__time64_t)time(nullptr);
  if (t) *t = v;
  return v;
}
inline int _itoa_s(int v, char* b, size_t n, int) { return snprintf(b, n, "%d", v) < 0; }
template <size_t N>
inline int _itoa_s(int v, char (&b)[N], int) { return snprintf(b, N, "%d", v) < 0; }
#define sprintf_s sprintf

// Process-creation stand-ins: the post-processing modules define helpers that
// start child processes but never call them in the paths the oracle runs; here
// every process creation fails.
typedef char* LPSTR;
typedef DWORD* LPDWORD;
#define INFINITE 0xffffffffu
#define CREATE_NO_WINDOW 0x08000000
struct STARTUPINFOA { DWORD cb; };
struct PROCESS_INFORMATION { HANDLE hProcess, hThread; DWORD dwProcessId, dwThreadId; };
#define ZeroMemory(p, n) memset((p), 0, (n))
inline int CreateProcessA(const char*, LPSTR, void*, void*, int, DWORD, void*, const char*, STARTUPINFOA*,
                          PROCESS_INFORMATION*) {
  return 0;
}
inline DWORD WaitForSingleObject(HANDLE, DWORD) { return 0; }
inline int GetExitCodeProcess(HANDLE, LPDWORD c) {
  if (c) *c = 1;
  return 0;
}
