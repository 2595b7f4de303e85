// Minimal Win32 stand-ins so the reference's MSVC sources compile with g++ on
// Linux (oracle build of the reference only; nothing in the product uses this).
// Named shared memory is only used by the reference in primary-secondary mode;
// here every mapping call fails, which direct mode never reaches.
#pragma once
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <ctime>

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

inline HANDLE OpenFileMapping(int, int, const wchar_t*) { return nullptr; }
inline void* MapViewOfFile(HANDLE, int, int, int, size_t) { return nullptr; }
inline int UnmapViewOfFile(const void*) { return 1; }
inline int CloseHandle(HANDLE) { return 1; }
inline DWORD GetLastError() { return 0; }
inline int MultiByteToWideChar(int, int, const char*, int, wchar_t* w, int n) {
  if (w && n > 0) w[0] = 0;
  return 0;
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
