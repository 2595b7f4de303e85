// LLP64 formatted-I/O stand-in (oracle build of the reference only).
//
// The reference was written for Windows, where `long` is 32 bits, and reads and
// prints `int` variables with "%ld" (e.g. CalcNonstat3DLine/vec_prep_data.cpp:188).
// Under Linux's LP64 model that conversion stores 8 bytes and overwrites the
// neighbouring struct member.  This header is force-included into the
// reference's translation units; it drops the `l` length modifier from integer
// conversions so every conversion stores or reads 4 bytes, exactly as on the
// platform the code was written for.  Floating-point ("%lf") and "%ll"
// conversions are left unchanged.  The reference never reads a real `long`
// through these functions.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <cstring>

inline const char* tdem_llp64_fmt(const char* in, char* out, size_t cap) {
  size_t o = 0;
  for (size_t i = 0; in[i] && o + 1 < cap; ++i) {
    out[o++] = in[i];
    if (in[i] != '%') continue;
    if (in[i + 1] == '%') { out[o++] = in[++i]; continue; }
    // flags, width, precision, assignment suppression
    while (in[i + 1] && strchr("-+ #0123456789.*", in[i + 1]) && o + 1 < cap) out[o++] = in[++i];
    if (in[i + 1] == 'l' && in[i + 2] != 'l' && in[i + 2] && strchr("diuxXon", in[i + 2])) ++i;
  }
  out[o] = 0;
  return out;
}

inline int tdem_llp64_fscanf(FILE* f, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  int r = vfscanf(f, tdem_llp64_fmt(fmt, buf, sizeof buf), ap);
  va_end(ap);
  return r;
}
inline int tdem_llp64_sscanf(const char* s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  int r = vsscanf(s, tdem_llp64_fmt(fmt, buf, sizeof buf), ap);
  va_end(ap);
  return r;
}
inline int tdem_llp64_fprintf(FILE* f, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  int r = vfprintf(f, tdem_llp64_fmt(fmt, buf, sizeof buf), ap);
  va_end(ap);
  return r;
}
inline int tdem_llp64_sprintf(char* s, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  int r = vsprintf(s, tdem_llp64_fmt(fmt, buf, sizeof buf), ap);
  va_end(ap);
  return r;
}
#define fscanf tdem_llp64_fscanf
#define sscanf tdem_llp64_sscanf
#define fprintf tdem_llp64_fprintf
#define sprintf tdem_llp64_sprintf
