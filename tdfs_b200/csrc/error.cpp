// error.cpp -- the thread-local error message behind tdfs_last_error(),
// shared by every entry point (host-only, no CUDA).
#include <cstdarg>
#include <cstdio>
#include <string>

#include "common.h"

namespace tdfs {

namespace {
thread_local std::string g_error;
}

void set_error(const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_error = buf;
}

int fail(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

}  // namespace tdfs

extern "C" const char *tdfs_last_error(void) { return tdfs::g_error.c_str(); }
