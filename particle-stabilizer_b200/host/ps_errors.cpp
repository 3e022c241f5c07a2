// ps_errors.cpp — the message channel behind ps_last_error(): every failing
// entry point, on the device side (ps_engine.cu) or the host side (file
// formats, post-processing), records its message here for the calling
// thread and returns its status code.
#include <string>

#include "particle_stabilizer_b200.h"

namespace {
thread_local std::string g_last_error;
}  // namespace

extern "C" int ps_internal_fail(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

extern "C" const char* ps_last_error(void) { return g_last_error.c_str(); }
