// Thread-local last-error message behind gpgmp_last_error().
#include <cstdarg>
#include <cstdio>
#include <string>
#include "host_common.h"
#include "../../include/gpgmp_c.h"

namespace gpgmp {
namespace {
thread_local std::string g_last_error;
}
int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}
}  // namespace gpgmp

extern "C" const char* gpgmp_last_error(void) { return gpgmp::g_last_error.c_str(); }
