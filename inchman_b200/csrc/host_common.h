// Error reporting shared by the host translation units of the C ABI.
#pragma once
#include <cstdarg>
#include <cstdio>
#include <string>

namespace gpgmp {
// Records a message for gpgmp_last_error() on the calling thread and returns code.
int set_error(int code, const char* fmt, ...);
}  // namespace gpgmp
