// errors.cpp — per-thread last error of the C ABI.
#include "errors.hpp"

namespace crush {

static thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}
const std::string& last_error() { return g_last_error; }
void clear_error() { g_last_error.clear(); }

}  // namespace crush

extern "C" const char* crush_last_error(void) { return crush::last_error().c_str(); }
