// errors.cpp — per-thread last error of the C ABI.
#include "errors.hpp"

namespace crush {

static thread_local std::string g_last_error;
static thread_local const char* g_last_literal = nullptr;

int fail(int code, const std::string& msg) {
    g_last_literal = nullptr;
    g_last_error = msg;
    return code;
}
int fail_literal(int code, const char* msg) {
    g_last_literal = msg;
    return code;
}
const std::string& last_error() { return g_last_error; }
void clear_error() {
    g_last_literal = nullptr;
    g_last_error.clear();
}

}  // namespace crush

extern "C" const char* crush_last_error(void) {
    return crush::g_last_literal ? crush::g_last_literal : crush::last_error().c_str();
}
