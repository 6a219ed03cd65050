// errors.hpp — status codes and the per-thread last-error message of the C ABI.
#pragma once
#include <string>

#include "crush.h"

namespace crush {

// Records `msg` as the calling thread's last error and returns `code`.
int fail(int code, const std::string& msg);
// The same for a message with static storage: records the pointer only, so
// the error path itself allocates nothing.
int fail_literal(int code, const char* msg);
const std::string& last_error();
void clear_error();

}  // namespace crush
