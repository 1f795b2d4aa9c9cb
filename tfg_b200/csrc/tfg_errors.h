// Error reporting shared by every entry point: a thread-local message for
// tfgGetLastErrorString() and helpers that turn CUDA failures into return
// codes.
#pragma once

#include <string>

namespace tfg {

void set_error(int code, const std::string& msg);
int fail(int code, const std::string& msg);
int ok();

}  // namespace tfg
