// Error reporting shared by the C ABI entry points.
#pragma once
#include <string>

namespace mvmcb {
void set_last_error(const std::string& msg);
}
