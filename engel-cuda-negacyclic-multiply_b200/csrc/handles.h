// Opaque handle types of the C ABI, shared by the translation units that implement it.
#pragma once

#include <string>

#include "engine.h"

struct nc_plan {
    nc::Plan* p;
};

namespace nc {
// Sets the message nc_last_error() returns on this thread.
void set_last_error(const std::string& msg);
}  // namespace nc
