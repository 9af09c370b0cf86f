// cn_internal.h -- error reporting shared by the C ABI translation units.
#pragma once

#include <string>

#include "../../include/cn_physics.h"

namespace cn {

// Records `message` as this thread's last error and returns `status`.
cn_status setError(cn_status status, const std::string &message);
void clearError();

} // namespace cn
