// Host-side declarations shared by the library's translation units (no CUDA types).
#pragma once

#include <string>

namespace synx {

// Records `msg` as the calling thread's last global error, the text synx_last_error(NULL)
// returns, and passes `code` through.
int set_global_error(int code, const std::string& msg);

}  // namespace synx
