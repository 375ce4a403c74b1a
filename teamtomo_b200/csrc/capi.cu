// Library-wide C entry points: version and per-thread error text.
#include <string>

#include "capi_util.cuh"

namespace tt {
std::string& last_error_slot() {
    thread_local std::string msg;
    return msg;
}
}  // namespace tt

extern "C" int tt_version(void) { return 100; }

extern "C" const char* tt_last_error(void) { return tt::last_error_slot().c_str(); }
