// capi.cu -- error reporting and version of the C ABI.
#include <string>

#include "vam_internal.cuh"

namespace vam {
namespace {
thread_local std::string g_last_error;
}

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

void clear_error() { g_last_error.clear(); }

}  // namespace vam

extern "C" const char* vam_last_error_string(void) { return vam::g_last_error.c_str(); }

extern "C" const char* vam_version(void) { return "vamcore 1.0 sm_100a"; }
