// errors.cpp -- last-error text for sheen_get_last_error().
//
// The reference keeps one static 512-byte buffer (api/sheen_c_api.cu:21-26)
// that every failing call overwrites.  Here the buffer is per thread, which
// keeps the reference's single-threaded behaviour (the message of this
// thread's last failing call) and stays correct when several threads drive
// the request loop.
#include <cstdio>
#include <cstring>

namespace sheen {

static thread_local char g_error[512] = "no error";

void set_error(const char* msg) {
    std::strncpy(g_error, msg ? msg : "unknown error", sizeof(g_error) - 1);
    g_error[sizeof(g_error) - 1] = '\0';
}

void set_errorf(const char* fmt, const char* a) {
    std::snprintf(g_error, sizeof(g_error), fmt, a);
}

}  // namespace sheen

extern "C" const char* sheen_get_last_error(void) { return sheen::g_error; }
