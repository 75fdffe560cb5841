// Library-wide C entry points: version and the per-thread error message.
#include "b2c_common.cuh"

namespace b2c {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

}  // namespace b2c

extern "C" int32_t b2c_version(void) { return 100; }
extern "C" const char *b2c_last_error(void) { return b2c::g_err; }
