// Error recording shared by the libraries built from this tree: the C ABI
// returns void or a status code, so a failure is recorded here (per thread)
// and read back with otf_last_status / otf_last_error.
#include <cstdio>
#include <string>
#include "otf_common.cuh"

namespace otf {

static thread_local int g_status = 0;
static thread_local std::string g_msg;

void set_error(int code, const char *what, const char *file, int line)
{
    g_status = code ? code : -1;
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString((cudaError_t)code), file,
             line);
    g_msg = buf;
}
void set_error_msg(int code, const std::string &msg)
{
    g_status = code ? code : -1;
    g_msg = msg;
}
void clear_error()
{
    g_status = 0;
    g_msg.clear();
}
int last_status() { return g_status; }
const char *last_error() { return g_msg.c_str(); }

}  // namespace otf
