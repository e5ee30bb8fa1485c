// Error reporting and version of the C ABI (per host thread, no allocation on the device).
#include "cs_common.cuh"

namespace cs {
namespace {
thread_local char g_err[1024] = {0};
}

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

const char* last_error() { return g_err; }

}  // namespace cs

extern "C" int cs_last_error(char* buf, int32_t len) {
    const char* e = cs::last_error();
    int n = int(strlen(e));
    if (buf && len > 0) {
        int k = n < len - 1 ? n : len - 1;
        memcpy(buf, e, size_t(k));
        buf[k] = 0;
    }
    return n;
}

extern "C" const char* cs_version(void) { return "cerebrosim_b200 0.1 (sm_100a)"; }

extern "C" size_t cs_abi_sizeof(int32_t which) {
    switch (which) {
        case 0: return sizeof(cs_opening);
        case 1: return sizeof(cs_step_desc);
        case 2: return CS_SEG_STRIDE;
        case 3: return sizeof(cs_batch_desc);
        default: return 0;
    }
}
