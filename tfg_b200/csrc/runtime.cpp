// Error state and device checks shared by all entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "../../include/tfg_pt.h"
#include "tfg_errors.h"
#include "tfg_runtime.h"

namespace tfg {

namespace {
thread_local std::string g_last_error;
thread_local int g_last_code = 0;
}  // namespace

void set_error(int code, const std::string& msg) {
    g_last_code = code;
    g_last_error = msg;
}

int fail(int code, const std::string& msg) {
    set_error(code, msg);
    return code;
}

int ok() { return 0; }

int require_sm100(int dev) {
    if (dev < 0 || dev >= kMaxDevices)
        return fail(TFG_E_INVALID, "device ordinal " + std::to_string(dev) + " is out of range: the library keeps "
                                   "per-device state for ordinals 0-" + std::to_string(kMaxDevices - 1));
    static int checked[kMaxDevices] = {0};   // 0 unknown, 1 ok, 2 bad
    int& c = checked[dev];
    if (c == 0) {
        int major = 0;
        cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        if (e != cudaSuccess) return fail((int)e, std::string("device query: ") + cudaGetErrorString(e));
        c = (major == 10) ? 1 : 2;
    }
    if (c != 1) return fail(TFG_E_UNSUPPORTED, "this library is built for sm_100a (B200) only");
    return 0;
}

}  // namespace tfg

extern "C" const char* tfgGetLastErrorString(void) { return tfg::g_last_error.c_str(); }
