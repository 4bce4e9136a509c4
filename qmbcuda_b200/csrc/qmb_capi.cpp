// qmb_capi.cpp -- error reporting and process-level entry points of the C ABI.
#include <cuda_runtime.h>

#include <string>

#include "qmb_b200.h"

namespace qmb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

qmb_status fail(qmb_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

}  // namespace qmb

extern "C" int qmb_abi_version(void) { return QMB_ABI_VERSION; }

extern "C" const char* qmb_last_error(void) { return qmb::g_last_error.c_str(); }

extern "C" const char* qmb_status_string(qmb_status s) {
    switch (s) {
        case QMB_OK: return "ok";
        case QMB_ERR_INVALID: return "invalid argument";
        case QMB_ERR_CUDA: return "CUDA error";
        case QMB_ERR_NOMEM: return "out of memory";
        case QMB_ERR_ELL_OVERFLOW: return "ELL row overflow";
        case QMB_ERR_NOT_CONVERGED: return "not converged";
        case QMB_ERR_TIMEOUT: return "device wait timed out";
        case QMB_ERR_UNSUPPORTED: return "unsupported";
        case QMB_ERR_NO_DEVICE: return "no CUDA device";
        case QMB_ERR_IO: return "file I/O error";
        case QMB_ERR_CORRUPT: return "corrupt table file";
        default: return "unknown status";
    }
}

extern "C" int qmb_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}
