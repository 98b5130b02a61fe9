// Library identity and status strings for the C ABI.
#include "tsb_common.cuh"

extern "C" const char *tsb_version(void) { return "tsb 0.1.0 sm_100a"; }

extern "C" const char *tsb_status_string(int status) {
  switch (status) {
    case TSB_OK: return "ok";
    case TSB_ERR_INVALID_ARG: return "invalid argument";
    case TSB_ERR_CAPACITY: return "capacity exceeded (regrow and retry)";
    case TSB_ERR_NONFINITE: return "non-finite input";
    case TSB_ERR_TIMEOUT: return "bounded device wait timed out";
    case TSB_ERR_CUDA: return "CUDA launch error";
    case TSB_ERR_UNSUPPORTED: return "unsupported configuration";
    case TSB_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
  }
}
