// capi.cu -- library-wide C entry points (status strings, version).
#include "loits_b200.h"

extern "C" const char* loits_status_string(int status) {
  switch (status) {
    case LOITS_OK: return "ok";
    case LOITS_ERR_INVALID: return "invalid argument";
    case LOITS_ERR_UNSUPPORTED: return "unsupported size or configuration";
    case LOITS_ERR_CUDA: return "CUDA runtime error";
    case LOITS_ERR_TIMEOUT: return "a bounded device-side wait ran out";
    case LOITS_ERR_CAPACITY: return "buffer or workspace too small";
    case LOITS_ERR_EPSILON: return "epsilon must be the reference's 1e-5";
    default: return "unknown status";
  }
}

extern "C" int loits_version(void) { return 100; }
