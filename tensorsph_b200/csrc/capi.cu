// Library-wide C entry points: status strings and ABI version.
#include "common.cuh"

extern "C" {

int tsph_abi_version(void) { return 2; }

const char* tsph_status_string(int code) {
  switch (code) {
    case TSPH_OK: return "ok";
    case TSPH_ERR_ARG: return "invalid argument";
    case TSPH_ERR_NONFINITE: return "positions must contain only finite values";
    case TSPH_ERR_CUDA: return "CUDA runtime error";
    case TSPH_ERR_WORKSPACE: return "workspace smaller than the queried size";
    case TSPH_ERR_CAPACITY: return "fixed-capacity structure overflowed";
    case TSPH_ERR_UNSUPPORTED: return "option not supported by this build";
    case TSPH_ERR_INDEX: return "pair index out of range";
    case TSPH_ERR_GRID: return "cell grid extent too large";
    case TSPH_ERR_STATE: return "non-finite or invalid engine state";
    case TSPH_ERR_TIMEOUT: return "bounded device wait gave up";
    default: return "unknown status";
  }
}

}  // extern "C"
