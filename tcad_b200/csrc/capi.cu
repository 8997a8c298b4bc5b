// ABI helpers of the tcad_b200 library.
#include "common.cuh"

extern "C" size_t tcad_pack_sizeof(void) { return sizeof(tcad_pack_t); }

extern "C" const char* tcad_version(void) { return "tcad_b200 0.1 sm_100a"; }
