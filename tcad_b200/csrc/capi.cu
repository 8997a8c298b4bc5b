// ABI helpers of the tcad_b200 library.
#include <atomic>

#include "common.cuh"

namespace tcad {
static std::atomic<uint64_t> g_launches{0};
void note_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace tcad

extern "C" uint64_t tcad_launch_count(void) { return tcad::g_launches.load(); }

extern "C" size_t tcad_pack_sizeof(void) { return sizeof(tcad_pack_t); }

extern "C" const char* tcad_version(void) { return "tcad_b200 0.1 sm_100a"; }
