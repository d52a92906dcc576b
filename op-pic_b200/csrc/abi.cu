// Library identification and status strings of the C ABI.

#include <atomic>

#include "oppb_common.cuh"

namespace oppb {
namespace {
std::atomic<uint64_t> g_launches{0};
oppb_tuning g_tuning = {OPPB_DEPOSIT_WARP_ATOMIC, 8, 2, 16, 1, 8, 0, 0, 256, 4, 0};
}  // namespace
void count_launches(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
const oppb_tuning& tuning() { return g_tuning; }
}  // namespace oppb

extern "C" uint64_t oppb_kernel_launches(void) { return oppb::g_launches.load(std::memory_order_relaxed); }

extern "C" int oppb_set_tuning(const oppb_tuning* t) {
    if (!t || (t->deposit != OPPB_DEPOSIT_WARP_ATOMIC && t->deposit != OPPB_DEPOSIT_CTA_TABLE &&
               t->deposit != OPPB_DEPOSIT_EXACT))
        return OPPB_ERR_ARG;
    if (t->replicas < 1 || t->replicas > 64) return OPPB_ERR_ARG;
    if (t->advec_items != 1 && t->advec_items != 2 && t->advec_items != 4) return OPPB_ERR_ARG;
    if (t->sort_gather_cols < 1 || t->sort_gather_cols > 16) return OPPB_ERR_ARG;
    if (t->move_lanes < 0 || t->move_lanes > 2) return OPPB_ERR_ARG;
    if (t->move_occupancy != 0 && t->move_occupancy != 5 && t->move_occupancy != 8) return OPPB_ERR_ARG;
    if (t->sort_scatter != 0 && t->sort_scatter != 1) return OPPB_ERR_ARG;
    if (t->move_stage != 0 && t->move_stage != 1) return OPPB_ERR_ARG;
    if (t->move_block != 0 && t->move_block != 128 && t->move_block != 256 && t->move_block != 512)
        return OPPB_ERR_ARG;
    if (t->cabana_occupancy != 0 && t->cabana_occupancy != 4 && t->cabana_occupancy != 5) return OPPB_ERR_ARG;
    if (t->move_walk32 < 0 || t->move_walk32 > 2) return OPPB_ERR_ARG;
    oppb::g_tuning = *t;
    if (oppb::g_tuning.move_lanes == 0) oppb::g_tuning.move_lanes = 1;
    if (oppb::g_tuning.move_occupancy == 0) oppb::g_tuning.move_occupancy = 8;
    if (oppb::g_tuning.move_block == 0) oppb::g_tuning.move_block = 256;
    return OPPB_OK;
}

extern "C" void oppb_get_tuning(oppb_tuning* out) {
    if (out) *out = oppb::g_tuning;
}

extern "C" const char* oppb_version(void) { return "oppb 0.1 (sm_100a)"; }

extern "C" const char* oppb_status_string(int status) {
    switch (status) {
        case OPPB_OK: return "ok";
        case OPPB_ERR_ARG: return "invalid argument";
        case OPPB_ERR_LAUNCH: return "CUDA launch error";
        case OPPB_ERR_WORKSPACE: return "workspace too small";
        case OPPB_ERR_HOP_LIMIT: return "particle exceeded the hop limit";
        case OPPB_ERR_CELL_RANGE: return "cell index out of range";
        case OPPB_ERR_CAPACITY: return "particle set capacity exceeded";
        case OPPB_ERR_NO_DEVICE: return "no CUDA device";
        case OPPB_ERR_SCRATCH_LIMIT: return "request exceeds the fixed scratch of an allocation-free entry point";
        case OPPB_ERR_WAIT_LIMIT: return "a bounded wait for an asynchronous copy ran out";
        default: return "unknown status";
    }
}
