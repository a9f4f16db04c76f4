// cpu_offload_counters.cpp — the two offload counters levmarq_solver.cpp reads
// (comp_light_cuda.h:23, set_star_grid_cuda.h:24) for a build of lcurve_re's
// CPU path (TEST INFRASTRUCTURE ONLY). The reference defines them only in its
// CUDA sources; a CPU-only build offloads nothing, so both stay zero.
#include <cstdint>

namespace Lcurve {
std::uint64_t cuda_flux_evaluation_count() { return 0; }
std::uint64_t cuda_grid_evaluation_count() { return 0; }
}  // namespace Lcurve
