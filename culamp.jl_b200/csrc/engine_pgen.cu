// engine_pgen.cu -- pair-pass kernel instantiations for cost mode P_GEN.
#include "engine_launch.cuh"

namespace culamp_host {

cudaError_t launch_pair_gen(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st) {
    return launch_pair_pm<P_GEN>(P, acc, sh, st);
}

}  // namespace culamp_host
