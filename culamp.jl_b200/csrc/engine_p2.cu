// engine_p2.cu -- pair-pass kernel instantiations for cost mode P_SQ.
#include "engine_launch.cuh"

namespace culamp_host {

cudaError_t launch_pair_sq(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st) {
    return launch_pair_pm<P_SQ>(P, acc, sh, st);
}

}  // namespace culamp_host
