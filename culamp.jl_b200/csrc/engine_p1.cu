// engine_p1.cu -- pair-pass kernel instantiations for cost mode P_L1.
#include "engine_launch.cuh"

namespace culamp_host {

cudaError_t launch_pair_l1(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st) {
    return launch_pair_pm<P_L1>(P, acc, sh, st);
}

}  // namespace culamp_host
