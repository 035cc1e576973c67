// engine_pinf.cu -- pair-pass kernel instantiations for cost mode P_INF.
#include "engine_launch.cuh"

namespace culamp_host {

cudaError_t launch_pair_inf(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st) {
    return launch_pair_pm<P_INF>(P, acc, sh, st);
}

}  // namespace culamp_host
