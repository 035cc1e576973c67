// engine_bat.cu -- batched pair-pass kernel instantiations (many instances per launch).
#include "engine_launch.cuh"

namespace culamp_host {

cudaError_t launch_pass_batched(const PassParams *plist, const int *block_start, int count,
                                int total_blocks, size_t smem, int pm, int d, int acc, bool mom,
                                bool fixed_ref, cudaStream_t st) {
    if (count < 1 || total_blocks < 1) return cudaSuccess;
    if (acc != ACC_LSE) return cudaErrorInvalidValue;
    if (pm == P_SQ) return launch_bp<P_SQ>(plist, block_start, count, total_blocks, smem, d, mom, fixed_ref, st);
    if (pm == P_L1) return launch_bp<P_L1>(plist, block_start, count, total_blocks, smem, d, mom, fixed_ref, st);
    return cudaErrorNotSupported;
}

}  // namespace culamp_host
