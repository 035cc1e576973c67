// engine_launch.cuh -- launch templates of the pair-pass kernel, shared by the
// per-cost translation units (engine_p*.cu) so the many instantiations build in
// parallel.
#pragma once

#include <cstring>

#include "internal.h"

namespace culamp_host {

using namespace culamp_dev;

template <int PM, int D, int ACC, int R, bool MOM, bool FR = false, bool F32 = false>
inline cudaError_t launch_t(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    auto kern = pair_pass_kernel<PM, D, ACC, R, MOM, FR, false, F32>;
    if (sh.smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sh.smem);
        if (e != cudaSuccess) return e;
    }
    // programmatic stream serialisation: this pass may launch while the previous
    // kernel finishes its tail; the kernel waits (griddepcontrol.wait) before it
    // reads anything that kernel writes
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(sh.rb, sh.splits);
    cfg.blockDim = dim3(TPB);
    cfg.dynamicSmemBytes = sh.smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_launches() ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, P, (const PassParams *)nullptr, (const int *)nullptr, 0);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

template <int PM, int D, int ACC>
inline cudaError_t launch_v(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    if constexpr (ACC == ACC_LSE) {
        if (P.want_moment) return launch_t<PM, D, ACC, RPT, true>(P, sh, st);
        if constexpr (D > 0) {
            if constexpr (PM == P_SQ) {
                if (P.use_ref && P.fp32) {
                    if (sh.R == RPT_BIG) return launch_t<PM, D, ACC, RPT_BIG, false, true, true>(P, sh, st);
                    if (sh.R == RPT_MID) return launch_t<PM, D, ACC, RPT_MID, false, true, true>(P, sh, st);
                    return launch_t<PM, D, ACC, RPT, false, true, true>(P, sh, st);
                }
            }
            if (P.use_ref) {
                if (sh.R == RPT_BIG) return launch_t<PM, D, ACC, RPT_BIG, false, true>(P, sh, st);
                if (sh.R == RPT_MID) return launch_t<PM, D, ACC, RPT_MID, false, true>(P, sh, st);
                return launch_t<PM, D, ACC, RPT, false, true>(P, sh, st);
            }
            if (sh.R == RPT_BIG) return launch_t<PM, D, ACC, RPT_BIG, false>(P, sh, st);
            if (sh.R == RPT_MID) return launch_t<PM, D, ACC, RPT_MID, false>(P, sh, st);
        }
    }
    return launch_t<PM, D, ACC, RPT, false>(P, sh, st);
}

template <int PM, int ACC>
inline cudaError_t launch_d(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    switch (P.d) {
        case 1: return launch_v<PM, 1, ACC>(P, sh, st);
        case 2: return launch_v<PM, 2, ACC>(P, sh, st);
        case 3: return launch_v<PM, 3, ACC>(P, sh, st);
        default: return launch_v<PM, 0, ACC>(P, sh, st);
    }
}

template <int PM, int D, bool MOM, bool FR>
inline cudaError_t launch_b(const PassParams *plist, const int *block_start, int count, int total_blocks,
                            size_t smem, cudaStream_t st) {
    auto kern = pair_pass_kernel<PM, D, ACC_LSE, RPT, MOM, FR, true>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    PassParams dummy;
    memset(&dummy, 0, sizeof(dummy));
    kern<<<total_blocks, TPB, smem, st>>>(dummy, plist, block_start, count);
    return cudaGetLastError();
}

template <int PM, int D>
inline cudaError_t launch_bd(const PassParams *plist, const int *block_start, int count, int total_blocks,
                             size_t smem, bool mom, bool fr, cudaStream_t st) {
    if (mom) return launch_b<PM, D, true, false>(plist, block_start, count, total_blocks, smem, st);
    if (fr && D > 0) return launch_b<PM, D, false, (D > 0)>(plist, block_start, count, total_blocks, smem, st);
    return launch_b<PM, D, false, false>(plist, block_start, count, total_blocks, smem, st);
}

template <int PM>
inline cudaError_t launch_bp(const PassParams *plist, const int *block_start, int count, int total_blocks,
                             size_t smem, int d, bool mom, bool fr, cudaStream_t st) {
    switch (d) {
        case 1: return launch_bd<PM, 1>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        case 2: return launch_bd<PM, 2>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        case 3: return launch_bd<PM, 3>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        default: return launch_bd<PM, 0>(plist, block_start, count, total_blocks, smem, mom, fr, st);
    }
}

// One translation unit per cost mode instantiates these.
template <int PM>
cudaError_t launch_pair_pm(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st) {
    switch (acc) {
        case ACC_LSE: return launch_d<PM, ACC_LSE>(P, sh, st);
        case ACC_MAX: return launch_d<PM, ACC_MAX>(P, sh, st);
        default: return launch_d<PM, ACC_MIN>(P, sh, st);
    }
}

}  // namespace culamp_host
