// engine.cu -- template instantiations of the pair-pass kernel and the launcher.
#include <cmath>

#include <cstring>

#include "internal.h"

namespace culamp_host {

using namespace culamp_dev;

int pmode_of(double p) {
    if (p == 1.0) return P_L1;
    if (p == 2.0) return P_SQ;
    if (std::isinf(p)) return P_INF;
    return P_GEN;
}

LaunchShape pass_shape(int n, int m, int d, int acc, int sm_count, bool mom) {
    LaunchShape s{};
    const bool packed = d >= 1 && d <= MAXD_PACKED;
    const int sms = sm_count > 0 ? sm_count : 148;
    // More rows per thread amortise each broadcast column over more pairs;
    // used when there are enough row blocks to fill the GPU with few column
    // splits. Measured (row pass, d = 3): 4 rows beat 8 by 16 % at 16384^2
    // (4 CTAs per SM instead of 3), 8 beat 4 by 4 % at 65536^2.
    const bool big = acc == ACC_LSE && packed && !mom;
    s.R = (big && n >= 32768) ? RPT_BIG : ((big && n >= 16384) ? RPT_MID : RPT);
    const int rows = TPB * s.R;
    s.rb = (n + rows - 1) / rows;
    if (s.rb < 1) s.rb = 1;
    // column splits are whole tiles: measured at n = m = 4096, finer splits
    // (64 / 128 columns) cost more in per-CTA overhead and merging than the
    // extra CTAs win back
    const int ch = packed ? CHUNK : CHUNK_G;
    // Resident CTAs per SM: the kernels' launch bounds (3 for 8 rows per
    // thread, 4 otherwise). All CTAs of a pass do the same work, so the pass
    // takes ceil(CTAs / slots) waves of (columns per split) each: pick the
    // split count that minimises that, preferring fewer splits on ties (fewer
    // partials to merge). E.g. 65536^2: 64 row blocks on 444 slots -> 20 splits
    // (2.9 waves, 95 % of the ideal) rather than 10 (1.4 waves, 72 %).
    const long long slots = (long long)sms * (s.R > RPT_MID ? 3 : 4);
    const int max_splits = (m + ch - 1) / ch;
    int best_splits = 1, best_cps = ((m + ch - 1) / ch) * ch;
    double best_cost = 1e300;
    for (int sp = 1; sp <= max_splits; ++sp) {
        int cps = (m + sp - 1) / sp;
        cps = ((cps + ch - 1) / ch) * ch;
        const int spr = (m + cps - 1) / cps;
        if (spr != sp) continue;                  // same shape as a smaller count
        const long long ctas = (long long)s.rb * spr;
        const long long waves = (ctas + slots - 1) / slots;
        const double cost = (double)waves * (double)cps * (1.0 + 0.002 * spr);
        if (cost < best_cost * (1.0 - 1e-9)) {
            best_cost = cost;
            best_splits = spr;
            best_cps = cps;
        }
    }
    s.splits = best_splits;
    s.cols_per_split = best_cps;
    s.smem = (size_t)(packed ? CHUNK * 4 : CHUNK_G * (d + 1)) * sizeof(double);
    s.part_bytes = s.splits > 1 ? (size_t)s.splits * (size_t)n * 3 * sizeof(double) : 0;
    s.sms = sms;
    (void)acc;
    return s;
}

template <int PM, int D, int ACC, int R, bool MOM, bool FR = false>
static cudaError_t launch_t(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    auto kern = pair_pass_kernel<PM, D, ACC, R, MOM, FR>;
    if (sh.smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sh.smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid(sh.rb, sh.splits);
    kern<<<grid, TPB, sh.smem, st>>>(P, nullptr, nullptr, 0);
    return cudaGetLastError();
}

template <int PM, int D, int ACC>
static cudaError_t launch_v(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    if constexpr (ACC == ACC_LSE) {
        if (P.want_moment) return launch_t<PM, D, ACC, RPT, true>(P, sh, st);
        if constexpr (D > 0) {
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
static cudaError_t launch_d(const PassParams &P, const LaunchShape &sh, cudaStream_t st) {
    switch (P.d) {
        case 1: return launch_v<PM, 1, ACC>(P, sh, st);
        case 2: return launch_v<PM, 2, ACC>(P, sh, st);
        case 3: return launch_v<PM, 3, ACC>(P, sh, st);
        default: return launch_v<PM, 0, ACC>(P, sh, st);
    }
}

template <int ACC>
static cudaError_t launch_p(const PassParams &P, int pm, const LaunchShape &sh, cudaStream_t st) {
    switch (pm) {
        case P_L1: return launch_d<P_L1, ACC>(P, sh, st);
        case P_SQ: return launch_d<P_SQ, ACC>(P, sh, st);
        case P_INF: return launch_d<P_INF, ACC>(P, sh, st);
        default: return launch_d<P_GEN, ACC>(P, sh, st);
    }
}

template <int PM, int D, bool MOM, bool FR>
static cudaError_t launch_b(const PassParams *plist, const int *block_start, int count, int total_blocks,
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
static cudaError_t launch_bd(const PassParams *plist, const int *block_start, int count, int total_blocks,
                             size_t smem, bool mom, bool fr, cudaStream_t st) {
    if (mom) return launch_b<PM, D, true, false>(plist, block_start, count, total_blocks, smem, st);
    if (fr && D > 0) return launch_b<PM, D, false, (D > 0)>(plist, block_start, count, total_blocks, smem, st);
    return launch_b<PM, D, false, false>(plist, block_start, count, total_blocks, smem, st);
}

template <int PM>
static cudaError_t launch_bp(const PassParams *plist, const int *block_start, int count, int total_blocks,
                             size_t smem, int d, bool mom, bool fr, cudaStream_t st) {
    switch (d) {
        case 1: return launch_bd<PM, 1>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        case 2: return launch_bd<PM, 2>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        case 3: return launch_bd<PM, 3>(plist, block_start, count, total_blocks, smem, mom, fr, st);
        default: return launch_bd<PM, 0>(plist, block_start, count, total_blocks, smem, mom, fr, st);
    }
}

cudaError_t launch_pass_batched(const PassParams *plist, const int *block_start, int count,
                                int total_blocks, size_t smem, int pm, int d, int acc, bool mom,
                                bool fixed_ref, cudaStream_t st) {
    if (count < 1 || total_blocks < 1) return cudaSuccess;
    if (acc != ACC_LSE) return cudaErrorInvalidValue;
    if (pm == P_SQ) return launch_bp<P_SQ>(plist, block_start, count, total_blocks, smem, d, mom, fixed_ref, st);
    if (pm == P_L1) return launch_bp<P_L1>(plist, block_start, count, total_blocks, smem, d, mom, fixed_ref, st);
    return cudaErrorNotSupported;
}

cudaError_t launch_pass_at(PassParams P, int pm, int acc, const LaunchShape &sh, double *part,
                           unsigned *tickets, double *blk, cudaStream_t st) {
    if (P.want_moment && sh.R != RPT) return cudaErrorInvalidValue;
    P.splits = sh.splits;
    P.cols_per_split = sh.cols_per_split;
    P.part = part;
    P.rb_ticket = tickets;
    P.grid_ticket = tickets + sh.rb;
    P.blk = blk;
    switch (acc) {
        case ACC_LSE: return launch_p<ACC_LSE>(P, pm, sh, st);
        case ACC_MAX: return launch_p<ACC_MAX>(P, pm, sh, st);
        default: return launch_p<ACC_MIN>(P, pm, sh, st);
    }
}

cudaError_t launch_pass(PassParams P, int pm, int acc, const LaunchShape &sh, Scratch &scr,
                        cudaStream_t st) {
    if (P.fx) return launch_feat_pass(P, acc, scr, sh.sms, st);       // tensor-core feature path
    if (P.want_moment && sh.R != RPT) return cudaErrorInvalidValue;   // shape built without mom
    P.splits = sh.splits;
    P.cols_per_split = sh.cols_per_split;
    P.part = scr.part.as<double>();
    P.rb_ticket = scr.tickets.as<unsigned>();
    P.grid_ticket = scr.tickets.as<unsigned>() + sh.rb;
    P.blk = scr.blk.as<double>();
    if (scr.part.bytes < sh.part_bytes || scr.tickets.bytes < (size_t)(sh.rb + 1) * sizeof(unsigned) ||
        scr.blk.bytes < (size_t)sh.rb * 4 * sizeof(double))
        return cudaErrorInvalidValue;
    switch (acc) {
        case ACC_LSE: return launch_p<ACC_LSE>(P, pm, sh, st);
        case ACC_MAX: return launch_p<ACC_MAX>(P, pm, sh, st);
        default: return launch_p<ACC_MIN>(P, pm, sh, st);
    }
}

}  // namespace culamp_host
