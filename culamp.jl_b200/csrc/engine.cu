// engine.cu -- launch shape of the pair passes and the launch dispatch.
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "internal.h"

namespace culamp_host {

using namespace culamp_dev;

static thread_local int t_pdl_off = 0;

bool pdl_launches() {
    static const bool on = std::getenv("CULAMP_NO_PDL") == nullptr;
    return on && t_pdl_off == 0;
}

PdlOff::PdlOff() { ++t_pdl_off; }
PdlOff::~PdlOff() { --t_pdl_off; }

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

// Per-cost launchers (engine_p1.cu, engine_p2.cu, engine_pinf.cu, engine_pgen.cu)
// and the batched launcher (engine_bat.cu).
cudaError_t launch_pair_l1(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st);
cudaError_t launch_pair_sq(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st);
cudaError_t launch_pair_inf(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st);
cudaError_t launch_pair_gen(const PassParams &P, int acc, const LaunchShape &sh, cudaStream_t st);

static cudaError_t launch_any(const PassParams &P, int pm, int acc, const LaunchShape &sh, cudaStream_t st) {
    switch (pm) {
        case P_L1: return launch_pair_l1(P, acc, sh, st);
        case P_SQ: return launch_pair_sq(P, acc, sh, st);
        case P_INF: return launch_pair_inf(P, acc, sh, st);
        default: return launch_pair_gen(P, acc, sh, st);
    }
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
    return launch_any(P, pm, acc, sh, st);
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
    return launch_any(P, pm, acc, sh, st);
}

}  // namespace culamp_host
