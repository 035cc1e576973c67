// feature.cu -- the feature-cost reduction passes on the 5th-generation tensor
// cores (sm_100a: tcgen05.mma with TMEM accumulators).
//
// For high-dimensional points (feature vectors, d >= 32) with the squared
// Euclidean cost C_ij = |x_i|^2 + |y_j|^2 - 2 <x_i, y_j>, the pair loop of the
// log-sum-exp passes (warp_logsumexp_cellsim_fused!, SinkhornCellSim.jl:153-238,
// and the Sinkhorn / LAMP passes SinkhornKernel.jl:341-444, MirrorProxKernel.jl:
// 833-938, 941-1016 with a dot-product cost) is dominated by the inner products.
// They are computed here as a GEMM on the tensor cores:
//
//  * Split precision. Each FP64 feature is split into bf16 pieces
//    x = x0 + x1 (+ x2) (each piece the bf16 rounding of what the previous ones
//    leave). BF16x3 sums the products x0y0 + x0y1 + x1y0 (about 16 significant
//    bits per product), BF16x6 adds x0y2 + x1y1 + x2y0 (about 24 bits). All
//    products accumulate in FP32 in TMEM, small terms first.
//  * Operand layout. The pieces are written once per solve in exactly the
//    shared-memory image the MMA reads: 128-row x 64-element (128-byte) blocks,
//    K-major, 128-byte swizzled (16-byte chunk c of row r stored at chunk
//    c ^ (r % 8)). One pipeline stage is then a handful of contiguous 16 KB
//    cp.async.bulk copies -- no tensor maps, no multicast.
//  * Warp roles (192 threads, one CTA per SM, persistent over work units):
//    warp 0 issues the bulk copies, warp 1 issues tcgen05.mma (M = N = 128,
//    K = 16 per instruction) into one of two 128-column TMEM accumulators,
//    warps 2-5 read the finished accumulator (tcgen05.ld, one row per thread)
//    and fold it into an FP32 online log-sum-exp (or min / max) while the
//    tensor cores fill the other accumulator.
//  * A work unit is (128-row tile, slice of column tiles); each writes a
//    per-row (max, sum, moment) partial and feat_merge_kernel merges the
//    slices and runs the same per-row epilogue and finish step as the pair
//    passes, so every solver runs unchanged on this path.
//
// Every wait on an mbarrier is bounded (FT_WAIT_NS); a role that gives up sets
// the CTA's abort flag, the others leave their loops, outstanding copies and
// MMAs are drained (again bounded), TMEM is freed and the solver's control
// block records a device timeout.
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"

namespace {

using namespace culamp_dev;

constexpr int FT_M = 128;                          // rows per tile = TMEM lanes; packed block height
constexpr int FT_K = 64;                           // K elements per block (128 bytes of bf16)
constexpr int FT_PIECE_ELEMS = FT_M * FT_K;        // one 128 x 64 block: 16 KB
constexpr int FT_PIECE_BYTES = FT_PIECE_ELEMS * 2;
constexpr int FT_THREADS = 192;
constexpr unsigned long long FT_WAIT_NS = 2000000000ull;
constexpr int FT_CTRL_BYTES = 10240;               // barriers, TMEM slot, per-warp column terms

// N: columns per tile (MMA N, TMEM columns per accumulator). One stage holds
// the A pieces (NP x 16 KB) and the B pieces (NP x N/128 x 16 KB) of one K
// block. BF16x3 uses N = 256: each A piece then feeds twice the columns, so
// two 96 KB stages buffer ~3000 tensor cycles of work against the copies'
// latency (three 64 KB stages of N = 128 buffered ~2300). BF16x6 keeps
// N = 128 (two 96 KB stages).
template <int NP> struct FtCfg;
template <> struct FtCfg<2> { static constexpr int NS = 2, NPROD = 3, N = 256; };
template <> struct FtCfg<3> { static constexpr int NS = 2, NPROD = 6, N = 128; };

// (A piece, B piece) of product q, small terms first.
template <int NP>
__device__ __forceinline__ void prod_pieces(int q, int &pa, int &pb) {
    if (NP == 2) {
        constexpr int A[3] = {1, 0, 0}, B[3] = {0, 1, 0};
        pa = A[q]; pb = B[q];
    } else {
        constexpr int A[6] = {2, 1, 0, 1, 0, 0}, B[6] = {0, 1, 2, 0, 1, 0};
        pa = A[q]; pb = B[q];
    }
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity; false after limit_ns (the abort
// flag is then set) or, when honor_abort, as soon as another role aborted.
__device__ __noinline__ bool ft_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag,
                                     bool honor_abort, unsigned long long limit_ns = FT_WAIT_NS) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_try(bar, parity)) return true;
        if (honor_abort && *abort_flag) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            *abort_flag = 1;
            return false;
        }
    }
}

// Lane 0 waits; the whole warp takes its result (phase reached, or gave up).
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int *abort_flag) {
    bool ok = true;
    if ((threadIdx.x & 31) == 0) ok = ft_wait(bar, parity, abort_flag, true);
    return __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int NP>
__host__ __device__ constexpr size_t ft_stage_bytes() {
    return (size_t)NP * FT_PIECE_BYTES * (1 + FtCfg<NP>::N / FT_M);
}
template <int NP>
constexpr size_t ft_smem_bytes() {
    return 1024 + (size_t)FtCfg<NP>::NS * ft_stage_bytes<NP>() + FT_CTRL_BYTES;
}

// Unit u's parameters: the kernel argument, or (batched) the instance i with
// unit_start[i] <= u < unit_start[i + 1]; `local` = u's index in its instance.
template <bool BAT>
__device__ __forceinline__ const PassParams &unit_params(const PassParams &P0, const PassParams *plist,
                                                        const int *unit_start, int count, int u,
                                                        int &local) {
    if (!BAT) {
        local = u;
        return P0;
    }
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (unit_start[mid] <= u) lo = mid;
        else hi = mid - 1;
    }
    local = u - unit_start[lo];
    return plist[lo];
}

// The pass does not run for this instance now (solver stopped, or gated).
__device__ __forceinline__ bool pass_skipped(const PassParams &Q) {
    const Ctl *c = Q.ctl;
    if (!c) return false;
    if (c->stop) return true;
    if (Q.gate == GATE_CHECK && !c->do_check) return true;
    if (Q.gate == GATE_NOCHECK && c->do_check) return true;
    return false;
}

// One CTA per SM; units (row tile, column-tile slice) strided over the grid.
// BAT: units of many instances (plist / unit_start, total_units in all);
// otherwise the units of P0 (P0.ft_rtiles x P0.ft_splits).
template <int NP, int ACC, bool MOM, bool BAT>
__global__ void __launch_bounds__(FT_THREADS, 1)
    feat_reduce_kernel(const __grid_constant__ PassParams P0, const PassParams *plist,
                       const int *unit_start, int count, int total_units, int *batch_err) {
    constexpr int NS = FtCfg<NP>::NS;
    constexpr int NPROD = FtCfg<NP>::NPROD;
    constexpr int FT_N = FtCfg<NP>::N;
    constexpr int NB = FT_N / FT_M;                      // packed blocks per column tile
    constexpr uint32_t FT_TMEM_COLS = 2u * FT_N;         // two accumulators
    constexpr uint32_t STAGE = (uint32_t)ft_stage_bytes<NP>();
    constexpr uint32_t BOFF = (uint32_t)(NP * FT_PIECE_BYTES);   // B pieces after the A pieces
    extern __shared__ unsigned char ft_raw[];

    if (!BAT && pass_skipped(P0)) return;
    const int units = BAT ? total_units : P0.ft_rtiles * P0.ft_splits;

    const uint32_t raw = smem_u32(ft_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;            // swizzle atoms need 1024-byte alignment
    unsigned char *ctrl = ft_raw + (base - raw) + (size_t)NS * STAGE;
    const uint32_t bar0 = smem_u32(ctrl);                    // full[NS], empty[NS], accf[2], acce[2], drain
    const uint32_t FULL = bar0, EMPTY = bar0 + 8u * NS, ACCF = bar0 + 16u * NS,
                   ACCE = ACCF + 16u, DRAIN = ACCE + 16u;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(ctrl + 8 * (2 * NS + 5));
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    float *colterm = reinterpret_cast<float *>(ctrl + 1024);  // [4 warps][2][FT_N]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(FULL + 8u * s, 1);
            mbar_init(EMPTY + 8u * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(ACCF + 8u * b, 1);
            mbar_init(ACCE + 8u * b, 4);
        }
        mbar_init(DRAIN, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(FT_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t *>(tmem_slot);

    if (warp == 0) {
        // ------------------------------------------------ producer
        int it = 0;
        int last_use[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) last_use[s] = -1;
        bool ok = true;
        for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
            int local;
            const PassParams &Q = unit_params<BAT>(P0, plist, unit_start, count, u, local);
            if (BAT && pass_skipped(Q)) continue;
            const int splits = Q.ft_splits, tps = Q.ft_tps, ctiles = Q.ft_ctiles;
            const int rblk = Q.ft_rblk, cblk = Q.ft_cblk, nkb = Q.fkb;
            const int rt = local / splits, sp = local - (local / splits) * splits;
            const int ct0 = sp * tps, ct1 = min(ctiles, ct0 + tps);
            for (int ct = ct0; ok && ct < ct1; ++ct) {
                for (int kb = 0; kb < nkb; ++kb, ++it) {
                    const int s = it % NS;
                    const uint32_t use = (uint32_t)(it / NS);
                    if (!warp_wait(EMPTY + 8u * s, (use & 1u) ^ 1u, abort_flag)) { ok = false; break; }
                    if (lane == 0) {
                        const uint32_t dst = base + (uint32_t)s * STAGE;
                        mbar_expect_tx(FULL + 8u * s, STAGE);
#pragma unroll
                        for (int p = 0; p < NP; ++p)
                            bulk_g2s(dst + p * FT_PIECE_BYTES,
                                     Q.fx + ((size_t)(p * rblk + rt) * nkb + kb) * FT_PIECE_ELEMS,
                                     FT_PIECE_BYTES, FULL + 8u * s);
#pragma unroll
                        for (int p = 0; p < NP; ++p)
#pragma unroll
                            for (int hb = 0; hb < NB; ++hb)
                                bulk_g2s(dst + BOFF + (p * NB + hb) * FT_PIECE_BYTES,
                                         Q.fy + ((size_t)(p * cblk + ct * NB + hb) * nkb + kb) * FT_PIECE_ELEMS,
                                         FT_PIECE_BYTES, FULL + 8u * s);
#pragma unroll
                        for (int s2 = 0; s2 < NS; ++s2)
                            if (s2 == s) last_use[s2] = (int)use;
                    }
                    __syncwarp();
                }
            }
        }
        // every issued copy has landed before the CTA may exit
        if (lane == 0) {
#pragma unroll
            for (int s = 0; s < NS; ++s)
                if (last_use[s] >= 0) ft_wait(FULL + 8u * s, (uint32_t)last_use[s] & 1u, abort_flag, false);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issue
        // kind::f16 instruction descriptor: D f32, A/B bf16, both K-major, N, M
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(FT_N >> 3) << 17) |
                               ((uint32_t)(FT_M >> 4) << 24);
        int it = 0, tc = 0;
        bool ok = true;
        for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
            int local;
            const PassParams &Q = unit_params<BAT>(P0, plist, unit_start, count, u, local);
            if (BAT && pass_skipped(Q)) continue;
            const int splits = Q.ft_splits, tps = Q.ft_tps, ctiles = Q.ft_ctiles, nkb = Q.fkb;
            const int sp = local - (local / splits) * splits;
            const int ct0 = sp * tps, ct1 = min(ctiles, ct0 + tps);
            for (int ct = ct0; ok && ct < ct1; ++ct, ++tc) {
                const int b = tc & 1;
                const uint32_t ub = (uint32_t)(tc >> 1);
                if (!warp_wait(ACCE + 8u * b, (ub & 1u) ^ 1u, abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t dacc = tmem + (uint32_t)(b * FT_N);
                for (int kb = 0; kb < nkb; ++kb, ++it) {
                    const int s = it % NS;
                    const uint32_t use = (uint32_t)(it / NS);
                    if (!warp_wait(FULL + 8u * s, use & 1u, abort_flag)) { ok = false; break; }
                    tc_fence_after();
                    if (lane == 0) {
                        const uint32_t sa = base + (uint32_t)s * STAGE;
#pragma unroll
                        for (int q = 0; q < NPROD; ++q) {
                            int pa, pb;
                            prod_pieces<NP>(q, pa, pb);
#pragma unroll
                            for (int k4 = 0; k4 < FT_K / 16; ++k4) {
                                const uint64_t ad = sw128_desc(sa + pa * FT_PIECE_BYTES + k4 * 32);
                                const uint64_t bd = sw128_desc(sa + BOFF + pb * NB * FT_PIECE_BYTES + k4 * 32);
                                umma_bf16(dacc, ad, bd, idesc, (kb | q | k4) != 0 ? 1u : 0u);
                            }
                        }
                        umma_commit(EMPTY + 8u * s);   // stage s free once these MMAs are done
                    }
                    __syncwarp();
                }
                if (!ok) break;
                if (lane == 0) umma_commit(ACCF + 8u * b);   // accumulator b complete
                __syncwarp();
            }
        }
        // no MMA may still write TMEM when it is freed
        if (lane == 0) {
            umma_commit(DRAIN);
            ft_wait(DRAIN, 0u, abort_flag, false);
        }
        __syncwarp();
    } else {
        // ------------------------------------------------ epilogue (warps 2-5)
        const int quad = warp & 3;                  // TMEM lanes this warp may read
        const int rloc = quad * 32 + lane;          // row within the tile
        float *gw = colterm + (size_t)(warp - 2) * 2 * FT_N;   // this warp's column terms
        float *yw = gw + FT_N;
        int tc = 0;
        bool ok = true;
        for (int u = blockIdx.x; ok && u < units; u += gridDim.x) {
            int local;
            const PassParams &Q = unit_params<BAT>(P0, plist, unit_start, count, u, local);
            if (BAT && pass_skipped(Q)) continue;
            double alpha = 0.0, beta = 0.0;
            if (ACC == ACC_LSE) resolve_coefs(Q, alpha, beta);
            const double a2 = alpha * LOG2E;
            const double cb = Q.colpot_unit ? LOG2E : beta * LOG2E;
            const float k2 = (float)(-2.0 * a2);    // log2 exponent per unit of <x, y>
            const int splits = Q.ft_splits, tps = Q.ft_tps, ctiles = Q.ft_ctiles;
            const int rt = local / splits, sp = local - (local / splits) * splits;
            const int ct0 = sp * tps, ct1 = min(ctiles, ct0 + tps);
            const int n = Q.n, m = Q.m;
            const int row = rt * FT_M + rloc;
            const float xnf = (MOM && row < n) ? (float)Q.xn[row] : 0.f;
            float M = (ACC == ACC_MIN) ? INFINITY : ((ACC == ACC_MAX) ? -INFINITY : -1e30f);
            KSum S;
            S.s = 0.f;
            S.c = 0.f;
            float MO = 0.f;
            for (int ct = ct0; ct < ct1; ++ct, ++tc) {
                const int b = tc & 1;
                const uint32_t ub = (uint32_t)(tc >> 1);
                // column terms of this tile (each warp keeps its own copy)
                __syncwarp();
#pragma unroll
                for (int i = 0; i < FT_N / 32; ++i) {
                    const int jj = i * 32 + lane;
                    const int j = ct * FT_N + jj;
                    float g, yv = 0.f;
                    if (j < m) {
                        const double pot = Q.colpot ? Q.colpot[j] : 0.0;
                        const double ynj = Q.yn[j];
                        if (ACC == ACC_LSE) g = (float)(((cb == 0.0) ? 0.0 : cb * pot) + a2 * ynj);
                        else if (ACC == ACC_MIN) g = (float)(ynj + Q.minmax_scale * pot);
                        else g = (float)ynj;
                        yv = (float)ynj;
                    } else {
                        g = (ACC == ACC_MIN) ? INFINITY : -INFINITY;
                    }
                    gw[jj] = g;
                    if (MOM) yw[jj] = yv;
                }
                __syncwarp();
                if (!warp_wait(ACCF + 8u * b, ub & 1u, abort_flag)) { ok = false; break; }
                tc_fence_after();
                const uint32_t taddr = tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(b * FT_N);
#pragma unroll 1
                for (int c = 0; c < FT_N / 32; ++c) {
                    uint32_t r[32];
                    tmem_ld32(taddr + (uint32_t)(c * 32), r);
                    const float *gc = gw + c * 32;
                    if (ACC == ACC_LSE) {
                        float v[32];
                        float vm = -INFINITY;
#pragma unroll
                        for (int k = 0; k < 32; ++k) {
                            v[k] = fmaf(k2, __uint_as_float(r[k]), gc[k]);
                            vm = fmaxf(vm, v[k]);
                        }
                        if (vm > M) {
                            const float f = ex2_approx(M - vm);
                            S.scale(f);
                            if (MOM) MO *= f;
                            M = vm;
                        }
                        float cs = 0.f;
#pragma unroll
                        for (int k = 0; k < 32; ++k) {
                            const float ev = ex2_approx(v[k] - M);
                            cs += ev;
                            if (MOM) {
                                const float cst = fmaf(-2.f, __uint_as_float(r[k]), xnf + yw[c * 32 + k]);
                                MO = fmaf(ev, cst, MO);
                            }
                        }
                        S.add(cs);
                    } else if (ACC == ACC_MIN) {
#pragma unroll
                        for (int k = 0; k < 32; ++k) M = fminf(M, fmaf(-2.f, __uint_as_float(r[k]), gc[k]));
                    } else {
#pragma unroll
                        for (int k = 0; k < 32; ++k) M = fmaxf(M, fmaf(-2.f, __uint_as_float(r[k]), gc[k]));
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(ACCE + 8u * b);   // accumulator b may be overwritten
            }
            if (!ok) break;
            if (row < n) {
                double *pp = Q.part + ((size_t)sp * n + row) * 3;
                if (ACC == ACC_LSE) {
                    pp[0] = (double)M;
                    pp[1] = (double)S.s - (double)S.c;
                    if (MOM) pp[2] = (double)MO;
                } else {
                    pp[0] = (double)M + Q.xn[row];
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(FT_TMEM_COLS)
                     : "memory");
    if (threadIdx.x == 0 && *abort_flag) {
        if (BAT) {
            if (batch_err) atomicExch(batch_err, CULAMP_ERR_DEVICE_TIMEOUT);
        } else if (P0.ctl) {
            P0.ctl->error = CULAMP_ERR_DEVICE_TIMEOUT;
            P0.ctl->stop = 1;
        }
    }
}

// Merge the column-slice partials of each row and run the pass epilogue.
// BAT: blocks of many instances (block_start[i] .. block_start[i+1]-1 are the
// row blocks of instance i, P.nrb of them).
template <int ACC, bool MOM, bool BAT>
__global__ void __launch_bounds__(TPB)
    feat_merge_kernel(const __grid_constant__ PassParams P0, const PassParams *plist,
                      const int *block_start, int count) {
    __shared__ double red[4 * (TPB / 32)];
    __shared__ int s_last;
    __shared__ int s_blk[2];
    __shared__ __align__(16) PassParams sP;
    if constexpr (BAT) {
        if (threadIdx.x == 0) {
            int lo = 0, hi = count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (block_start[mid] <= (int)blockIdx.x) lo = mid;
                else hi = mid - 1;
            }
            s_blk[0] = (int)blockIdx.x - block_start[lo];
            s_blk[1] = lo;
        }
        __syncthreads();
        const int *src = reinterpret_cast<const int *>(plist + s_blk[1]);
        int *dst = reinterpret_cast<int *>(&sP);
        for (int k = threadIdx.x; k < (int)(sizeof(PassParams) / sizeof(int)); k += TPB) dst[k] = src[k];
        __syncthreads();
    }
    const PassParams &P = *(BAT ? &sP : &P0);
    const int rb = BAT ? s_blk[0] : (int)blockIdx.x;
    const int nrb = BAT ? P.nrb : (int)gridDim.x;
    Ctl *ctl = P.ctl;
    if (ctl) {
        if (ctl->stop) return;
        if (P.gate == GATE_CHECK && !ctl->do_check) return;
        if (P.gate == GATE_NOCHECK && ctl->do_check) return;
    }
    double alpha = 0.0, beta = 0.0;
    if (ACC == ACC_LSE) resolve_coefs(P, alpha, beta);
    const int row_base = rb * (TPB * RPT);
    double Mv[RPT], Sv[RPT], MOMv[RPT], Hv[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int row = row_base + threadIdx.x + r * TPB;
        double M = (ACC == ACC_MIN) ? INFINITY : -INFINITY, S = 0.0, MO = 0.0;
        if (row < P.n) {
            for (int s = 0; s < P.splits; ++s) {
                const double *pp = P.part + ((size_t)s * P.n + row) * 3;
                const double m2 = pp[0];
                if (ACC == ACC_LSE) merge_lse(M, S, MO, m2, pp[1], MOM ? pp[2] : 0.0);
                else if (ACC == ACC_MAX) M = fmax(M, m2);
                else M = fmin(M, m2);
            }
        }
        Mv[r] = M;
        Sv[r] = S;
        MOMv[r] = MO;
        Hv[r] = (ACC == ACC_LSE && row < P.n) ? alpha * LOG2E * P.xn[row] : 0.0;
    }
    row_epilogue<ACC, RPT>(P, rb, row_base, beta, Mv, Sv, MOMv, Hv, red, s_last, nrb);
}

// Round to the nearest bf16 value, ties to even, on the FP64 bit pattern (keep
// 7 of the 52 stored mantissa bits); returns the rounded value as a double and
// its bf16 encoding. Exact for the magnitudes features take (no overflow, no
// float subnormals).
__device__ __forceinline__ double bf16_round(double v, uint16_t &bits) {
    unsigned long long b = (unsigned long long)__double_as_longlong(v);
    b += 0x0FFFFFFFFFFFull + ((b >> 45) & 1ull);
    b &= ~0x1FFFFFFFFFFFull;
    const double r = __longlong_as_double((long long)b);
    bits = (uint16_t)(__float_as_uint((float)r) >> 16);
    return r;
}

// Split one cloud into bf16 pieces in the swizzled tile image; one thread per
// 16-byte chunk (8 consecutive features of one point). Piece p is the bf16
// rounding of what pieces 0..p-1 leave of the value.
__global__ void feat_pack_kernel(uint16_t *out, const double *X, int n, int d, int tiles, int nkb, int np) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)tiles * FT_M * nkb * 8;
    if (idx >= total) return;
    const int c = (int)(idx & 7);
    const long long t = idx >> 3;
    const int kb = (int)(t % nkb);
    const int row = (int)(t / nkb);
    double v[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        const int k = kb * FT_K + c * 8 + e;
        v[e] = (row < n && k < d) ? X[(size_t)row * d + k] : 0.0;
    }
    const int rt = row / FT_M, r = row % FT_M;
    for (int p = 0; p < np; ++p) {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            uint16_t b0, b1;
            v[2 * i] -= bf16_round(v[2 * i], b0);
            v[2 * i + 1] -= bf16_round(v[2 * i + 1], b1);
            w[i] = (uint32_t)b0 | ((uint32_t)b1 << 16);
        }
        uint16_t *dst = out + ((size_t)(p * tiles + rt) * nkb + kb) * FT_PIECE_ELEMS + (size_t)r * FT_K +
                        (size_t)((c ^ (r & 7)) * 8);
        *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// |x_i|^2 in FP64, one warp per point.
__global__ void feat_norm_kernel(double *out, const double *X, int n, int d) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int k = lane; k < d; k += 32) {
        const double v = X[(size_t)row * d + k];
        s = fma(v, v, s);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) out[row] = s;
}

template <int NP, int ACC, bool MOM, bool BAT>
cudaError_t launch_ft(const PassParams &P, const PassParams *plist, const int *unit_start,
                      const int *block_start, int count, int total_units, int merge_blocks,
                      int grid, int *batch_err, cudaStream_t st) {
    auto kern = feat_reduce_kernel<NP, ACC, MOM, BAT>;
    constexpr size_t smem = ft_smem_bytes<NP>();
    static bool attr_set = false;   // per instantiation; same value on every device
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    kern<<<grid, FT_THREADS, smem, st>>>(P, plist, unit_start, count, total_units, batch_err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    feat_merge_kernel<ACC, MOM, BAT><<<merge_blocks, TPB, 0, st>>>(P, plist, block_start, count);
    return cudaGetLastError();
}

template <bool BAT>
cudaError_t launch_ft_any(int np, int acc, bool mom, const PassParams &P, const PassParams *plist,
                          const int *unit_start, const int *block_start, int count, int total_units,
                          int merge_blocks, int grid, int *batch_err, cudaStream_t st) {
#define CULAMP_FT(NP_, ACC_, MOM_) \
    launch_ft<NP_, ACC_, MOM_, BAT>(P, plist, unit_start, block_start, count, total_units, merge_blocks, grid, batch_err, st)
    if (np == 2) {
        if (acc == ACC_LSE) return mom ? CULAMP_FT(2, ACC_LSE, true) : CULAMP_FT(2, ACC_LSE, false);
        if (acc == ACC_MAX) return CULAMP_FT(2, ACC_MAX, false);
        return CULAMP_FT(2, ACC_MIN, false);
    }
    if (acc == ACC_LSE) return mom ? CULAMP_FT(3, ACC_LSE, true) : CULAMP_FT(3, ACC_LSE, false);
    if (acc == ACC_MAX) return CULAMP_FT(3, ACC_MAX, false);
    return CULAMP_FT(3, ACC_MIN, false);
#undef CULAMP_FT
}

}  // namespace

namespace culamp_host {

int feat_kblocks(int d) { return (d + FT_K - 1) / FT_K; }

// 128-point blocks of a packed cloud: an even count, so that any cloud can be
// read as 256-column tiles (zero points pad the last block pair).
int feat_blocks(int n) { return 2 * ((n + 2 * FT_M - 1) / (2 * FT_M)); }

int feat_tile_cols(int pieces) { return pieces == 2 ? FtCfg<2>::N : FtCfg<3>::N; }

size_t feat_piece_elems(int n, int d, int pieces) {
    return (size_t)pieces * (size_t)feat_blocks(n) * FT_M * (size_t)feat_kblocks(d) * FT_K;
}

// Work units: 128-row tiles x slices of N-column tiles. The slice count is
// the smallest that minimises the tiles of the busiest CTA (one CTA per SM),
// plus a small charge per slice for the partials and their merge.
FeatShape feat_shape(int n, int m, int sm_count, int pieces) {
    FeatShape fs{};
    const int sms = sm_count > 0 ? sm_count : 148;
    const int N = feat_tile_cols(pieces);
    fs.rtiles = (n + FT_M - 1) / FT_M;
    fs.ctiles = (m + N - 1) / N;
    fs.rblk = feat_blocks(n);
    fs.cblk = feat_blocks(m);
    fs.ncols = N;
    double best = 1e300;
    const int smax = fs.ctiles < 64 ? fs.ctiles : 64;
    for (int s = 1; s <= smax; ++s) {
        const int tps = (fs.ctiles + s - 1) / s;
        const int sp = (fs.ctiles + tps - 1) / tps;
        const long long units = (long long)fs.rtiles * sp;
        const long long grid = units < sms ? units : sms;
        const long long waves = (units + grid - 1) / grid;
        const double cost = (double)waves * tps + 0.05 * sp;
        if (cost < best - 1e-9) {
            best = cost;
            fs.splits = sp;
            fs.tps = tps;
            fs.units = (int)units;
            fs.grid = (int)grid;
        }
    }
    fs.merge_rb = (n + TPB * RPT - 1) / (TPB * RPT);
    fs.part_bytes = (size_t)fs.splits * (size_t)n * 3 * sizeof(double);
    return fs;
}

cudaError_t feat_prepare(uint16_t *pieces, double *norms, const double *X, int n, int d, int np,
                         cudaStream_t st) {
    const int tiles = feat_blocks(n);
    const int nkb = feat_kblocks(d);
    const long long total = (long long)tiles * FT_M * nkb * 8;
    feat_pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(pieces, X, n, d, tiles, nkb, np);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    feat_norm_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(norms, X, n, d);
    return cudaGetLastError();
}

cudaError_t launch_feat_pass(PassParams P, int acc, Scratch &scr, int sm_count, cudaStream_t st) {
    if (!P.fx || !P.fy || !P.xn || !P.yn || P.fkb < 1 || (P.fpieces != 2 && P.fpieces != 3))
        return cudaErrorInvalidValue;
    const FeatShape fs = feat_shape(P.n, P.m, sm_count, P.fpieces);
    if (scr.part.bytes < fs.part_bytes || scr.tickets.bytes < (size_t)(fs.merge_rb + 1) * sizeof(unsigned) ||
        scr.blk.bytes < (size_t)fs.merge_rb * 4 * sizeof(double))
        return cudaErrorInvalidValue;
    set_feat_geometry(P, fs);
    P.part = scr.part.as<double>();
    P.rb_ticket = scr.tickets.as<unsigned>();
    P.grid_ticket = scr.tickets.as<unsigned>() + fs.merge_rb;
    P.blk = scr.blk.as<double>();
    return launch_ft_any<false>(P.fpieces, acc, P.want_moment != 0, P, nullptr, nullptr, nullptr, 1,
                                fs.units, fs.merge_rb, fs.grid, nullptr, st);
}

void set_feat_geometry(PassParams &P, const FeatShape &fs) {
    P.splits = fs.splits;
    P.cols_per_split = fs.tps * fs.ncols;
    P.nrb = fs.merge_rb;
    P.ft_rtiles = fs.rtiles;
    P.ft_ctiles = fs.ctiles;
    P.ft_rblk = fs.rblk;
    P.ft_cblk = fs.cblk;
    P.ft_splits = fs.splits;
    P.ft_tps = fs.tps;
}

cudaError_t launch_feat_batched(int np, int acc, bool mom, const PassParams *plist, const int *unit_start,
                                const int *block_start, int count, int total_units, int merge_blocks,
                                int sm_count, int *batch_err, cudaStream_t st) {
    if (count < 1 || total_units < 1) return cudaSuccess;
    PassParams dummy;
    memset(&dummy, 0, sizeof(dummy));
    const int grid = total_units < sm_count ? total_units : sm_count;
    return launch_ft_any<true>(np, acc, mom, dummy, plist, unit_start, block_start, count, total_units,
                               merge_blocks, grid, batch_err, st);
}

}  // namespace culamp_host

// ---------------------------------------------------------------------------
// Probe of the bounded wait above: one CTA waits, with the given limit, on an
// mbarrier phase that nothing completes (no thread arrives, no copy is
// issued), so the wait must give up, set the abort flag and return -- the
// path every role of feat_reduce_kernel takes when a copy or an MMA never
// completes. The host reads the outcome; the context stays usable.
namespace {
__global__ void wait_probe_kernel(unsigned long long limit_ns, int *out) {
    __shared__ __align__(8) unsigned long long bar;
    __shared__ int abort_flag;
    const uint32_t b = smem_u32(&bar);
    if (threadIdx.x == 0) {
        mbar_init(b, 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    bool ok = true;
    if (threadIdx.x == 0) ok = ft_wait(b, 0u, &abort_flag, false, limit_ns);
    __syncthreads();
    if (threadIdx.x == 0) {
        out[0] = ok ? 0 : 1;
        out[1] = abort_flag;
    }
}
}  // namespace

extern "C" int culamp_probe_wait(culamp_handle h, uint64_t limit_ns, void *stream) {
    if (!h) return CULAMP_ERR_INVALID_ARG;
    if (limit_ns == 0 || limit_ns > 10000000000ull)
        return culamp_set_error(h, CULAMP_ERR_INVALID_ARG, "wait limit must be in (0, 10 s]");
    cudaSetDevice(h->device);
    cudaStream_t st = (cudaStream_t)stream;
    if (h->tmpA.reserve(2 * sizeof(int)) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_ALLOC, "probe buffer");
    int *dev = h->tmpA.as<int>();
    wait_probe_kernel<<<1, 32, 0, st>>>((unsigned long long)limit_ns, dev);
    int out[2] = {-1, -1};
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(out, dev, sizeof(out), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return culamp_set_error(h, CULAMP_ERR_CUDA, "wait probe failed");
    if (out[0] == 1 && out[1] == 1)
        return culamp_set_error(h, CULAMP_ERR_DEVICE_TIMEOUT, "bounded wait gave up after %llu ns",
                                (unsigned long long)limit_ns);
    return culamp_set_error(h, CULAMP_ERR_CUDA, "bounded wait did not give up (%d, %d)", out[0], out[1]);
}
