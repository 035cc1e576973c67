// maxcost.cu -- W_inf = max_ij C(x_i, y_j), exact, register-tiled FP64.
//
// The normaliser of every solver (MirrorProxKernel.jl:280-326, the max pass
// the Sinkhorn and LAMP drivers call before iterating) is the largest pair
// cost. The row-per-thread pair loop re-reads each row's d coordinates per
// pair and runs at a few per cent of the FP64 pipe for d >= 32; here a CTA
// takes a 64 x 64 tile of pairs, stages both clouds through shared memory in
// 16-coordinate chunks and each thread holds a 4 x 4 block of partial costs in
// registers (8 shared loads per 16 pair updates). Every pair's cost is formed
// exactly as the pair loops form it -- coordinates in ascending order,
// (x_k - y_k) then fma / add / max / pow -- so the maximum is bit-identical.
//
// Costs are >= +0, so their IEEE bit patterns order like unsigned integers and
// each CTA folds its maximum into the destination with one 64-bit atomicMax;
// the destination must hold +0 (all-zero bits) before the launch. One launch
// covers any number of (X, Y) jobs: blocks loop over the tiles of all jobs
// (a prefix table over the jobs' tile counts), so small and large instances
// share one grid.
#include <cuda_runtime.h>

#include <cstring>

#include "internal.h"

namespace culamp_dev {

constexpr int MC_T = 64;        // tile rows = tile columns
constexpr int MC_K = 16;        // coordinates per shared-memory chunk
constexpr int MC_THREADS = 256; // 16 x 16 threads, 4 x 4 pairs each

struct MaxCostJob {
    const double *X, *Y;        // point-major, ld = d
    int n, m, d;
    int col_tiles;
    unsigned long long *dst;    // bits of a double holding +0 before the launch
};

struct MaxCostArgs {
    const MaxCostJob *jobs;     // device table (null: `one` is the only job)
    const long long *tile_start;// count + 1 prefix of tiles per job (device)
    int count;
    long long total_tiles;
    double pexp;
    MaxCostJob one;
};

template <int PM>
__device__ __forceinline__ void mc_step(double &acc, double df, double pexp) {
    if (PM == P_SQ) acc = fma(df, df, acc);
    else if (PM == P_L1) acc += fabs(df);
    else if (PM == P_INF) acc = fmax(acc, fabs(df));
    else acc += pow(fabs(df), pexp);
}

template <int PM>
__global__ void __launch_bounds__(MC_THREADS) max_cost_kernel(const __grid_constant__ MaxCostArgs A) {
    __shared__ double xs[MC_K][MC_T];
    __shared__ double ys[MC_K][MC_T];
    __shared__ double red[MC_THREADS / 32];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    for (long long t = blockIdx.x; t < A.total_tiles; t += gridDim.x) {
        int job = 0;
        if (A.jobs) {
            int lo = 0, hi = A.count - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (A.tile_start[mid] <= t) lo = mid;
                else hi = mid - 1;
            }
            job = lo;
        }
        const MaxCostJob J = A.jobs ? A.jobs[job] : A.one;
        const long long local = t - (A.jobs ? A.tile_start[job] : 0);
        const int r0 = (int)(local / J.col_tiles) * MC_T;
        const int c0 = (int)(local % J.col_tiles) * MC_T;
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
        for (int k0 = 0; k0 < J.d; k0 += MC_K) {
            __syncthreads();
            // 64 points x 16 coordinates of each cloud; out-of-range entries are 0
            // (their pairs are masked out below)
            for (int e = tid; e < MC_T * MC_K; e += MC_THREADS) {
                const int p = e / MC_K, k = e % MC_K;
                const int kk = k0 + k;
                const int rx = r0 + p, cy = c0 + p;
                xs[k][p] = (rx < J.n && kk < J.d) ? J.X[(size_t)rx * J.d + kk] : 0.0;
                ys[k][p] = (cy < J.m && kk < J.d) ? J.Y[(size_t)cy * J.d + kk] : 0.0;
            }
            __syncthreads();
            const int kn = min(MC_K, J.d - k0);
            for (int k = 0; k < kn; ++k) {
                double a[4], b[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = xs[k][ty + 16 * i];
#pragma unroll
                for (int j = 0; j < 4; ++j) b[j] = ys[k][tx + 16 * j];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) mc_step<PM>(acc[i][j], a[i] - b[j], A.pexp);
            }
        }
        double mx = 0.0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (r0 + ty + 16 * i < J.n && c0 + tx + 16 * j < J.m) mx = fmax(mx, acc[i][j]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
        if ((tid & 31) == 0) red[tid >> 5] = mx;
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < MC_THREADS / 32; ++w) mx = fmax(mx, red[w]);
            atomicMax(J.dst, (unsigned long long)__double_as_longlong(mx));
        }
    }
}

}  // namespace culamp_dev

namespace culamp_host {

using culamp_dev::MaxCostArgs;
using culamp_dev::MaxCostJob;

static cudaError_t launch_max_cost_args(const MaxCostArgs &A, int pmode, int sm_count, cudaStream_t st) {
    if (A.total_tiles <= 0) return cudaSuccess;
    // persistent: up to 8 CTAs per SM loop over the tiles
    const long long cap = (long long)sm_count * 8;
    const unsigned grid = (unsigned)(A.total_tiles < cap ? A.total_tiles : cap);
    switch (pmode) {
        case culamp_dev::P_SQ: culamp_dev::max_cost_kernel<culamp_dev::P_SQ><<<grid, culamp_dev::MC_THREADS, 0, st>>>(A); break;
        case culamp_dev::P_L1: culamp_dev::max_cost_kernel<culamp_dev::P_L1><<<grid, culamp_dev::MC_THREADS, 0, st>>>(A); break;
        case culamp_dev::P_INF: culamp_dev::max_cost_kernel<culamp_dev::P_INF><<<grid, culamp_dev::MC_THREADS, 0, st>>>(A); break;
        default: culamp_dev::max_cost_kernel<culamp_dev::P_GEN><<<grid, culamp_dev::MC_THREADS, 0, st>>>(A); break;
    }
    return cudaGetLastError();
}

static int tiles_of(int k) { return (k + culamp_dev::MC_T - 1) / culamp_dev::MC_T; }

cudaError_t launch_max_cost(const double *X, const double *Y, int n, int m, int d, double p,
                            double *dst, int sm_count, cudaStream_t st) {
    MaxCostArgs A;
    std::memset(&A, 0, sizeof(A));
    A.count = 1;
    A.pexp = p;
    A.one.X = X;
    A.one.Y = Y;
    A.one.n = n;
    A.one.m = m;
    A.one.d = d;
    A.one.col_tiles = tiles_of(m);
    A.one.dst = reinterpret_cast<unsigned long long *>(dst);
    A.total_tiles = (long long)tiles_of(n) * tiles_of(m);
    return launch_max_cost_args(A, pmode_of(p), sm_count, st);
}

size_t max_cost_table_bytes(int count) {
    return (size_t)count * sizeof(MaxCostJob) + (size_t)(count + 1) * sizeof(long long) + 16;
}

cudaError_t launch_max_cost_batched(const MaxCostInput *in, int count, double p, void *table,
                                    std::vector<unsigned char> &host_table, int sm_count,
                                    cudaStream_t st) {
    if (count <= 0) return cudaSuccess;
    host_table.assign(max_cost_table_bytes(count), 0);
    MaxCostJob *jobs = reinterpret_cast<MaxCostJob *>(host_table.data());
    long long *start = reinterpret_cast<long long *>(host_table.data() + (size_t)count * sizeof(MaxCostJob));
    long long tot = 0;
    for (int i = 0; i < count; ++i) {
        jobs[i].X = in[i].X;
        jobs[i].Y = in[i].Y;
        jobs[i].n = in[i].n;
        jobs[i].m = in[i].m;
        jobs[i].d = in[i].d;
        jobs[i].col_tiles = tiles_of(in[i].m);
        jobs[i].dst = reinterpret_cast<unsigned long long *>(in[i].dst);
        start[i] = tot;
        tot += (long long)tiles_of(in[i].n) * tiles_of(in[i].m);
    }
    start[count] = tot;
    cudaError_t e = cudaMemcpyAsync(table, host_table.data(), host_table.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return e;
    MaxCostArgs A;
    std::memset(&A, 0, sizeof(A));
    A.jobs = reinterpret_cast<const MaxCostJob *>(table);
    A.tile_start = reinterpret_cast<const long long *>(reinterpret_cast<unsigned char *>(table) +
                                                       (size_t)count * sizeof(MaxCostJob));
    A.count = count;
    A.total_tiles = tot;
    A.pexp = p;
    return launch_max_cost_args(A, pmode_of(p), sm_count, st);
}

}  // namespace culamp_host
