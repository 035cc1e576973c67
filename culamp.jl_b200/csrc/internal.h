// internal.h -- host-side internals shared by the libculamp_b200 translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/culamp.h"
#include "engine.cuh"

namespace culamp_host {

using culamp_dev::Ctl;
using culamp_dev::PassParams;

// Growable device buffer owned by a handle.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t want, bool zero = false) {
        if (want <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, want);
        if (e != cudaSuccess) { ptr = nullptr; return e; }
        bytes = want;
        if (zero) e = cudaMemset(ptr, 0, want);
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return reinterpret_cast<T *>(ptr); }
};

// Scratch used by one pair pass (split partials, tickets, block partials).
struct Scratch {
    DevBuf part;       // splits * rows * 3 doubles
    DevBuf tickets;    // row blocks + 1 unsigned, zero-initialised, re-armed by kernels
    DevBuf blk;        // row blocks * 4 doubles
    cudaError_t reserve(size_t part_bytes, size_t nrb) {
        cudaError_t e = part.reserve(part_bytes > 0 ? part_bytes : 8);
        if (e != cudaSuccess) return e;
        e = tickets.reserve((nrb + 1) * sizeof(unsigned), true);
        if (e != cudaSuccess) return e;
        return blk.reserve(nrb * 4 * sizeof(double) + 32);
    }
    void release() { part.release(); tickets.release(); blk.release(); }
};

struct LaunchShape {
    int R;             // output rows per thread (RPT or RPT_BIG)
    int rb;            // row blocks
    int splits;        // column splits
    int cols_per_split;
    size_t smem;       // dynamic shared memory bytes
    size_t part_bytes; // split scratch bytes
    int sms;           // SM count the shape was made for
};

// Grid and scratch requirement of a pass over n output rows and m columns.
// `mom`: the pass accumulates the cost moment (selects the RPT variant).
LaunchShape pass_shape(int n, int m, int d, int acc, int sm_count, bool mom = false);

// Launch one pair pass. The scratch must already hold pass_shape(...) bytes
// (so the call is legal inside stream capture).
cudaError_t launch_pass(PassParams P, int pmode, int acc, const LaunchShape &sh, Scratch &scr,
                        cudaStream_t st);

// The same with explicit scratch (partials, row-block tickets + grid ticket,
// block scalars) sized by the caller for `sh`.
cudaError_t launch_pass_at(PassParams P, int pmode, int acc, const LaunchShape &sh, double *part,
                           unsigned *tickets, double *blk, cudaStream_t st);

int pmode_of(double p);   // P_L1 / P_SQ / P_INF / P_GEN

// Whether pair passes launch with programmatic stream serialisation (PDL):
// on unless CULAMP_NO_PDL is set in the environment (read once) or a PdlOff
// guard is alive on this thread.
bool pdl_launches();
struct PdlOff {
    PdlOff();
    ~PdlOff();
    PdlOff(const PdlOff &) = delete;
    PdlOff &operator=(const PdlOff &) = delete;
};

// ---- W_inf = max_ij C(x_i, y_j) (maxcost.cu): exact FP64, register-tiled.
// `dst` must hold +0.0 before the launch (the kernel folds in with atomicMax).
cudaError_t launch_max_cost(const double *X, const double *Y, int n, int m, int d, double p,
                            double *dst, int sm_count, cudaStream_t st);
struct MaxCostInput {
    const double *X, *Y;
    int n, m, d;
    double *dst;
};
// Device table bytes for `count` jobs; one launch over all of them. host_table
// keeps the uploaded table alive until the copy has been consumed.
size_t max_cost_table_bytes(int count);
cudaError_t launch_max_cost_batched(const MaxCostInput *in, int count, double p, void *table,
                                    std::vector<unsigned char> &host_table, int sm_count,
                                    cudaStream_t st);

// ---- feature-cost path (feature.cu): p = 2, d >= FEAT_MIN_D, tensor cores
constexpr int FEAT_MIN_D = 32;

struct FeatShape {
    int rtiles, ctiles;   // 128-row tiles of the output rows, ncols-column tiles
    int rblk, cblk;       // 128-point blocks of the packed row / column clouds (piece strides)
    int ncols;            // columns per tile (MMA N)
    int splits, tps;      // column slices, column tiles per slice
    int units, grid;      // work units (row tile x slice), CTAs (<= SMs)
    int merge_rb;         // CTAs of the merge / epilogue kernel
    size_t part_bytes;    // partials: splits * n * 3 doubles
};

FeatShape feat_shape(int n, int m, int sm_count, int pieces);
int feat_blocks(int n);                 // 128-point blocks of a packed cloud (even)
int feat_tile_cols(int pieces);         // columns per tile for BF16x3 (2) / BF16x6 (3)
int feat_kblocks(int d);
size_t feat_piece_elems(int n, int d, int pieces);   // bf16 elements of one packed cloud
// Pack one cloud (n x d, FP64) into `pieces` bf16 pieces and its squared norms.
cudaError_t feat_prepare(uint16_t *pieces, double *norms, const double *X, int n, int d, int np,
                         cudaStream_t st);
// Reduction on the tensor cores + merge / epilogue; P.fx .. P.fpieces set.
cudaError_t launch_feat_pass(PassParams P, int acc, Scratch &scr, int sm_count, cudaStream_t st);
// Work-unit geometry of a feature pass (splits, tiles, merge row blocks) into P.
void set_feat_geometry(PassParams &P, const FeatShape &fs);
// One batched feature pass over `count` instances (device parameter list,
// unit and merge-block prefix tables with count + 1 entries).
cudaError_t launch_feat_batched(int np, int acc, bool mom, const PassParams *plist, const int *unit_start,
                                const int *block_start, int count, int total_units, int merge_blocks,
                                int sm_count, int *batch_err, cudaStream_t st);
// One batched pair pass (pair_pass_kernel<..., BAT = true>) over `count`
// instances of dimension d (d <= 3 packed, else generic), RPT rows per thread.
cudaError_t launch_pass_batched(const PassParams *plist, const int *block_start, int count,
                                int total_blocks, size_t smem, int pmode, int d, int acc, bool mom,
                                bool fixed_ref, cudaStream_t st);

// ---- whole Sinkhorn loop in one persistent cooperative launch (persist.cu):
// small problems (p = 1, 2 or Inf with the same cost in the check, d <= 3).
constexpr int PERSIST_MAX_POINTS = 8192;   // per side: <= 16 FP32 terms per thread partial
int persist_grid(int sm_count, int d, int pm);          // CTAs (0: not launchable)
bool persist_eligible(int n, int m, int d, int pm_iter, int pm_resid, int grid);
size_t persist_scratch_bytes(int grid);
// The loop from the control block's state to its stop; `scratch` holds
// persist_scratch_bytes(grid) bytes. Completes the control block like the
// pass-per-launch loop (iteration counters, stop reason, residual, log).
cudaError_t launch_sk_persist(const double *X, const double *Y, const double *r, const double *c,
                              double *phi, double *psi, int n, int m, int d, int pm, double pexp,
                              Ctl *ctl, void *scratch, int grid, cudaStream_t st);

// LAMP's loop (MirrorProxKernel.jl:1019-1132) in one persistent launch, same
// problem sizes, eta_p > 0. Completes the control block like the graph loop.
struct LampPersistArgs {
    const double *X, *Y, *r, *c;
    double *nu, *nub, *theta, *thetab;
    const double *eta_mu;
    double *logz, *aux;
    int n, m, d, pm;
    double pexp, eta_mu_exp, minv, maxv;
    Ctl *ctl;
    void *scratch;             // lamp_persist_scratch_bytes(grid)
};
int lamp_persist_grid(int sm_count, int d, int pm);
size_t lamp_persist_scratch_bytes(int grid);
cudaError_t launch_lamp_persist(const LampPersistArgs &a, int grid, cudaStream_t st);

}  // namespace culamp_host

// The opaque handle.
struct culamp_handle_s {
    int device = 0;
    int sm_count = 148;
    std::string err;
    culamp_host::Scratch scratch;      // pass-level scratch
    culamp_host::DevBuf pass_ctl;      // Ctl for pass-level / post-loop calls
    culamp_host::DevBuf tmpA, tmpB;    // pass-level temporaries
    struct Solver;                     // solver workspaces and cached graphs
    Solver *solver = nullptr;
    struct Batch;                      // batched-solve workspace, tuned shapes, graph
    Batch *batch = nullptr;
    struct Dense;                      // dense-cost solver workspace (W^T, check rows)
    Dense *dense = nullptr;
};

int culamp_set_error(culamp_handle h, int code, const char *fmt, ...);
