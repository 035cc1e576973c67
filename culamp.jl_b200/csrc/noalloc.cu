// noalloc.cu -- culamp_lse_rows_sk_noalloc: the Sinkhorn row pass
// (warp_logsumexp_ct_fused!) with no device allocation at all.
//
// Who needs it. Some callers cannot let a library allocate device memory when
// they call it: hosts that own every byte of device memory through their own
// pool or a fixed budget (serving runtimes, engines that embed the solver next
// to a model) and forbid third-party cudaMalloc / cudaFree, because an
// allocation they did not plan for can fail or fragment their pool mid-run.
// The handle-based culamp_lse_rows_sk grows its scratch with cudaMalloc on
// demand, so it cannot serve them; this entry point takes no handle and uses
// only the fixed scratch below.
//
// Scratch: two file-scope __device__ arrays, resident on every GPU that loads
// this library until the process exits --
//   * g_noalloc_part: NOALLOC_PART_ENTRIES (split, row) partial results of three
//     doubles each (3 MiB); when n * splits would exceed it the pass uses fewer
//     column splits (a single split needs no partials at all);
//   * g_noalloc_tickets: NOALLOC_TICKETS row-block tickets (256 KiB). A row
//     block holds at least 128 rows (one per thread), so n is limited to
//     NOALLOC_MAX_ROWS = (NOALLOC_TICKETS - 1) * 128 = 8,388,608 rows for every
//     d; larger n is rejected with CULAMP_ERR_UNSUPPORTED before any launch.
// Every call shares these arrays and they keep the last call's contents: each
// call clears the tickets it uses (cudaMemsetAsync, no allocation) before its
// launch, and the partials are always written before they are read. Calls
// that overlap on the GPU (concurrent streams, or several host threads) race
// on the shared arrays and give wrong results: serialise them.
//
// Set-up: the first call on a device (with that device current) resolves the
// arrays' device addresses with cudaGetSymbolAddress; a host-side name of a
// __device__ array is only a stand-in and must never be passed to a kernel.
// That first call may load the module, so make it before any stream capture.
// A set-up that fails (CULAMP_ERR_CUDA) is not remembered: the next call on
// that device tries again.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace {

constexpr int NOALLOC_PART_ENTRIES = 1 << 17;
constexpr int NOALLOC_TICKETS = (1 << 16) + 1;
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr int64_t NOALLOC_MAX_ROWS = (int64_t)(NOALLOC_TICKETS - 1) * culamp_dev::TPB;

__device__ __align__(256) double g_noalloc_part[3 * NOALLOC_PART_ENTRIES];
__device__ __align__(256) unsigned int g_noalloc_tickets[NOALLOC_TICKETS];

struct NoallocDevice {
    bool ready = false;          // addresses resolved (set only on success)
    double *part = nullptr;
    unsigned int *tickets = nullptr;
    int sm_count = 0;
};
NoallocDevice g_devices[NOALLOC_MAX_DEVICES];
std::mutex g_setup_mutex;

// Resolves the device addresses of the fixed arrays for `dev` (current). On
// failure nothing is recorded, so a later call retries the set-up.
cudaError_t noalloc_setup(int dev, NoallocDevice **out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    NoallocDevice &d = g_devices[dev];
    if (!d.ready) {
        double *part = nullptr;
        unsigned int *tickets = nullptr;
        int sms = 0;
        cudaError_t e = cudaGetSymbolAddress((void **)&part, g_noalloc_part);
        if (e == cudaSuccess) e = cudaGetSymbolAddress((void **)&tickets, g_noalloc_tickets);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) {
            cudaGetLastError();   // clear it: the next call starts clean and retries
            return e;
        }
        d.part = part;
        d.tickets = tickets;
        d.sm_count = sms;
        d.ready = true;
    }
    *out = &d;
    return cudaSuccess;
}

}  // namespace

using namespace culamp_host;
using namespace culamp_dev;

extern "C" int culamp_lse_rows_sk_noalloc(double *out, const double *x, const double *y,
                                          int64_t n, int64_t m, int32_t d, const double *marg,
                                          const double *pot, double reg, double winf, double p,
                                          void *stream) {
    if (!out || !x || !y || !marg || !pot) return CULAMP_ERR_INVALID_ARG;
    if (n < 1 || m < 1 || n > (int64_t)INT32_MAX / 4 || m > (int64_t)INT32_MAX / 4)
        return CULAMP_ERR_INVALID_ARG;
    if (d < 1) return CULAMP_ERR_INVALID_ARG;
    if (d > MAXD) return CULAMP_ERR_UNSUPPORTED;
    if (!(p > 0.0)) return CULAMP_ERR_INVALID_ARG;
    if (n > NOALLOC_MAX_ROWS) return CULAMP_ERR_UNSUPPORTED;   // more row blocks than tickets
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CULAMP_ERR_CUDA;
    NoallocDevice *nd = nullptr;
    if (noalloc_setup(dev, &nd) != cudaSuccess) return CULAMP_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;

    LaunchShape sh = pass_shape((int)n, (int)m, d, ACC_LSE, nd->sm_count, false);
    if ((int64_t)sh.rb + 1 > NOALLOC_TICKETS) return CULAMP_ERR_UNSUPPORTED;
    if ((int64_t)sh.splits * n > NOALLOC_PART_ENTRIES) {
        // fewer column splits so every (split, row) partial fits the fixed array
        int splits = (int)(NOALLOC_PART_ENTRIES / n);
        if (splits < 1) splits = 1;
        const int ch = (d <= MAXD_PACKED) ? CHUNK : CHUNK_G;
        int cps = (int)((m + splits - 1) / splits);
        cps = ((cps + ch - 1) / ch) * ch;
        sh.splits = (int)((m + cps - 1) / cps);
        sh.cols_per_split = cps;
        sh.part_bytes = sh.splits > 1 ? (size_t)sh.splits * (size_t)n * 3 * sizeof(double) : 0;
    }
    if (cudaMemsetAsync(nd->tickets, 0, (size_t)(sh.rb + 1) * sizeof(unsigned int), st) != cudaSuccess)
        return CULAMP_ERR_CUDA;

    // Non-owning views of the fixed arrays. This pass has no finish step, so
    // the block-partial buffer is never touched; it aliases the partials.
    Scratch scr;
    scr.part.ptr = nd->part;
    scr.part.bytes = sizeof(double) * 3 * (size_t)NOALLOC_PART_ENTRIES;
    scr.tickets.ptr = nd->tickets;
    scr.tickets.bytes = sizeof(unsigned int) * (size_t)NOALLOC_TICKETS;
    scr.blk = scr.part;

    PassParams P;
    memset(&P, 0, sizeof(P));
    P.X = x;
    P.Y = y;
    P.n = (int)n;
    P.m = (int)m;
    P.d = d;
    P.pexp = p;
    P.ctr = x;
    P.epi = EPI_SK_ROW;
    P.coef_mode = COEF_FIXED;
    P.alpha = -1.0 / (reg * winf);
    P.beta = 1.0;
    P.colpot = pot;
    P.marg = marg;
    P.out = out;
    P.use_ref = 1;   // out's incoming value is a hint only: any value gives the same result
    P.finish = FIN_NONE;
    const cudaError_t e = launch_pass(P, pmode_of(p), ACC_LSE, sh, scr, st);
    return e == cudaSuccess ? CULAMP_OK : CULAMP_ERR_CUDA;
}
