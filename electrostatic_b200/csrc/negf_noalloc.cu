// Allocation-free induced-charge entry point.
//
// Some callers cannot allocate device memory at the point where they need
// the charge: applications whose device memory is handed out by their own
// pool and that forbid the runtime allocator, or drop-in plugins that must not
// grow the footprint of the host program between its own allocations.  For
// them, negf_compute_charge_noalloc() runs the same RGF kernels as
// negf_compute_charge(), but every buffer of a call -- the launch tables,
// the per-warp partial rows and the segment checkpoints -- lives in one
// file-scope device array of kScratchBytes (32 MiB).  Every GPU that loads
// this library holds that array until the process exits.
//
// Rules of use (also stated in include/negf_b200.h):
//   * the charge output is a device pointer supplied by the caller;
//   * problems whose tables and scratch exceed the array are rejected with
//     NEGF_ERR_ARG and a message giving the bytes needed;
//   * every tube of a call must live on the current device (NEGF_ERR_ARG);
//   * the first call on a device looks up the array's device address (a
//     set-up step); make that first call before any stream capture;
//   * all calls share the array, so calls whose work overlaps on the GPU
//     (different streams, or different host threads) race; serialise them;
//   * nothing in the array needs to start at zero: every word a call reads
//     is written earlier in the same call.

#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/negf_b200.h"
#include "negf_internal.h"

namespace negf {
namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};  // device address of g_scratch, per device ordinal

// Host staging of the launch tables (fixed capacity, no allocation).
constexpr int kTubeCap = 64;
constexpr size_t kChainCap = 1 << 15;
constexpr size_t kWarpCap = kChainCap / kWarp;
constexpr size_t kUnitCap = 1 << 15;
TubeDev h_tubes[kTubeCap];
ReduceTube h_rts[kTubeCap];
ChainRec h_chains[kChainCap];
WarpRec h_warps[kWarpCap];
SegUnit h_units[kUnitCap];

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// Set-up, once per device with that device current: the host-side name
// g_scratch is not a device address; the runtime gives the real one.
int scratch_address(unsigned char** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return report(NEGF_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return report(NEGF_ERR_CUDA, "device ordinal out of range");
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            std::snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the scratch array failed: %s",
                          cudaGetErrorString(e));
            return report(NEGF_ERR_CUDA, msg);
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return NEGF_OK;
}

}  // namespace
}  // namespace negf

extern "C" int negf_compute_charge_noalloc(negf_tube* const* tubes, int num_tubes, double* d_Q, void* stream) {
    using namespace negf;
    if (!d_Q) return report(NEGF_ERR_ARG, "null charge output (a device pointer is required)");
    // the host tables below are shared: planning and their upload run under
    // the host layer's lock (a pageable-memory copy has consumed its source
    // when cudaMemcpyAsync returns)
    std::unique_lock<std::mutex> lk = api_lock();
    FixedPlan fp{};
    fp.tubes = h_tubes;
    fp.rts = h_rts;
    fp.chains = h_chains;
    fp.warps = h_warps;
    fp.units = h_units;
    fp.tube_cap = kTubeCap;
    fp.chain_cap = kChainCap;
    fp.warp_cap = kWarpCap;
    fp.unit_cap = kUnitCap;
    int rc = plan_charge_fixed(tubes, num_tubes, fp);
    if (rc != NEGF_OK) return rc;

    // carve the scratch array: tables, partial rows, checkpoints
    const size_t o_tubes = 0;
    const size_t o_rts = o_tubes + align256(sizeof(TubeDev) * fp.num_tubes);
    const size_t o_warps = o_rts + align256(sizeof(ReduceTube) * fp.num_tubes);
    const size_t o_units = o_warps + align256(sizeof(WarpRec) * fp.num_warps);
    const size_t o_chains = o_units + align256(sizeof(SegUnit) * fp.num_units);
    const size_t o_partial = o_chains + align256(sizeof(ChainRec) * fp.num_chains);
    const size_t o_ck = o_partial + align256(sizeof(double) * fp.partial_doubles);
    const size_t need = o_ck + align256(sizeof(double) * fp.scratch_doubles);
    if (need > kScratchBytes) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "problem needs %zu bytes of device scratch; the allocation-free entry point holds %zu "
                      "(use negf_compute_charge)",
                      need, kScratchBytes);
        return report(NEGF_ERR_ARG, msg);
    }
    unsigned char* base = nullptr;
    rc = scratch_address(&base);
    if (rc != NEGF_OK) return rc;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaSuccess;
    auto up = [&](size_t off, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, s);
    };
    up(o_tubes, h_tubes, sizeof(TubeDev) * fp.num_tubes);
    up(o_rts, h_rts, sizeof(ReduceTube) * fp.num_tubes);
    up(o_warps, h_warps, sizeof(WarpRec) * fp.num_warps);
    up(o_units, h_units, sizeof(SegUnit) * fp.num_units);
    up(o_chains, h_chains, sizeof(ChainRec) * fp.num_chains);
    if (e != cudaSuccess) return report(NEGF_ERR_CUDA, cudaGetErrorString(e));
    e = launch_rgf(reinterpret_cast<const TubeDev*>(base + o_tubes), reinterpret_cast<const ChainRec*>(base + o_chains),
                   reinterpret_cast<const WarpRec*>(base + o_warps), (int)fp.num_warps,
                   reinterpret_cast<const SegUnit*>(base + o_units), (int)fp.num_units,
                   reinterpret_cast<double*>(base + o_partial), base + o_ck, 4, s, nullptr);
    if (e != cudaSuccess) return report(NEGF_ERR_CUDA, cudaGetErrorString(e));
    e = launch_reduce(reinterpret_cast<const ReduceTube*>(base + o_rts), fp.num_tubes, fp.max_N,
                      reinterpret_cast<const double*>(base + o_partial), d_Q, s);
    if (e != cudaSuccess) return report(NEGF_ERR_CUDA, cudaGetErrorString(e));
    return NEGF_OK;
}
