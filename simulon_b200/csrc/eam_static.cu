// sim_eam_forces_static: the two-pass EAM force call with its scratch held in
// a fixed array inside this library instead of caller-allocated buffers.
//
// Who needs it: a host code that hands out all of its device memory up front
// from its own pool, or that binds this library over a plain C FFI with no
// device allocator at hand, cannot allocate the per-atom records and reduction
// partials that sim_eam_forces reads from SimEngine.  This entry point takes
// them from `g_eam_scratch` below and allocates nothing itself: no cudaMalloc,
// no cudaFree, no library routine that allocates.
//
// What lives in the array (one 256-byte aligned block, 4,456,704 bytes):
//   [0, 256)            last-block counters of the two passes (uint32)
//   [256, 262400)       per-block FP64 reduction partials, up to 2048 blocks
//   [262400, end)       the 16-byte {x, y, z, F'(rho)} record per atom slot
//                       written by the density pass and gathered by the force
//                       pass, up to SIM_STATIC_MAX_ATOMS slots
// The counters must be zero when a pass starts; every call clears them with
// cudaMemsetAsync on the caller's stream.  The partials and records are written
// before they are read within the call, so nothing else needs clearing.
//
// The device address of the array is looked up on every call, with the
// caller's device current, by cudaGetSymbolAddress (a host-side lookup with no
// stream work), so a device reset or a re-created primary context that moves
// the array is followed.  The first call on a device also loads the array's
// module there: make that first call before any stream capture.  The array is
// one per device and shared by every call: two calls that may overlap in time
// (different streams or host threads on one device) race on it, and the caller
// must serialise them.
//
// The in-cutoff mask (e->cut_mask) is per-atom scratch as well, so it is not
// used here: the density pass writes no mask and the force pass tests every
// list entry against the cutoff itself, which visits the same pairs in the
// same order and gives the same results.
#include <cstdio>
#include "common.cuh"

namespace simb200 {

static constexpr size_t kCounterBytes = 256;
static constexpr int kStaticMaxBlocks = 2048;
static constexpr size_t kPartialBytes = (size_t)kStaticMaxBlocks * SIM_RED_SLOTS * sizeof(double);
static constexpr size_t kRecordOffset = kCounterBytes + kPartialBytes;
static constexpr size_t kScratchBytes = kRecordOffset + (size_t)SIM_STATIC_MAX_ATOMS * 16;
static_assert(kRecordOffset % 256 == 0, "per-atom records must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_eam_scratch[kScratchBytes];

// Device address of g_eam_scratch on the current device.
static int scratch_on_current_device(void** out) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_eam_scratch);
    if (err != cudaSuccess || !p) {
        set_cuda_error(err, "sim_eam_forces_static: cudaGetSymbolAddress of the scratch array");
        return SIM_ERR_CUDA;
    }
    *out = p;
    return SIM_OK;
}

}  // namespace simb200

using namespace simb200;

extern "C" int sim_eam_forces_static(const SimEngine* ep, const SimEAMTables* tp, void* stream) {
    if (!ep || !tp || ep->n <= 0) return SIM_ERR_ARG;
    if (ep->n_pad > SIM_STATIC_MAX_ATOMS || ep->n > ep->n_pad) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "sim_eam_forces_static: %lld atom slots exceed the static scratch limit of %d "
                 "(SIM_STATIC_MAX_ATOMS); use sim_eam_forces with caller-allocated buffers",
                 (long long)ep->n_pad, SIM_STATIC_MAX_ATOMS);
        set_error_text(msg);
        return SIM_ERR_ARG;
    }
    void* base = nullptr;
    int rc = scratch_on_current_device(&base);
    if (rc != SIM_OK) return rc;
    unsigned char* b = static_cast<unsigned char*>(base);
    SimEngine e = *ep;
    e.red_counter = reinterpret_cast<uint32_t*>(b);
    e.partials = reinterpret_cast<double*>(b + kCounterBytes);
    e.posfp = reinterpret_cast<int32_t*>(b + kRecordOffset);
    e.cut_mask = nullptr;
    e.n_blocks_max = kStaticMaxBlocks;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t err = cudaMemsetAsync(e.red_counter, 0, kCounterBytes, st);
    if (err != cudaSuccess) {
        set_cuda_error(err, "sim_eam_forces_static: clearing the counters");
        return SIM_ERR_CUDA;
    }
    rc = sim_eam_density(&e, tp, stream);
    if (rc != SIM_OK) return rc;
    return sim_eam_force(&e, tp, stream);
}
