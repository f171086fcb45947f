// wcb_rows_select_noalloc: the path-record selection of wcb_rows_select with
// its scratch in a fixed array that lives in this library's device image, so
// the call itself allocates nothing.
//
// Who needs it: callers that may not allocate device memory at call time --
// code running inside a caching allocator's out-of-memory handler, real-time
// loops that forbid allocator calls (cudaMalloc synchronises the device and
// can stall for milliseconds), and hosts whose memory pools are sized once at
// start-up and then frozen.  They hand over the records and the output index
// buffer; everything else the sort, dedup and max_paths stages need comes
// from g_select_scratch below.
//
// Set-up: every call looks up the array's device address on the current
// device with cudaGetSymbolAddress (nothing is cached, so a cudaDeviceReset
// or a different context on the device never leaves a stale address behind).
// The first lookup on a device may make the CUDA runtime load this library's
// module there, so make the first call on a device before any stream capture
// begins; later lookups are a table read.
//
// Synchronisation: like wcb_rows_select, the call reads its counts back to
// the host and synchronises `stream` before it returns, so it blocks the
// calling thread for the duration of the selection.
//
// Sharing: every call on a device uses the same array and leaves its last
// contents there.  Each stage writes the scratch words it later reads (the
// buffers that must start at zero, the key-width maxima and the per-pair keep
// flags, are cleared by the call itself), so no state leaks from one call
// into the next; but two
// calls that overlap in time -- on two streams, or from two host threads --
// race on the array and corrupt each other's results.  Serialise them.
#include <cuda_runtime.h>

#include "../../include/witwin_channel_b200.h"
#include "internal.h"

namespace wcb {
namespace {

constexpr long long kScratchBytes = WCB_ROWS_SELECT_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_select_scratch[kScratchBytes];

// Device address of g_select_scratch in the current device's context.  In
// host code the array's name is only a host-side handle; the kernels get this
// address.
int scratch_address(void** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_select_scratch) != cudaSuccess || p == nullptr) return WCB_ERR_CUDA;
    *out = p;
    return WCB_OK;
}

}  // namespace
}  // namespace wcb

extern "C" int wcb_rows_select_noalloc(const void* rows, int64_t num_rows, int32_t width, int64_t max_paths,
                                       int32_t scope, int64_t* selected, int64_t* num_selected, void* stream) {
    if (num_selected == nullptr || num_rows < 0 || (num_rows > 0 && (rows == nullptr || selected == nullptr)))
        return WCB_ERR_INVALID_ARGUMENT;
    if (width < 0 || width > 5 || (scope != 0 && scope != 1)) return WCB_ERR_INVALID_ARGUMENT;
    *num_selected = 0;
    int64_t need = 0;
    if (wcb::rows_select_workspace(num_rows, &need) != 0) return WCB_ERR_INVALID_ARGUMENT;
    if (need > wcb::kScratchBytes) return WCB_ERR_CAPACITY;
    void* scratch = nullptr;
    const int rc = wcb::scratch_address(&scratch);
    if (rc != WCB_OK) return rc;
    return wcb::rows_select(rows, num_rows, width, max_paths, scope, selected, num_selected, scratch,
                            wcb::kScratchBytes, static_cast<cudaStream_t>(stream));
}
