// olc_stage_sort_pairs_noalloc: the stable radix sort of olc_stage_sort_pairs
// for callers that cannot allocate device memory.
//
// Who needs it: a host process whose device memory is owned by an allocator it
// does not expose (for example a serving process that reserved the free HBM up
// front and hands out only tensors), or a caller on a latency-critical path
// where cudaMalloc's implicit device-wide synchronisation would stall work on
// other streams.  Such callers still own their keys and values; what they
// cannot provide is the sort's temporary memory.  This entry point takes that
// temporary memory from a file-scope device array instead.
//
// Limits and sharing:
//   * at most kNoAllocMaxKeys (1,048,576) keys per call; larger inputs are
//     rejected with OLC_ERR_CAPACITY;
//   * the array (about 9.4 MB) is part of libolc.so's device image: every GPU
//     that loads the library holds it until the process exits;
//   * every call shares the one array, which keeps the previous call's
//     contents; the sort clears what must start at zero (histograms, look-back
//     words, status word) on the call's stream before using it.  Calls whose
//     work overlaps on the GPU (other streams, other host threads) race on the
//     array and must be serialised by the caller;
//   * every call outside stream capture looks up the array's device address
//     (cudaGetSymbolAddress) with the caller's device current, so a device
//     reset between calls is followed; a call on a capturing stream uses the
//     address the last uncaptured call on that device found, so make one
//     call on a device before capturing any;
//   * the sort's bounded look-back waits report a timeout in the array's
//     status word, which olc_sort_noalloc_status reads back: a set
//     OLC_STATUS_TIMEOUT bit means that call's output is unreliable.
// No cudaMalloc, cudaFree or allocating library routine is called here.
#include "olc_internal.h"

#include <mutex>

namespace {

constexpr olc_u32 kNoAllocMaxKeys = 1u << 20;
constexpr int kMaxDevices = 64;

constexpr size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

// The layout carve_sort_scratch builds for kNoAllocMaxKeys keys and 32-bit keys
// (4 passes): histograms, scanned bases, tile counters, status word, look-back
// words, alternate keys and values.
constexpr size_t kNoAllocBytes =
    al256(olc::MAX_PASSES * olc::RADIX * 4) * 2 + al256(olc::MAX_PASSES * 4) + al256(4) +
    al256((size_t)olc::MAX_PASSES * ((kNoAllocMaxKeys + olc::SORT_TILE - 1) / olc::SORT_TILE) * olc::RADIX * 4) +
    2 * al256((size_t)kNoAllocMaxKeys * 4);

}  // namespace

// File-scope device scratch of the allocation-free sort.
static __device__ __align__(256) unsigned char g_noalloc_sort_scratch[kNoAllocBytes];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kMaxDevices] = {};

// The array's device address on device `dev` (current): looked up afresh
// unless `st` is capturing, when the address the last uncaptured call found
// is used (a capture records the address into its graph).
int noalloc_base(int dev, cudaStream_t st, void** out) {
    using namespace olc;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        cs = cudaStreamCaptureStatusActive;  // unknown: do not call into the runtime's symbol table
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_sort_scratch);
        if (e != cudaSuccess) return cuda_status(e, "olc_stage_sort_pairs_noalloc: cudaGetSymbolAddress");
        g_noalloc_addr[dev] = p;
    } else if (!g_noalloc_addr[dev]) {
        set_error("olc_stage_sort_pairs_noalloc: first call on this device is inside a stream capture; "
                  "make one call outside capture first");
        return OLC_ERR_STATE;
    }
    *out = g_noalloc_addr[dev];
    return OLC_OK;
}
}  // namespace

extern "C" int olc_stage_sort_pairs_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                            uint32_t* vals_out, uint32_t n, int key_bits, void* stream) {
    using namespace olc;
    if (key_bits < 1 || key_bits > 32) {
        set_error("olc_stage_sort_pairs_noalloc: key_bits must be in [1, 32]");
        return OLC_ERR_ARG;
    }
    if (n > kNoAllocMaxKeys) {
        set_error("olc_stage_sort_pairs_noalloc: " + std::to_string(n) + " keys exceed the static scratch limit of " +
                  std::to_string(kNoAllocMaxKeys) + " keys; use olc_stage_sort_pairs with caller scratch");
        return OLC_ERR_CAPACITY;
    }
    if (n == 0) return OLC_OK;
    if (!keys_in || !keys_out || !vals_out) {
        set_error("olc_stage_sort_pairs_noalloc: null buffer");
        return OLC_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "olc_stage_sort_pairs_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("olc_stage_sort_pairs_noalloc: device index out of range");
        return OLC_ERR_ARG;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void* base = nullptr;
    const int rc = noalloc_base(dev, st, &base);
    if (rc != OLC_OK) return rc;
    SortScratch sc;
    if (!carve_sort_scratch(base, kNoAllocBytes, n, key_bits, &sc)) {
        set_error("olc_stage_sort_pairs_noalloc: static scratch layout does not fit");
        return OLC_ERR_STATE;
    }
    e = cudaMemsetAsync(sc.status, 0, 4, st);
    if (e != cudaSuccess) return cuda_status(e, "olc_stage_sort_pairs_noalloc: clear status");
    // run_sort clears the histograms and look-back words before the passes
    run_sort(keys_in, vals_in, keys_out, vals_out, nullptr, n, n, key_bits, sc, false, nullptr, 0, st);
    return cuda_status(cudaGetLastError(), "olc_stage_sort_pairs_noalloc");
}

extern "C" int olc_sort_noalloc_status(uint32_t* status_out, void* stream) {
    using namespace olc;
    if (!status_out) {
        set_error("olc_sort_noalloc_status: null status_out");
        return OLC_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e, "olc_sort_noalloc_status: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("olc_sort_noalloc_status: device index out of range");
        return OLC_ERR_ARG;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    void* base = nullptr;
    const int rc = noalloc_base(dev, st, &base);
    if (rc != OLC_OK) return rc;
    SortScratch sc;
    if (!carve_sort_scratch(base, kNoAllocBytes, 1, 32, &sc)) {
        set_error("olc_sort_noalloc_status: static scratch layout does not fit");
        return OLC_ERR_STATE;
    }
    olc_u32 w = 0;
    e = cudaMemcpyAsync(&w, sc.status, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "olc_sort_noalloc_status: read status");
    // the sort's status bits are the device's OLC_ST_* values (OLC_STATUS_* in olc.h)
    *status_out = w;
    return OLC_OK;
}
