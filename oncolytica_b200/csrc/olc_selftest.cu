// olc_selftest_bounded_waits: makes the library's two kinds of bounded
// device wait run out, so that a test can check that each returns and
// records OLC_ST_TIMEOUT instead of hanging.
//
//   * look-back: one block publishes tile 1 of a decoupled look-back
//     (olc_lookback, the sort's and the births' prefix walk) whose tile-0
//     word nobody ever publishes;
//   * TMA tile: one block arms an mbarrier for a 64-byte transaction that is
//     never issued and waits on it with olc_mbar_wait_bounded (the wait of
//     every TMA stencil kernel).
//
// Both use the production device functions with a caller-given poll limit
// (the kernels use OLC_SPIN_LIMIT).  No memory is accessed out of bounds and
// no copy is left in flight: the armed barrier has no transaction behind it.
// The words live in a small file-scope device array, so the entry point
// allocates nothing.  No counterpart in the reference (whose waits are not
// bounded: it has none).
#include "olc_internal.h"

namespace {

// [0, 4): look-back words of tiles 0..3 (tile 0 stays unpublished)
// [4]: look-back status, [5]: mbarrier status, [6]: prefix the walk returned
__device__ __align__(16) olc_u32 g_selftest_words[8];

__global__ void k_selftest_lookback(olc_u32* words, olc_u32* status, olc_u32* prefix_out, olc_u32 limit) {
    if (threadIdx.x == 0) *prefix_out = olc_lookback(words, 1, 1, 5u, status, limit);
}

__global__ void k_selftest_mbar(olc_u32* status, olc_u32 limit) {
    __shared__ alignas(8) unsigned long long bar;
    const olc_u32 bar_a = static_cast<olc_u32>(__cvta_generic_to_shared(&bar));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        // the single arrival, with 64 bytes of transaction that never come
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(64u) : "memory");
    }
    __syncthreads();
    if (olc_mbar_wait_bounded(bar_a, 0, status, limit)) {
        // unreachable: the phase cannot complete; record it as a distinct bit
        atomicOr(status, 0x80000000u);
    }
}

}  // namespace

extern "C" int olc_selftest_bounded_waits(uint32_t limit, uint32_t out[3], void* stream) {
    using namespace olc;
    if (!out || limit == 0 || limit > 65536u) {
        set_error("olc_selftest_bounded_waits: out must be non-null and limit in [1, 65536]");
        return OLC_ERR_ARG;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    olc_u32* w = nullptr;
    cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&w), g_selftest_words);
    if (e != cudaSuccess) return cuda_status(e, "olc_selftest_bounded_waits: cudaGetSymbolAddress");
    e = cudaMemsetAsync(w, 0, sizeof(olc_u32) * 8, st);
    if (e != cudaSuccess) return cuda_status(e, "olc_selftest_bounded_waits: clear");
    k_selftest_lookback<<<1, 32, 0, st>>>(w, w + 4, w + 6, limit);
    k_selftest_mbar<<<1, 64, 0, st>>>(w + 5, limit);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "olc_selftest_bounded_waits: launch");
    olc_u32 h[8];
    e = cudaMemcpyAsync(h, w, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e, "olc_selftest_bounded_waits: read");
    out[0] = h[4];  // look-back status (OLC_STATUS_TIMEOUT expected)
    out[1] = h[5];  // mbarrier status (OLC_STATUS_TIMEOUT expected)
    out[2] = h[6];  // the walk's prefix: 0 (the unpublished tile counts as an empty prefix)
    return OLC_OK;
}
