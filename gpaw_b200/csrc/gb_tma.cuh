// Plane tiles through the Tensor Memory Accelerator (TMA) for 16-byte
// (complex128) grids.
//
// A batch of C-contiguous grids (nb, n0, n1, n2) of 16-byte elements is
// described to the TMA as a 4-D tensor of 8-byte words (2 n2, n1, n0, nb):
// every stride is a multiple of 16 bytes for any grid size, which is what
// tensor copies require.  One elected thread copies a whole (rows x cols)
// window of one plane into shared memory with a single instruction; parts of
// the window outside the tensor (a negative or too-large row, column or
// plane) arrive as zeros, which is the zero boundary.  Periodic wrap-around
// and Bloch phases are applied afterwards by the kernels (the TMA has no
// periodic mode).  Completion is signalled on an mbarrier that the copy
// charges with its byte count.
//
// Every wait here is bounded by wall-clock time (%globaltimer): a wait that
// runs out records GB_FAULT_TMA_TIMEOUT in a device flag that the host reads
// with gb_device_fault(), and the kernel finishes without the data instead of
// hanging.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace gb {

// Device-side fault flag (0 = none; the first fault wins).  Each
// translation unit that includes this header has its own copy (no
// relocatable device code); take_unit_fault() reads and clears it and the
// units' readers are combined by gb_device_fault().
static __device__ int g_device_fault;
constexpr int GB_FAULT_TMA_TIMEOUT = 1;

static inline int take_unit_fault(int* code) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_device_fault, sizeof v) != cudaSuccess) return -1;
    if (v) {
        const int zero = 0;
        if (cudaMemcpyToSymbol(g_device_fault, &zero, sizeof zero) != cudaSuccess) return -1;
    }
    *code = v;
    return 0;
}

// ----------------------------------------------------------------- host
// Encode the tensor map of a batch of grids of 16-byte elements with a
// (box_rows x box_cols) window box.  Returns 0, or -1 when the driver
// refuses (message in *why).
int make_plane_map16(CUtensorMap* map, const void* base, long long nb, int n0, int n1, int n2,
                     int box_rows, int box_cols, const char** why);

// ---------------------------------------------------------------- device
__device__ __forceinline__ unsigned tma_smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(tma_smem_u32(bar)),
                 "r"(count));
}

// make barrier initialisation visible to the async proxy (before the first
// copy that signals it)
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(
                     tma_smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// One potentially blocking test of the phase: the hardware may suspend the
// warp for up to about a microsecond (the hint, in ns) until it completes.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(tma_smem_u32(bar)), "r"(parity), "r"(1000u)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar` to complete, at most `limit_ns`
// nanoseconds; false (and the device fault flag set) when it did not.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          uint64_t limit_ns = 1000000000ull) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (unsigned it = 1;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0 && global_ns() - t0 > limit_ns) {
            atomicCAS(&g_device_fault, 0, GB_FAULT_TMA_TIMEOUT);
            return false;
        }
    }
}

// Copy the window of plane `plane` of grid `b` whose first row is `row` and
// first column `col` (in elements; any of them may lie outside the grid)
// into `dst`; completion charges `bar` with the window's bytes.
__device__ __forceinline__ void tma_load_window16(void* dst, const CUtensorMap* map, int col,
                                                  int row, int plane, int b, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(tma_smem_u32(dst)),
        "l"((uint64_t)map), "r"(2 * col), "r"(row), "r"(plane), "r"(b),
        "r"(tma_smem_u32(bar))
        : "memory");
}

}  // namespace gb
