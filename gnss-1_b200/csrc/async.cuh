// async.cuh -- bulk asynchronous copies (global -> shared) completed on an
// mbarrier, with bounded waits.
//
// Only the CTA-local, non-multicast form of cp.async.bulk is used.  Every wait
// polls a bounded number of times; a wait that runs out reports failure to
// its caller, which records it in a device error word that the host reads
// (gnss_check) instead of hanging.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gnss {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes the initialised barrier visible to the async proxy
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy ones (re-filling a buffer that threads have just read)
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bytes and both addresses must be multiples of 16
__device__ __forceinline__ void bulk_g2s(void *dst_smem, const void *src_gmem, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; gives up after
// `limit` polls (by default 2^24, a few seconds) and returns false.
constexpr unsigned WAIT_POLLS = 1u << 24;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, unsigned limit = WAIT_POLLS) {
    for (unsigned i = 0; i < limit; ++i) {
        if (mbar_test(bar, parity)) return true;
        if (i > 32) __nanosleep(128);
    }
    return false;
}

// Control of the bounded waits of a kernel, read from err[1] (err[0] is the
// error word): 0 in normal operation.  A nonzero value v is a test of the
// time-out path: every wait gives up after v polls, and block 0 arms its
// first mbarrier phase without issuing the copies that would complete it,
// so that wait runs out with no copy in flight.
struct WaitCtl {
    unsigned limit;
    bool withhold;   // this block withholds the copies of its first phase
    __device__ __forceinline__ explicit WaitCtl(const unsigned *err) {
        const unsigned v = err ? err[1] : 0u;
        limit = v ? v : WAIT_POLLS;
        withhold = v != 0 && blockIdx.x == 0;
    }
};

// Named barrier `id` (1..15; 0 is __syncthreads) over `nthreads` threads,
// whole warps; true on every participant when pred is true on any of them.
__device__ __forceinline__ bool bar_named_or(unsigned id, unsigned nthreads, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\tselp.u32 %0, 1, 0, q;\n}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// ------------------------------------------------- programmatic dependent launch
// A step kernel launched with programmatic stream serialization may start
// (its prologue: twiddle tables, shared-memory barriers) on SMs the previous
// kernel in the stream has left.  pdl_wait() blocks until that kernel has
// completed and its memory is visible; a kernel calls it before its first
// access to global memory another step kernel writes or reads.
// pdl_trigger() lets the next kernel launch once every block of this one has
// called it or exited.  The short kernels (update, Hermitian projection,
// statistics) call it at their start; the persistent ones do not, and their
// blocks trigger by exiting (a trigger tested inside their main loops cost
// the 512^3 FP64 step 1%).  Without that launch attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// (no memory clobber: the trigger only lets the next grid be scheduled; its
// pdl_wait, not the trigger, orders the memory)
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

// ---------------------------------------------------------------- cp.async
// Per-thread asynchronous copies global -> shared (LDGSTS).  src_bytes = 0
// fills the destination with zeros without reading the source.
__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst_smem)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst_smem, const void *src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst_smem)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

}  // namespace gnss
