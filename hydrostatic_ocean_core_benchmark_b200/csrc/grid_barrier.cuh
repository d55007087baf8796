// Bounded grid-wide barrier of the persistent cooperative solvers. Each CTA
// calls grid_sync_begin once at the start of a launch, then grid_sync at every
// barrier; all CTAs of the launch must pass the same number of barriers.
#pragma once

#include "ocean_b200.h"

namespace oc {

static constexpr long long kBarrierCycles = 2000000000LL;
static constexpr unsigned long long kBarrierEpoch = 1ULL << 32;

// Grid barrier over a 64-bit arrival counter that only grows: barrier n of a
// launch completes when the counter reaches base + (n + 1) * ncta, so it needs
// no reset and no generation word. Every launch starts at a multiple of 2^32
// (grid_sync_end moves the counter there after a launch's last barrier), so the
// first barrier of a launch learns the base from its own arrival (an atomic add
// with release semantics) whatever the number of CTAs of this launch or of the
// one before; later arrivals are release reductions, whose value nobody waits
// for. A launch makes fewer than 2^32 arrivals. The wait is an
// acquire spin on the counter, bounded in time. A CTA that gives up records
// OC_ERR_TIMEOUT in the status word, which the waiting CTAs poll, so every CTA
// leaves the solve; the status is sticky, so a later launch that finds it set
// makes no arrivals and the counter stays a multiple of the grid. Thread 0
// hands the outcome to its CTA through shared memory.
struct GridBar {
    unsigned long long next;  // counter value that completes the next barrier; 0 before the first
    int ok;
};
static __shared__ GridBar s_gbar;

static __device__ __forceinline__ void grid_sync_begin(const int* status) {
    if (threadIdx.x == 0) {
        s_gbar.next = 0;
        s_gbar.ok = *((volatile const int*)status) == 0;
    }
}

// thread 0's arrival and wait, out of line: the solve calls the barrier from many places.
// ncta: the CTAs taking part (the launch's grid, or one member's share of it)
static __device__ __noinline__ void grid_arrive_wait(unsigned long long* cnt, int* status, unsigned ncta,
                                                     long long bound) {
    unsigned long long target = s_gbar.next;
    if (target == 0) {
        unsigned long long old;
        asm volatile("atom.add.release.gpu.u64 %0, [%1], 1;" : "=l"(old) : "l"(cnt) : "memory");
        target = (old & ~(kBarrierEpoch - 1)) + ncta;
    } else {
        asm volatile("red.add.release.gpu.u64 [%0], 1;" ::"l"(cnt) : "memory");
    }
    s_gbar.next = target + ncta;
    const long long t0 = clock64();
    for (unsigned spin = 1;; ++spin) {
        unsigned long long v;
        asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(cnt) : "memory");
        if (v >= target) break;
        if ((spin & 63) == 0 || spin == 2) {  // the second spin too: a bound of a few cycles runs out
            if (*((volatile int*)status) != 0) {
                s_gbar.ok = 0;
                break;
            }
            if (clock64() - t0 > bound) {
                atomicExch(status, OC_ERR_TIMEOUT);
                s_gbar.ok = 0;
                break;
            }
        }
    }
}

static __device__ __forceinline__ bool grid_sync(unsigned long long* cnt, int* status, unsigned ncta,
                                                 long long bound = kBarrierCycles) {
    __syncthreads();
    if (threadIdx.x == 0 && s_gbar.ok) grid_arrive_wait(cnt, status, ncta, bound);
    __syncthreads();
    return s_gbar.ok != 0;
}

static __device__ __forceinline__ bool grid_sync(unsigned long long* cnt, int* status) {
    return grid_sync(cnt, status, gridDim.x);
}

// After the launch's last barrier, by one thread of one CTA (`leader`): every
// CTA has made all its arrivals, so the counter moves to the next multiple of
// 2^32, where the next launch on this counter starts. A launch that made no
// arrival, or whose barriers gave up, leaves it as it is.
static __device__ __forceinline__ void grid_sync_end(unsigned long long* cnt, bool leader) {
    if (!leader || threadIdx.x != 0 || !s_gbar.ok || s_gbar.next == 0) return;
    unsigned long long v;
    asm volatile("ld.acquire.gpu.u64 %0, [%1];" : "=l"(v) : "l"(cnt) : "memory");
    const unsigned long long pad = (v & ~(kBarrierEpoch - 1)) + kBarrierEpoch - v;
    asm volatile("red.add.release.gpu.u64 [%0], %1;" ::"l"(cnt), "l"(pad) : "memory");
}

}  // namespace oc
