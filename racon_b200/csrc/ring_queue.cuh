// Device half of the shared work queues (RingService, ring_service.cpp):
// claiming an item and reporting it done. Included by the kernels that
// serve a queue (poa_consensus.cu, nw_align.cu).
//
// Queue state lives in device memory: the host writes batch records, then
// items, then the tail with copies in one stream (each copy starts after the
// previous one completes), so a warp that sees the new tail in L2 finds the
// items and records there too. Idle warps poll that L2 word, never host
// memory: polling over the bus, or acquire loads at system scope, would slow
// the warps still computing on the same SMs.
#pragma once

#include "rb_internal.hpp"

namespace rb {
namespace {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Claims the next item, ring 0 (smallest jobs) first, or the last ring
// first when large_first: returns (batch slot << 32) | index, or ~0 when the
// kernel closes or stop is set. The kernel closes as a whole: a warp that
// has found no work for idle_ns while no warp of the kernel is working sets
// the closing word, and every warp leaves at its next poll. (Warps that left one by one would leave work arriving later
// to the few still busy.) Bounded: once no item is in flight, the kernel
// ends within idle_ns plus one poll. Out of line with scalar arguments, so
// its registers do not add to the item code's. Lane 0 only.
__device__ __noinline__ unsigned long long svc_claim(const uint2* items, const unsigned long long* tail,
                                                     unsigned long long* head, unsigned int* live,
                                                     unsigned long long ring_mask, const unsigned int* stop,
                                                     unsigned long long idle_ns, bool large_first) {
    const unsigned long long t0 = global_ns();
    unsigned int nap = 512;
    volatile unsigned int* vlive = live;
    for (;;) {
        if (*reinterpret_cast<const volatile unsigned int*>(stop) || vlive[1]) return ~0ull;
        for (int k = 0; k < kSvcQueues; ++k) {
            const int q = large_first ? kSvcQueues - 1 - k : k;
            const unsigned long long t = reinterpret_cast<const volatile unsigned long long*>(tail)[q];
            unsigned long long h = reinterpret_cast<volatile unsigned long long*>(head)[q];
            while (h < t) {
                const unsigned long long prev = atomicCAS(head + q, h, h + 1);
                if (prev == h) {
                    atomicAdd(live, 1u);
                    __threadfence();
                    const volatile unsigned int* it = reinterpret_cast<const volatile unsigned int*>(
                        items + size_t(q) * (ring_mask + 1) + (h & ring_mask));
                    return (static_cast<unsigned long long>(it[0]) << 32) | it[1];
                }
                h = prev;
            }
        }
        if (global_ns() - t0 > idle_ns && vlive[0] == 0) {
            atomicExch(live + 1, 1u);
            return ~0ull;
        }
        __nanosleep(nap);
        nap = nap < 32768 ? nap * 2 : nap;
    }
}

// Warp `slot` of the kernel claims its next item.
__device__ __forceinline__ unsigned long long svc_claim(const SvcQueueDev& q, uint32_t slot) {
    const bool large_first = q.large_first_every != 0 && slot % q.large_first_every == q.large_first_every - 1;
    return svc_claim(q.items, q.tail, q.head, q.live, q.ring_mask, q.stop, q.idle_ns, large_first);
}

// Lane 0, after the item's writes are fenced: counts the item done for its
// batch, and the batch's last item raises the batch's flag in host memory.
// The warp then no longer counts as working.
__device__ __forceinline__ void svc_item_done(const SvcQueueDev& q, uint32_t slot, uint32_t total, uint32_t gen) {
    const unsigned int d = atomicAdd(&q.done[slot], 1u) + 1u;
    if (d == total) {
        __threadfence_system();
        q.finished[slot] = gen;
    }
    atomicSub(q.live, 1u);
}

}  // namespace
}  // namespace rb
