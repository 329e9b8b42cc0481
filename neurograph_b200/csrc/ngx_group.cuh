// Groups of CTAs that work on one source tile together (sm_100a).
//
// A group is `size` consecutive CTAs of a persistent launch sharing one workspace slot. Their common state (the tile's
// control block: queue lengths, bucket bound, level bounds, counters) lives in global memory and is changed only
// (a) by atomics on counters and (b) by the last CTA to arrive at a group barrier, which applies the barrier's update
// before it releases the others. After every barrier each CTA copies the control block into its shared memory, so
// between barriers all CTAs of a group read the same values. With size 1 the control block may be the CTA's own shared
// copy (ctl == &local), the barrier is __syncthreads() and the update runs on thread 0; with size > 1 the launch is cooperative (all CTAs resident) and every wait is bounded in time: a CTA
// that waits longer than kGroupWaitNs records NGX_TIMEOUT in the run's error flag and stops, and so, bounded the same
// way, do the others.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "ngx_common.cuh"

namespace ngx {

// Barrier words of one group: CTAs arrived at the current barrier, barriers completed.
struct GroupBarrier {
    unsigned arrive;
    unsigned gen;
};

// Longest wait of a CTA for the rest of its group at one barrier (10 s, far beyond any phase of a tile).
constexpr unsigned long long kGroupWaitNs = 10ull * 1000 * 1000 * 1000;
// bar_target of a CTA that gave up waiting and left its group.
constexpr unsigned kGroupLeft = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Copies `words` 8-byte words from global memory (through L2) into shared memory.
__device__ __forceinline__ void copy_from_l2(void* dst, const void* src, int words) {
    auto* d = static_cast<unsigned long long*>(dst);
    const auto* s = static_cast<const unsigned long long*>(src);
    for (int i = 0; i < words; ++i) {
        d[i] = __ldcg(&s[i]);
    }
}

// One CTA's view of its group.
template <typename Ctl>
struct Group {
    Ctl* ctl;               // the group's control block (global memory)
    GroupBarrier* bar;      // the group's barrier words (global memory)
    unsigned long long* parts;  // one word per CTA of the group (block partial sums of the group scans)
    int size;               // CTAs in the group
    int rank;               // this CTA's index in the group
    int* error;             // the run's device error flag

    // Barrier of the group. The last CTA to arrive runs update(*ctl) on its thread 0; then every CTA copies the
    // control block into `local` (its shared memory). bar_target is the CTA's count of barriers passed (shared). A
    // CTA that gave up waiting is out of the group for the rest of the launch: its bar_target becomes kGroupLeft, it
    // joins no later barrier, and its local control block is halted (Ctl::halt: no work left), so it runs to the end
    // of the kernel without touching the group's state; the run then reports NGX_TIMEOUT.
    template <typename Update>
    __device__ __forceinline__ void sync(Ctl& local, unsigned& bar_target, Update&& update) const {
        __syncthreads();
        if (threadIdx.x == 0) {
            bool timed_out = bar_target == kGroupLeft;
            __threadfence();
            if (timed_out) {
                // out of the group already
            } else if (size == 1) {
                update(*ctl);
                __threadfence();
            } else {
                const unsigned target = bar_target + 1u;
                bar_target = target;
                if (atomicAdd(&bar->arrive, 1u) == static_cast<unsigned>(size) - 1u) {
                    atomicExch(&bar->arrive, 0u);
                    update(*ctl);
                    __threadfence();
                    st_release_gpu(&bar->gen, target);
                } else {
                    const unsigned long long t0 = global_ns();
                    while (static_cast<int>(ld_acquire_gpu(&bar->gen) - target) < 0) {
                        if (global_ns() - t0 > kGroupWaitNs) {
                            timed_out = true;
                            atomicCAS(error, kDevOk, kDevTimeout);
                            break;
                        }
                        __nanosleep(128);
                    }
                    __threadfence();
                }
            }
            static_assert(sizeof(Ctl) % 8 == 0, "control block must be whole 8-byte words");
            if (ctl != &local) {
                copy_from_l2(&local, ctl, static_cast<int>(sizeof(Ctl) / 8));
            }
            if (timed_out) {
                bar_target = kGroupLeft;
                local.halt();
            }
        }
        __syncthreads();
    }

    __device__ __forceinline__ void sync(Ctl& local, unsigned& bar_target) const {
        sync(local, bar_target, [](volatile Ctl&) {});
    }
};

// Exclusive prefix sum of in[0..len) into out[0..len] (out[len] = total) by the whole group; returns the total to
// every thread. Each CTA scans a contiguous chunk, offset by the sums of the chunks before it (one group barrier in
// between, one after). With one CTA this is a plain block scan. s_part holds blockDim.x + 3 words.
template <typename Ctl>
__device__ __forceinline__ unsigned long long group_exclusive_scan(const Group<Ctl>& grp, Ctl& local, unsigned& bar_target, const uint32_t* in,
                                                                   uint32_t* out, int64_t len, unsigned long long* s_part) {
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int64_t per_cta = (len + grp.size - 1) / grp.size;
    const int64_t cbeg = grp.rank * per_cta < len ? grp.rank * per_cta : len;
    const int64_t cend = cbeg + per_cta < len ? cbeg + per_cta : len;
    const int64_t clen = cend - cbeg;
    const int64_t chunk = (clen + nthreads - 1) / nthreads;
    const int64_t beg = cbeg + (tid * chunk < clen ? tid * chunk : clen);
    const int64_t end = beg + chunk < cend ? beg + chunk : cend;
    unsigned long long sum = 0;
    for (int64_t i = beg; i < end; ++i) {
        sum += __ldcg(&in[i]);
    }
    s_part[tid] = sum;
    __syncthreads();
    if (tid == 0) {
        unsigned long long run = 0;
        for (int t = 0; t < nthreads; ++t) {
            const unsigned long long x = s_part[t];
            s_part[t] = run;
            run += x;
        }
        s_part[nthreads] = run;
        if (grp.size > 1) {
            __stcg(&grp.parts[grp.rank], run);
        }
    }
    unsigned long long base = 0, total = 0;
    if (grp.size > 1) {
        grp.sync(local, bar_target);
        // every CTA adds the chunks before its own (at most a few hundred words, read by one thread)
        if (tid == 0) {
            unsigned long long before = 0, all = 0;
            for (int r = 0; r < grp.size; ++r) {
                const unsigned long long x = __ldcg(&grp.parts[r]);
                before += r < grp.rank ? x : 0ull;
                all += x;
            }
            s_part[nthreads + 1] = before;
            s_part[nthreads + 2] = all;
        }
        __syncthreads();
        base = s_part[nthreads + 1];
        total = s_part[nthreads + 2];
    } else {
        __syncthreads();
        total = s_part[nthreads];
    }
    unsigned long long run = base + s_part[tid];
    for (int64_t i = beg; i < end; ++i) {
        const uint32_t x = __ldcg(&in[i]);
        out[i] = static_cast<uint32_t>(run);
        run += x;
    }
    if (grp.rank == grp.size - 1 && tid == 0) {
        out[len] = static_cast<uint32_t>(total);
    }
    grp.sync(local, bar_target);
    // a CTA that left its group has partial sums of unknown state: it reports a total no list can hold
    return bar_target == kGroupLeft ? ~0ull : total;
}

}  // namespace ngx
