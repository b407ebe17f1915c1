// ne_solve.cuh -- island solver drivers shared by the FP64 path and the FP32
// form.
//
// The reference's contact solve (src/world.cpp:559-626) is, per island, a
// fixed sequence of updates: warm start of every contact in order, 8
// Gauss-Seidel sweeps over the contacts in order, then position correction in
// order.  The drivers here only schedule that sequence; what one update
// computes is the `Items` policy of the caller:
//
//   Items::warm(d, c)                   warm-start application of contact c
//   Items::sweep(d, c)                  one sequential-impulse update of c
//   Items::correct(d, c, beta, wout)    position correction of c + warm-cache value
//
// Small islands run one thread each, in order.  Big islands run on the
// dataflow scheduler below, which gives every body exactly the sequence of
// updates the in-order loop would, so both drivers compute the same bits.
#pragma once

#include <cuda/atomic>

#include "ne_step.cuh"

namespace neb {
namespace solve {

// Islands with at least kBigIsland contacts are queued for the dataflow
// solver, the rest are solved one thread per island.
constexpr uint32_t kBigIsland = 48;

// A warp that sees no update complete for this long gives up and reports
// (ctl->solve_timeout -> NE_ERR_TIMEOUT).  Legitimate waits are bounded by the
// island's critical path, well under a millisecond per update.
constexpr unsigned long long kStallNs = 2000000000ull;
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr int kMaxBigThreads = 512;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Island-local view of one contact's update (phase p, contact position pos).
struct BigItem {
    uint32_t c, i, j, pos, p;
    bool mi, mj;
};

__device__ __forceinline__ BigItem big_item(const DevWorld& d, const uint32_t* ord, uint32_t s, uint32_t m,
                                            uint32_t u) {
    BigItem it;
    it.p = u / m;
    it.pos = s + (u - it.p * m);
    it.c = ord[it.pos];
    it.i = d.ci[it.c];
    it.j = d.cj[it.c];
    it.mi = (d.meta[it.i].y & kFlagMutable) != 0;
    it.mj = (d.meta[it.j].y & kFlagMutable) != 0;
    return it;
}

// Number of earlier updates this update waits for: one per mutable body,
// except a body's very first update (phase 0, rank 0).
__device__ __forceinline__ uint32_t big_npred(const DevWorld& d, const BigItem& it) {
    uint32_t n = 0;
    if (it.mi && !(it.p == 0 && d.crank[2 * it.pos] == 0)) ++n;
    if (it.mj && !(it.p == 0 && d.crank[2 * it.pos + 1] == 0)) ++n;
    return n;
}

// The update that follows this one on body b (side 0 = i, 1 = j), or kEmpty.
__device__ __forceinline__ uint32_t big_successor(const DevWorld& d, const uint32_t* rv, const BigItem& it, int side,
                                                  uint32_t b, uint32_t s, uint32_t m) {
    const uint32_t r = d.crank[2 * it.pos + side];
    const uint32_t deg = d.bdeg[b];
    const uint32_t base = d.bstart[b];
    if (r + 1 < deg) return it.p * m + ((rv[base + r + 1] >> 1) - s);
    if (it.p < 9) return (it.p + 1) * m + ((rv[base] >> 1) - s);
    return kEmpty;
}

__device__ __forceinline__ void big_push(uint32_t* queue, uint32_t* tail, uint32_t u) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> t(*tail);
    const uint32_t slot = t.fetch_add(1u, cuda::memory_order_relaxed);
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> q(queue[slot]);
    q.store(u, cuda::memory_order_release);
}

__device__ __forceinline__ void big_notify(uint32_t* cnt, uint32_t* queue, uint32_t* tail, uint32_t u) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_block> c(cnt[u]);
    if (c.fetch_sub(1u, cuda::memory_order_acq_rel) == 1u) big_push(queue, tail, u);
}

// One thread per small island: warm start (src/world.cpp:559-568), 8
// Gauss-Seidel sweeps in the reference's contact order (:572-612), position
// correction (:615-616), warm-cache values (:619-626).  Islands share no
// mutable body, so concurrent islands reproduce the reference's single
// global sweep exactly.  Big islands are queued for island_solve_big.
template <class Items>
__device__ __forceinline__ void island_solve_small(const StepArgs& a, int ib) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctl->islands) return;
    const DevWorld& d = a.d;
    const uint32_t s = d.istart[t], e = d.istart[t + 1];
    atomicMax((unsigned long long*)&ctl->max_island, (unsigned long long)(e - s));
    if (e - s >= kBigIsland) {
        const uint32_t slot = atomicAdd(&ctl->nbig, 1u);
        d.big[slot] = (uint32_t)t;
        return;
    }
    const uint32_t* ord = d.iord[ib];
    if (a.warm)
        for (uint32_t k = s; k < e; ++k) Items::warm(d, ord[k]);
    for (int it = 0; it < 8; ++it)
        for (uint32_t k = s; k < e; ++k) Items::sweep(d, ord[k]);
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const double beta = a.wp[a.bw[d.ci[ord[s]]]].beta;
    for (uint32_t k = s; k < e; ++k) Items::correct(d, ord[k], beta, wout);
}

// Dataflow solver for the big islands, one CTA per island at a time.
//
// The reference's work on an island is a sequence of 10*m updates (phase 0 =
// warm start, phases 1-8 = the Gauss-Seidel sweeps, phase 9 = position
// correction; m contacts in order).  An update reads and writes only its two
// bodies, so it depends only on the previous update of each of those bodies
// in that sequence.  Each update counts its unfinished predecessors (<= 2);
// finishing an update decrements its successors' counts, and the update that
// reaches zero is appended to a ready queue.  Lanes claim queue slots in order
// and run the update in a slot once it is filled.  Every body therefore sees
// exactly the reference's sequence of updates (bit-identical result), and the
// schedule is greedy list scheduling, whose length is close to the
// dependency graph's critical path.  Progress is guaranteed: while updates
// remain, some update is ready, and the lowest unfilled slot is claimed by a
// waiting lane.  Lanes poll warp-synchronously (no lane spins alone, so a
// ready update is never starved by divergent waiters), and every wait is
// bounded and reports through ctl->solve_timeout.
template <class Items>
__device__ __forceinline__ void island_solve_big(const StepArgs& a, int ib, int rb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    __shared__ int s_fail;
    __shared__ uint32_t s_head, s_tail;
    const DevWorld& d = a.d;
    const uint32_t* ord = d.iord[ib];
    const uint32_t* rv = d.rval[rb];
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const uint32_t nbig = ctl->nbig;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t t = d.big[bi];
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        const uint32_t m = e - s;
        const uint32_t total = 10u * m;
        const double beta = a.wp[a.bw[d.ci[ord[s]]]].beta;
        uint32_t* cnt = d.bcnt10 + 10u * s;      // per-island slices of the 10*C scratch
        uint32_t* queue = d.bq10 + 10u * s;
        if (threadIdx.x == 0) { s_fail = 0; s_head = 0; s_tail = 0; }
        for (uint32_t u = threadIdx.x; u < total; u += blockDim.x) {
            cnt[u] = big_npred(d, big_item(d, ord, s, m, u));
            queue[u] = kEmpty;
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < m; k += blockDim.x)
            if (cnt[k] == 0) big_push(queue, &s_tail, k);
        __syncthreads();

        cuda::atomic_ref<uint32_t, cuda::thread_scope_block> head(s_head);
        uint32_t h = head.fetch_add(1u, cuda::memory_order_relaxed);
        unsigned long long last_progress = global_ns();
        uint32_t rounds = 0;
        while (true) {
            const bool live = h < total;
            if (!__any_sync(0xffffffffu, live)) break;
            uint32_t u = kEmpty;
            if (live) {
                cuda::atomic_ref<uint32_t, cuda::thread_scope_block> q(queue[h]);
                u = q.load(cuda::memory_order_acquire);
            }
            const bool ready = u != kEmpty;
            if (ready) {
                const BigItem it = big_item(d, ord, s, m, u);
                if (it.p == 0) {
                    if (a.warm) Items::warm(d, it.c);
                } else if (it.p <= 8) {
                    Items::sweep(d, it.c);
                } else {
                    Items::correct(d, it.c, beta, wout);
                }
                const uint32_t si = it.mi ? big_successor(d, rv, it, 0, it.i, s, m) : kEmpty;
                const uint32_t sj = it.mj ? big_successor(d, rv, it, 1, it.j, s, m) : kEmpty;
                if (si != kEmpty) big_notify(cnt, queue, &s_tail, si);
                if (sj != kEmpty) big_notify(cnt, queue, &s_tail, sj);
                h = head.fetch_add(1u, cuda::memory_order_relaxed);
            }
            // Check the clock every 64 idle rounds; lane 0's reading decides
            // for the warp so the exit is warp-uniform.
            bool stalled = false;
            if (__any_sync(0xffffffffu, ready)) {
                rounds = 0;
                last_progress = global_ns();
            } else if ((++rounds & 63u) == 0u) {
                stalled = __shfl_sync(0xffffffffu, global_ns() - last_progress > kStallNs ? 1 : 0, 0) != 0;
            }
            const bool failed = __any_sync(0xffffffffu, *(volatile int*)&s_fail != 0);   // warp-uniform
            if (stalled || failed) {
                if ((threadIdx.x & 31) == 0) {
                    s_fail = 1;
                    atomicExch(&ctl->solve_timeout, 1u);
                }
                break;
            }
        }
        __syncthreads();
    }
}

}  // namespace solve
}  // namespace neb
