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
// Small islands run one thread each, in order.  Big islands run on one of the
// dataflow schedulers below (one CTA per island, or a team of CTAs), which give
// every body exactly the sequence of updates the in-order loop would, so all
// drivers compute the same bits.
#pragma once

#include <cuda/atomic>

#include "ne_step.cuh"

namespace neb {
namespace solve {

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

// One thread per small island: warm start (src/world.cpp:559-568), 8
// Gauss-Seidel sweeps in the reference's contact order (:572-612), position
// correction (:615-616), warm-cache values (:619-626).  Islands share no
// mutable body, so concurrent islands reproduce the reference's single
// global sweep exactly.  Big islands are queued for the dataflow solvers.
//
// island_list (one thread per island) records the largest island and lists
// the big ones with their size classes first, so that the big-island solvers
// and the small-island solve can run side by side.
__device__ __forceinline__ void island_list(const StepArgs& a) {
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
        atomicAdd(&ctl->big_class[31 - __clz(e - s)], 1u);
    }
}

template <class Items>
__device__ __forceinline__ void island_solve_small(const StepArgs& a, int ib) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctl->islands) return;
    const DevWorld& d = a.d;
    const uint32_t s = d.istart[t], e = d.istart[t + 1];
    if (e - s >= kBigIsland) return;   // listed for the dataflow solvers
    const uint32_t* ord = d.iord[ib];
    if (a.warm)
        for (uint32_t k = s; k < e; ++k) Items::warm(d, ord[k]);
    for (int it = 0; it < 8; ++it)
        for (uint32_t k = s; k < e; ++k) Items::sweep(d, ord[k]);
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const double beta = a.wp[a.bw[d.ci[ord[s]]]].beta;
    for (uint32_t k = s; k < e; ++k) Items::correct(d, ord[k], beta, wout);
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

// Block-local dataflow solver: one CTA per big island at a time, ready queue
// head/tail in shared memory and block-scope atomics (team size 1).
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
__device__ __forceinline__ void island_solve_local(const StepArgs& a, int ib, int rb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    __shared__ int s_fail;
    __shared__ uint32_t s_head, s_tail;
    const DevWorld& d = a.d;
    const uint32_t* ord = d.iord[ib];
    const uint32_t* rv = d.rval[rb];
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const uint32_t nbig = ctl->nbig;
    __shared__ uint32_t s_stop;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t t = d.big[bi];
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        const uint32_t m = e - s;
        if (m <= a.local_cap) continue;          // island_solve_shared takes it
        if (threadIdx.x == 0) s_stop = *(volatile uint32_t*)&ctl->solve_timeout;
        __syncthreads();
        if (s_stop) break;                       // a wait ran out elsewhere: the step is an error
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

// ---- big islands: shared-memory dataflow solver (one CTA per island) -------
//
// The same update sequence and dependency rule as island_solve_local, with
// the bookkeeping taken off the critical path:
//
//  * big_rec (a grid-wide pass before the solve) writes one 32-byte record
//    per island position -- contact, bodies, mutability, phase-0 predecessor
//    count, and the island position of the next update on each body (same
//    phase, or bit 31 set: the body's first contact in the next phase) -- and
//    empties the island's queue slots.  An update then costs one record load
//    instead of a chain of index loads.
//  * Predecessor counters are bytes in shared memory, one per contact
//    position, reused by the ten phases: the update (p, q) re-arms its own
//    counter for (p + 1, q) before it notifies anyone.  Every predecessor of
//    (p + 1, q) comes after (p, q) on its body, so its decrement is ordered
//    after that re-arm through the acquire/release chain of the counters.
//    Four counters share a 32-bit word; a decrement never takes a byte below
//    zero, so there is no borrow between them.
//  * The lane whose decrement makes an update ready runs it next itself (a
//    continuation); only a second ready successor goes through the queue.
//
// Islands above local_cap contacts are left to island_solve_local.
__device__ __forceinline__ void big_rec(const StepArgs& a, int ib, int rb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const DevWorld& d = a.d;
    const uint64_t C = ctl->C;
    const uint32_t* ord = d.iord[ib];
    const uint32_t* rv = d.rval[rb];
    // Claim order of the big islands: larger size classes first.
    const uint32_t nbig = ctl->nbig;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nbig; g += gridDim.x * blockDim.x) {
        const uint32_t t = d.big[g];
        const uint32_t cls = 31 - __clz(d.istart[t + 1] - d.istart[t]);
        uint32_t off = 0;
        for (uint32_t k = cls + 1; k < 32; ++k) off += ctl->big_class[k];
        d.bigs[off + atomicAdd(&ctl->big_fill[cls], 1u)] = t;
    }
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < C; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = d.ioff[k] + d.iflag[k] - 1u;
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        if (e - s < kBigIsland) continue;
        const uint32_t c = ord[k];
        const uint32_t i = d.ci[c], j = d.cj[c];
        const bool mi = (d.meta[i].y & kFlagMutable) != 0, mj = (d.meta[j].y & kFlagMutable) != 0;
        uint32_t nxt[2] = {kEmpty, kEmpty}, npred0 = 0;
        #pragma unroll
        for (int side = 0; side < 2; ++side) {
            if (!(side ? mj : mi)) continue;
            const uint32_t b = side ? j : i;
            const uint32_t r = d.crank[2 * k + side];
            const uint32_t deg = d.bdeg[b], base = d.bstart[b];
            if (r != 0) ++npred0;
            nxt[side] = (r + 1 < deg) ? (rv[base + r + 1] >> 1) - s : (((rv[base] >> 1) - s) | 0x80000000u);
        }
        d.brec[2 * k] = make_uint4(c, i, j, (mi ? 1u : 0u) | (mj ? 2u : 0u) | (npred0 << 2));
        d.brec[2 * k + 1] = make_uint4(nxt[0], nxt[1], 0u, 0u);
        uint32_t* q = d.bq10 + 10 * k;
        #pragma unroll
        for (int r = 0; r < 10; ++r) q[r] = kEmpty;
    }
}

template <class Items>
__device__ __forceinline__ void island_solve_shared(const StepArgs& a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    extern __shared__ uint32_t s_cnt[];   // a.local_cap byte counters
    __shared__ uint32_t s_head, s_tail, s_done, s_bi;
    __shared__ int s_fail;
    const DevWorld& d = a.d;
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const uint32_t nbig = ctl->nbig;
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    constexpr uint32_t kNone = 0xfffffffeu;
    using BlockAtomic = cuda::atomic_ref<uint32_t, cuda::thread_scope_block>;
    while (true) {
        // Thread 0 claims the next island (largest size classes first) and
        // reads the failure flag; the block acts on both together.
        __syncthreads();   // every thread has read the previous claim
        if (threadIdx.x == 0)
            s_bi = *(volatile uint32_t*)&ctl->solve_timeout ? nbig : atomicAdd(&ctl->big_next, 1u);
        __syncthreads();
        const uint32_t bi = s_bi;
        if (bi >= nbig) break;   // no island left, or a wait ran out elsewhere (the step is an error)
        const uint32_t t = d.bigs[bi];
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        const uint32_t m = e - s;
        if (m > a.local_cap) continue;
        const uint32_t total = 10u * m;
        const uint4* rec = d.brec + 2 * (size_t)s;
        uint32_t* queue = d.bq10 + 10 * (size_t)s;
        const double beta = a.wp[a.bw[rec[0].y]].beta;
        if (threadIdx.x == 0) { s_head = 0; s_tail = 0; s_done = 0; s_fail = 0; }
        for (uint32_t wd = threadIdx.x; 4 * wd < m; wd += blockDim.x) {
            uint32_t word = 0;
            #pragma unroll
            for (int b = 0; b < 4; ++b)
                if (4 * wd + b < m) word |= ((rec[2 * (4 * wd + b)].w >> 2) & 3u) << (8 * b);
            s_cnt[wd] = word;
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < m; q += blockDim.x)
            if (((s_cnt[q >> 2] >> (8 * (q & 3))) & 0xffu) == 0u) {
                BlockAtomic tl(s_tail);
                BlockAtomic(queue[tl.fetch_add(1u, cuda::memory_order_relaxed)]).store(q, cuda::memory_order_relaxed);
            }
        __syncthreads();

        BlockAtomic head(s_head), tail(s_tail), done(s_done);
        uint32_t cont = kEmpty, slot = kNone;
        unsigned long long last_progress = global_ns();
        uint32_t rounds = 0;
        while (true) {
            // Lanes without work take queue entries that have been pushed
            // (never slots ahead of the tail): an entry goes to the first warp
            // with an idle lane that comes by, not to a lane whose warp is
            // still busy with a long update.
            const bool need = cont == kEmpty && slot == kNone;
            const uint32_t nb = __ballot_sync(0xffffffffu, need);
            if (nb) {
                uint32_t base = 0, take = 0;
                if (lane == __ffs(nb) - 1) {
                    uint32_t h = head.load(cuda::memory_order_relaxed);
                    for (int tries = 0; tries < 8; ++tries) {
                        const uint32_t avail = tail.load(cuda::memory_order_relaxed) - h;
                        take = min((uint32_t)__popc(nb), avail);
                        if (take == 0) break;
                        if (head.compare_exchange_weak(h, h + take, cuda::memory_order_relaxed)) { base = h; break; }
                        take = 0;
                    }
                }
                base = __shfl_sync(0xffffffffu, base, __ffs(nb) - 1);
                take = __shfl_sync(0xffffffffu, take, __ffs(nb) - 1);
                const uint32_t rank = __popc(nb & lt);
                if (need && rank < take) slot = base + rank;
            }
            // Ordering: an update's stores and its counter re-arm are released
            // by one fence before its notifications (relaxed counter
            // decrements); the lane that takes a successor -- as its
            // continuation, or from the queue -- fences once after seeing it
            // ready, which acquires every predecessor's stores.
            uint32_t u = cont;
            cont = kEmpty;
            if (u == kEmpty && slot < total) {
                const uint32_t x = BlockAtomic(queue[slot]).load(cuda::memory_order_relaxed);
                if (x != kEmpty) {
                    u = x;
                    slot = kNone;
                    cuda::atomic_thread_fence(cuda::memory_order_acq_rel, cuda::thread_scope_block);
                }
            }
            const bool ready = u != kEmpty;
            if (ready) {
                const uint32_t p = u / m, q = u - p * m;
                const uint4 r0 = rec[2 * q], r1 = rec[2 * q + 1];
                if (p == 0) {
                    if (a.warm) Items::warm(d, r0.x);
                } else if (p <= 8) {
                    Items::sweep(d, r0.x);
                } else {
                    Items::correct(d, r0.x, beta, wout);
                }
                const uint32_t sh = 8u * (q & 3u);
                if (p < 9) atomicAdd(&s_cnt[q >> 2], ((r0.w & 1u) + ((r0.w >> 1) & 1u)) << sh);
                cuda::atomic_thread_fence(cuda::memory_order_acq_rel, cuda::thread_scope_block);
                uint32_t extra = kEmpty;
                bool got = false;
                #pragma unroll
                for (int side = 0; side < 2; ++side) {
                    const uint32_t nx = side ? r1.y : r1.x;
                    if (nx == kEmpty) continue;
                    uint32_t np = p, nq = nx;
                    if (nx & 0x80000000u) {
                        if (p == 9) continue;
                        np = p + 1;
                        nq = nx & 0x7fffffffu;
                    }
                    const uint32_t nsh = 8u * (nq & 3u);
                    const uint32_t old = atomicSub(&s_cnt[nq >> 2], 1u << nsh);
                    if (((old >> nsh) & 0xffu) != 1u) continue;
                    got = true;
                    const uint32_t nu = np * m + nq;
                    if (cont == kEmpty) cont = nu; else extra = nu;
                }
                if (got) cuda::atomic_thread_fence(cuda::memory_order_acq_rel, cuda::thread_scope_block);
                if (extra != kEmpty) {
                    const uint32_t sl = tail.fetch_add(1u, cuda::memory_order_relaxed);
                    BlockAtomic(queue[sl]).store(extra, cuda::memory_order_relaxed);
                }
            }
            const uint32_t rb_ = __ballot_sync(0xffffffffu, ready);
            if (rb_ && lane == __ffs(rb_) - 1) done.fetch_add((uint32_t)__popc(rb_), cuda::memory_order_relaxed);
            if (rb_) {
                rounds = 0;
                last_progress = global_ns();
                continue;
            }
            if (__any_sync(0xffffffffu, cont != kEmpty)) continue;
            // Idle warp: finished island, failure elsewhere, or a stall.
            ++rounds;   // warp-uniform
            int stop = 0;
            if (lane == 0) {
                if (done.load(cuda::memory_order_relaxed) >= total) stop = 1;
                else if (*(volatile int*)&s_fail) stop = 1;
                else if ((rounds & 63u) == 0u && global_ns() - last_progress > kStallNs) stop = 2;
            }
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop == 2 && lane == 0) {
                s_fail = 1;
                atomicExch(&ctl->solve_timeout, 1u);
            }
            if (stop) break;
        }
        __syncthreads();
    }
}

// ---- big islands: a team of CTAs per island --------------------------------
//
// The reference's work on an island is a sequence of 10*m updates (phase 0 =
// warm start, phases 1-8 = the Gauss-Seidel sweeps, phase 9 = position
// correction; m contacts in order).  An update reads and writes only its two
// bodies, so it depends only on the previous update of each of those bodies
// in that sequence.  Each update counts its unfinished predecessors (<= 2);
// finishing an update decrements its successors' counts.  Every body
// therefore sees exactly the reference's sequence of updates (bit-identical
// result) whatever the schedule.
//
// Schedule: the lane whose decrement makes a successor ready runs it next
// itself (a continuation), so chains along the critical path never pass
// through a queue; a second ready successor is appended to the island's ready
// queue.  Idle lanes claim queue slots in order (one atomic per warp) and run
// the update in a slot once it is filled.  All counters, the queue and the
// mutable body state live in global memory with device-scope acquire/release
// ordering and L2-coherent loads, so an island can be worked on by a team of
// CTAs on many SMs: k_big_plan gives each big island a team proportional to
// its update count (at least one CTA; islands beyond the grid are taken in
// turn).  Progress: the lowest unfinished update is ready, and it is either a
// lane's continuation or in a queue slot that is, or will next be, claimed by
// a waiting lane.  Lanes poll warp-synchronously, and every wait is bounded
// and reports through ctl->solve_timeout.

// Coherent (L2) access to solver state that another SM may have written.
__device__ __forceinline__ D4 ldcg(const D4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldcg(q), b = __ldcg(q + 1);
    D4 r; r.x = a.x; r.y = a.y; r.z = b.x; r.w = b.y;
    return r;
}
__device__ __forceinline__ void stcg(D4* p, const D4& v) {
    double2* q = reinterpret_cast<double2*>(p);
    __stcg(q, make_double2(v.x, v.y));
    __stcg(q + 1, make_double2(v.z, v.w));
}
__device__ __forceinline__ F4 ldcg(const F4* p) {
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    F4 r; r.x = a.x; r.y = a.y; r.z = a.z; r.w = a.w;
    return r;
}
__device__ __forceinline__ void stcg(F4* p, const F4& v) {
    __stcg(reinterpret_cast<float4*>(p), make_float4(v.x, v.y, v.z, v.w));
}
__device__ __forceinline__ double2 ldcg(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ void stcg(double2* p, const double2& v) { __stcg(p, v); }

// Loads and stores of mutable solver state: plain for the one-thread small
// islands, coherent for the team solver.
template <bool Coherent, typename T>
__device__ __forceinline__ T ld_state(const T* p) {
    if constexpr (Coherent) return ldcg(p); else return *p;
}
template <bool Coherent, typename T>
__device__ __forceinline__ void st_state(T* p, const T& v) {
    if constexpr (Coherent) stcg(p, v); else *p = v;
}

// Island k of the team that virtual CTA v belongs to (bteam: team starts).
__device__ __forceinline__ uint32_t team_island(const uint32_t* bteam, uint32_t nbig, uint32_t v) {
    uint32_t lo = 0, hi = nbig - 1;   // last k with bteam[k] <= v
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (bteam[mid] <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Teams (single block of kPlanThreads): island k gets
// clamp(floor(G * m_k / sum m), 1, team_max) of the G CTAs; bteam = exclusive
// prefix of team sizes, bteam[nbig] = number of virtual CTAs.
constexpr int kPlanThreads = 1024;

__device__ __forceinline__ void big_plan(const StepArgs& a, uint32_t G) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const DevWorld& d = a.d;
    const uint32_t nbig = ctl->nbig;
    __shared__ unsigned long long s_sum[kPlanThreads / 32];
    __shared__ unsigned long long s_total;
    __shared__ uint32_t s_warp[kPlanThreads / 32], s_carry;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned long long acc = 0;
    for (uint32_t k = threadIdx.x; k < nbig; k += blockDim.x) {
        const uint32_t t = d.big[k];
        acc += d.istart[t + 1] - d.istart[t];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) s_sum[w] = acc;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long tot = 0;
        for (int k = 0; k < kPlanThreads / 32; ++k) tot += s_sum[k];
        s_total = tot ? tot : 1;
    }
    __syncthreads();
    const unsigned long long W = s_total;
    for (uint32_t base = 0; base < nbig; base += blockDim.x) {
        const uint32_t k = base + threadIdx.x;
        uint32_t team = 0;
        if (k < nbig) {
            const uint32_t t = d.big[k];
            const unsigned long long mk = d.istart[t + 1] - d.istart[t];
            team = (uint32_t)((unsigned long long)G * mk / W);
            team = team < 1u ? 1u : team;
            if (a.big_team_max > 0 && team > (uint32_t)a.big_team_max) team = (uint32_t)a.big_team_max;
        }
        uint32_t inc = team;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += x;
        }
        if (lane == 31) s_warp[w] = inc;
        __syncthreads();
        if (w == 0) {
            const uint32_t x = s_warp[lane];
            uint32_t xi = x;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, xi, o);
                if (lane >= o) xi += y;
            }
            s_warp[lane] = xi - x;
        }
        __syncthreads();
        if (k < nbig) d.bteam[k] = s_carry + s_warp[w] + inc - team;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) s_carry += s_warp[w] + inc;
        __syncthreads();
    }
    if (threadIdx.x == 0) d.bteam[nbig] = s_carry;
}

// Predecessor counts, an empty queue with the initially ready updates, and
// the control block of every big island; one block per island at a time.
__device__ __forceinline__ void big_init(const StepArgs& a, int ib) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const DevWorld& d = a.d;
    const uint32_t nbig = ctl->nbig;
    const uint32_t* ord = d.iord[ib];
    __shared__ uint32_t s_tail;
    for (uint32_t k = blockIdx.x; k < nbig; k += gridDim.x) {
        const uint32_t t = d.big[k];
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        const uint32_t m = e - s;
        const uint32_t total = 10u * m;
        uint32_t* cnt = d.bcnt10 + 10u * s;
        uint32_t* queue = d.bq10 + 10u * s;
        if (threadIdx.x == 0) s_tail = 0;
        for (uint32_t u = threadIdx.x; u < total; u += blockDim.x) {
            cnt[u] = big_npred(d, big_item(d, ord, s, m, u));
            queue[u] = kEmpty;
        }
        __syncthreads();
        for (uint32_t u = threadIdx.x; u < m; u += blockDim.x)   // only phase 0 can start ready
            if (cnt[u] == 0) queue[atomicAdd(&s_tail, 1u)] = u;
        __syncthreads();
        if (threadIdx.x == 0) {
            BigCtl c;
            c.head = 0; c.tail = s_tail; c.done = 0; c.fail = 0;
            d.bctl[k] = c;
        }
        __syncthreads();
    }
}

template <class Items>
__device__ __forceinline__ void island_solve_team(const StepArgs& a, int ib, int rb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const DevWorld& d = a.d;
    const uint32_t nbig = ctl->nbig;
    if (nbig == 0) return;
    const uint32_t* ord = d.iord[ib];
    const uint32_t* rv = d.rval[rb];
    double* wout = a.warm ? d.wimp[ctl->wsel ^ 1] : nullptr;
    const int lane = threadIdx.x & 31;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t nvirt = d.bteam[nbig];
    constexpr uint32_t kNone = 0xfffffffeu;
    for (uint32_t v = blockIdx.x; v < nvirt; v += gridDim.x) {
        const uint32_t k = team_island(d.bteam, nbig, v);
        const uint32_t t = d.big[k];
        const uint32_t s = d.istart[t], e = d.istart[t + 1];
        const uint32_t m = e - s;
        const uint32_t total = 10u * m;
        const double beta = a.wp[a.bw[d.ci[ord[s]]]].beta;
        uint32_t* cnt = d.bcnt10 + 10u * s;
        uint32_t* queue = d.bq10 + 10u * s;
        BigCtl* bc = d.bctl + k;
        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> head(bc->head), tail(bc->tail), done(bc->done),
            fail(bc->fail);
        uint32_t cont = kEmpty, slot = kNone;
        unsigned long long last_progress = global_ns();
        uint32_t rounds = 0;
        while (true) {
            // Lanes without work claim the next queue slots (one atomic per warp).
            const bool need = cont == kEmpty && slot == kNone;
            const uint32_t nb = __ballot_sync(0xffffffffu, need);
            if (nb) {
                uint32_t base = 0;
                if (lane == __ffs(nb) - 1) base = head.fetch_add((uint32_t)__popc(nb), cuda::memory_order_relaxed);
                base = __shfl_sync(0xffffffffu, base, __ffs(nb) - 1);
                if (need) slot = base + __popc(nb & lt);
            }
            uint32_t u = cont;
            cont = kEmpty;
            if (u == kEmpty && slot < total) {
                cuda::atomic_ref<uint32_t, cuda::thread_scope_device> q(queue[slot]);
                const uint32_t x = q.load(cuda::memory_order_acquire);
                if (x != kEmpty) { u = x; slot = kNone; }
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
                #pragma unroll
                for (int side = 0; side < 2; ++side) {
                    const uint32_t nx = side ? sj : si;
                    if (nx == kEmpty) continue;
                    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> c(cnt[nx]);
                    if (c.fetch_sub(1u, cuda::memory_order_acq_rel) != 1u) continue;
                    if (cont == kEmpty) {
                        cont = nx;
                    } else {
                        const uint32_t sl = tail.fetch_add(1u, cuda::memory_order_relaxed);
                        cuda::atomic_ref<uint32_t, cuda::thread_scope_device> q(queue[sl]);
                        q.store(nx, cuda::memory_order_release);
                    }
                }
            }
            const uint32_t rb_ = __ballot_sync(0xffffffffu, ready);
            if (rb_ && lane == __ffs(rb_) - 1) done.fetch_add((uint32_t)__popc(rb_), cuda::memory_order_release);
            if (rb_) {
                rounds = 0;
                last_progress = global_ns();
                continue;
            }
            if (__any_sync(0xffffffffu, cont != kEmpty)) continue;
            // Idle warp: finished island, failure elsewhere, or a stall.
            ++rounds;   // warp-uniform
            int stop = 0;
            if (lane == 0) {
                if (done.load(cuda::memory_order_acquire) >= total) stop = 1;
                else if (fail.load(cuda::memory_order_relaxed)) stop = 1;
                else if ((rounds & 63u) == 0u && global_ns() - last_progress > kStallNs) stop = 2;
            }
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop == 2 && lane == 0) {
                fail.store(1u, cuda::memory_order_relaxed);
                atomicExch(&ctl->solve_timeout, 1u);
            }
            if (stop) break;
            if (rounds >= 16) __nanosleep(64);   // long idle: ease the polling traffic
        }
    }
}

}  // namespace solve
}  // namespace neb
