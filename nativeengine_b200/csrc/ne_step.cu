// ne_step.cu -- the device kernels of one World::step() (src/world.cpp:133-146).
//
// Stage map (reference -> kernel):
//   integrate()            src/world.cpp:373-411   k_integrate
//   broadphasePairs()      src/world.cpp:424-501   k_cell_keys, radix sort, cell table (k_cell_flags,
//                                                  k_cell_table); reference-rule list: k_pair_count, k_pair_emit
//   pair filters + cull    src/world.cpp:513-516   k_surv_gather, k_surv_place (fused with the pair lists)
//   gatherContacts()       src/world.cpp:88-130    k_narrowphase (ne_geom.cuh), in class order when
//                                                  worlds mix shapes (k_pair_class + a radix sort);
//                                                  meshes and compounds: k_narrowphase_ext
//   constraint build       src/world.cpp:537-553   k_constraint_build (+ union-find hooking)
//   islands                src/world.cpp:332-343   k_island_label, radix sort, k_island_mark/_start,
//                                                  k_island_list
//   warm start + 8 SI + position correction + warm-cache store
//                          src/world.cpp:559-626   k_island_solve (small islands, side stream),
//                                                  k_big_rec + k_island_solve_shared (big islands),
//                                                  k_island_solve_local / k_island_solve_big
//   wrapPositions/applyWalls src/world.cpp:635-702 k_boundary
//
// Every kernel is a no-op once ctl->abort is set (a capacity overflow this
// step); the host then restores the pre-step snapshot, grows the buffer and
// re-runs the step, so an overflow never changes the result.
#include "ne_solve.cuh"

namespace neb {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ V3 v3of(const D4& a) { return mk(a.x, a.y, a.z); }
__device__ __forceinline__ Q qof(const D4& a) { return mkq(a.x, a.y, a.z, a.w); }
__device__ __forceinline__ D4 d4of(const V3& v, double w) { D4 r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }
__device__ __forceinline__ D4 d4ofq(const Q& q) { D4 r; r.x = q.w; r.y = q.x; r.z = q.y; r.w = q.z; return r; }

__device__ __forceinline__ bool grid_excluded(int shape) { return shape == SH_PLANE || shape == SH_MESH; }

__device__ __forceinline__ BodyG load_geom(const DevWorld& d, uint32_t i) {
    const D4 p = d.pos[i], q = d.quat[i], g = d.geom[i], e = d.ext[i];
    const uint4 m = d.meta[i];
    const uint2 vr = d.vrng[i];
    BodyG b;
    b.x = v3of(p);
    b.q = qof(q);
    b.he = v3of(e);
    b.radius = g.x;
    b.half_height = g.y;
    b.verts = d.verts + vr.x;
    b.nverts = (int)vr.y;
    b.shape = (int)m.x;
    return b;
}

__device__ __forceinline__ int bitlen_u64(unsigned long long x) { return x ? 64 - __clzll((long long)x) : 0; }

// Grid used by one broadphase pass: the reference's (cell = 2 * max bounding
// radius, planes excluded) or the internal one (large bodies excluded like
// planes, cell from the remaining bodies).
struct GridSel {
    double cell;
    long long nc[3];
    int brute;
    const uint32_t* xl;      // excluded bodies of the world, ascending
    uint32_t xb, xe;
};

__device__ __forceinline__ GridSel grid_sel(const StepArgs& a, const WorldP& W, int fast) {
    GridSel G;
    if (fast) {
        G.cell = W.fcell;
        for (int k = 0; k < 3; ++k) G.nc[k] = W.fnc[k];
        G.brute = W.fbrute;
        G.xl = a.d.xlist;
        G.xb = W.xl_begin;
        G.xe = W.xl_end;
    } else {
        G.cell = W.cell;
        for (int k = 0; k < 3; ++k) G.nc[k] = W.nc[k];
        G.brute = W.brute;
        G.xl = a.d.planes;
        G.xb = W.plane_begin;
        G.xe = W.plane_end;
    }
    return G;
}

__device__ __forceinline__ bool excluded(uint4 m, int fast) {
    return grid_excluded((int)m.x) || (fast && (m.y & kFlagLarge));
}

// Per-axis cell coordinate (src/world.cpp:458-466), in grid G of world W.
__device__ __forceinline__ long long cell_of(const WorldP& W, const GridSel& G, double c, int axis) {
    if (W.dom.periodic) {
        long long k = (long long)floor((c + W.dom.half) / G.cell);
        long long m = G.nc[axis];
        return ((k % m) + m) % m;
    }
    return (long long)floor(c / G.cell);
}

// Compact sort key layout: a bijection of the reference's 21-bit-masked cell
// coordinates (src/world.cpp:467-470) onto as few bits as the occupied range
// needs, so the radix sort touches only varying digits.  In a batch the world
// index sits above the local key (`prefix`), so cells of different worlds
// never compare equal.
struct KeyLayout {
    int bits[3];
    long long base[3];
    long long span[3];   // occupied offsets are [0, span] per axis
    int total;
    unsigned long long prefix;
};

__device__ __forceinline__ KeyLayout world_layout(const WorldP& W, const GridSel& G, const long long* ext) {
    KeyLayout L;
    for (int ax = 0; ax < 3; ++ax) {
        if (W.dom.periodic) {
            const long long m = G.nc[ax];
            L.bits[ax] = (m > (1ll << 21)) ? 21 : bitlen_u64((unsigned long long)(m - 1));
            L.base[ax] = 0;
            L.span[ax] = m - 1;
        } else {
            const long long span = ext[3 + ax] - ext[ax];
            L.bits[ax] = (span >= (1ll << 21) || span < 0) ? 21 : bitlen_u64((unsigned long long)span);
            L.base[ax] = ext[ax];
            L.span[ax] = span;
        }
    }
    L.total = L.bits[0] + L.bits[1] + L.bits[2];
    L.prefix = 0;
    return L;
}

// Layout of world w's keys; local keys of every world use the low
// `local_bits` bits (the widest world's total).
__device__ __forceinline__ KeyLayout key_layout(const StepArgs& a, uint32_t w, const GridSel& G, int local_bits) {
    KeyLayout L = world_layout(a.wp[w], G, a.cext + 6 * (size_t)w);
    L.prefix = (unsigned long long)w << local_bits;
    return L;
}

__device__ __forceinline__ unsigned long long compact_key(const KeyLayout& L, long long cx, long long cy,
                                                          long long cz) {
    const unsigned long long M = 0x1FFFFFull;
    unsigned long long x = (unsigned long long)(cx - L.base[0]) & M;
    unsigned long long y = (unsigned long long)(cy - L.base[1]) & M;
    unsigned long long z = (unsigned long long)(cz - L.base[2]) & M;
    return L.prefix | x | (y << L.bits[0]) | (z << (L.bits[0] + L.bits[1]));
}

// Key of a neighbour cell.  A cell outside the occupied offset range holds no
// body; with fewer than 21 bits per axis its offset would not fit its field
// and would alias another cell, so it gets kNoCell, which matches nothing.
// (With 21 bits every offset fits, and aliasing modulo 2^21 is exactly the
// reference's masking.)
constexpr unsigned long long kNoCell = ~0ull;

__device__ __forceinline__ unsigned long long neighbour_key(const KeyLayout& L, long long cx, long long cy,
                                                            long long cz) {
    const long long c[3] = {cx, cy, cz};
    for (int ax = 0; ax < 3; ++ax) {
        if (L.bits[ax] >= 21) continue;
        const long long off = c[ax] - L.base[ax];
        if (off < 0 || off > L.span[ax]) return kNoCell;
    }
    return compact_key(L, cx, cy, cz);
}

__device__ __forceinline__ long long wrap_cell(const WorldP& W, const GridSel& G, long long c, int axis) {
    if (!W.dom.periodic) return c;
    const long long m = G.nc[axis];
    return ((c % m) + m) % m;
}

// The distinct neighbour keys of a cell (27 offsets; wrapping can alias them).
__device__ __forceinline__ int neighbour_keys(const WorldP& W, const GridSel& G, const KeyLayout& L, long long cx,
                                              long long cy, long long cz, unsigned long long* out) {
    int nk = 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                unsigned long long k = neighbour_key(L, wrap_cell(W, G, cx + dx, 0), wrap_cell(W, G, cy + dy, 1),
                                                     wrap_cell(W, G, cz + dz, 2));
                bool dup = false;
                for (int t = 0; t < nk; ++t) dup |= (out[t] == k);
                if (!dup) out[nk++] = k;
            }
    return nk;
}

__device__ __forceinline__ uint32_t lower_bound_u64(const unsigned long long* a, uint32_t lo, uint32_t hi,
                                                    unsigned long long k) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t upper_bound_u64(const unsigned long long* a, uint32_t lo, uint32_t hi,
                                                    unsigned long long k) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] <= k) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t k) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < k) lo = mid + 1; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t* a, uint32_t lo, uint32_t hi, uint32_t k) {
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] <= k) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------

__global__ void k_step_begin(Ctl* ctl, int sticky) {
    if (sticky && ctl->halt) {
        ctl->abort = 1;   // an earlier step of this batch aborted: skip the step
        return;
    }
    ctl->abort = 0;
    ctl->flags = 0;
    ctl->need_bits = 0;
    ctl->P = ctl->S = ctl->C = 0;
    ctl->P_ref = 0;
    ctl->islands = 0;
    ctl->max_island = 0;
    ctl->epa_cap_hits = 0;
    ctl->nbig = 0;
    for (int k = 0; k < 32; ++k) ctl->big_class[k] = ctl->big_fill[k] = 0;
    ctl->big_next = 0;
    ctl->nlong = 0;
    ctl->solve_timeout = 0;
    ctl->S_stage = 0;
}

__device__ __forceinline__ long long warp_min_ll(long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t < v ? t : v;
    }
    return v;
}
__device__ __forceinline__ long long warp_max_ll(long long v) {
    for (int o = 16; o > 0; o >>= 1) {
        long long t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    return v;
}

// World::integrate() (src/world.cpp:373-411) + pre-step snapshot + union-find reset.
__global__ void __launch_bounds__(kT) k_integrate(StepArgs a) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    if (d.ctl->abort) return;   // halted batch: the pre-step snapshot stays that of the aborted step
    const WorldP& W = a.wp[a.bw[i]];
    D4 p = d.pos[i], q4 = d.quat[i], v4 = d.vel[i], w4 = d.omg[i], f4 = d.frc[i], t4 = d.trq[i];
    d.s_pos[i] = p; d.s_quat[i] = q4; d.s_vel[i] = v4; d.s_omg[i] = w4; d.s_frc[i] = f4; d.s_trq[i] = t4;
    d.parent[i] = i;
    const uint4 m = d.meta[i];
    V3 x = v3of(p), v = v3of(v4), wv = v3of(w4), F = v3of(f4), T = v3of(t4);
    Q q = qof(q4);
    const double invM = p.w, dt = W.dt;
    if (m.y & NE_BODY_KINEMATIC) {
        x = x + v * dt;
        q = integrate_orientation(q, wv, dt);
    } else if (invM <= 0.0) {
    } else {
        const D4 I = d.inert[i], g = d.geom[i], mt = d.mat[i];
        const V3 invI = v3of(I);
        v = v + (W.g * g.z + F * invM) * dt;
        x = x + v * dt;
        V3 L = angular_momentum(q, invI, wv);
        L = L + T * dt;
        q = integrate_orientation(q, wv, dt);
        wv = apply_inv_inertia(q, invI, L);
        if (mt.z > 0.0) v = v * (1.0 / (1.0 + mt.z * dt));
        if (mt.w > 0.0) wv = wv * (1.0 / (1.0 + mt.w * dt));
    }
    F = mk(0.0, 0.0, 0.0);
    T = F;
    d.pos[i] = d4of(x, invM);
    d.quat[i] = d4ofq(q);
    d.vel[i] = d4of(v, 0.0);
    d.omg[i] = d4of(wv, 0.0);
    d.frc[i] = d4of(F, 0.0);
    d.trq[i] = d4of(T, 0.0);
    if (a.f32) {
        // FP32 working copies for the narrowphase and the solver.
        const D4 I = d.inert[i], g = d.geom[i], e = d.ext[i];
        d.f_v[i] = F4{(float)v.x, (float)v.y, (float)v.z, (float)invM};
        d.f_w[i] = F4{(float)wv.x, (float)wv.y, (float)wv.z, 0.0f};
        d.f_q[i] = F4{(float)q.w, (float)q.x, (float)q.y, (float)q.z};
        d.f_I[i] = F4{(float)I.x, (float)I.y, (float)I.z, (float)g.y};
        d.f_e[i] = F4{(float)e.x, (float)e.y, (float)e.z, (float)g.x};
    }
}

__global__ void __launch_bounds__(kT) k_ext_reset(StepArgs a) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) a.d.ctl->local_bits = 0;
    if (t >= a.nworlds) return;
    for (int ax = 0; ax < 3; ++ax) {
        a.cext[6 * (size_t)t + ax] = 0x7fffffffffffffffll;
        a.cext[6 * (size_t)t + 3 + ax] = (long long)0x8000000000000000ull;
    }
}

// Cell extents of each open/reflective world's grid bodies (one atomic per
// warp when the warp's bodies share a world).
__global__ void __launch_bounds__(kT) k_extents(StepArgs a, int fast) {
    if (a.d.ctl->abort) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < a.n;
    const uint32_t w = live ? a.bw[i] : 0xffffffffu;
    long long lo[3] = {0x7fffffffffffffffll, 0x7fffffffffffffffll, 0x7fffffffffffffffll};
    long long hi[3] = {(long long)0x8000000000000000ull, (long long)0x8000000000000000ull,
                       (long long)0x8000000000000000ull};
    bool track = false;
    if (live) {
        const WorldP& W = a.wp[w];
        const GridSel G = grid_sel(a, W, fast);
        if (!G.brute && !W.dom.periodic && !excluded(a.d.meta[i], fast)) {
            const D4 p = a.d.pos[i];
            const double c[3] = {p.x, p.y, p.z};
            for (int ax = 0; ax < 3; ++ax) lo[ax] = hi[ax] = cell_of(W, G, c[ax], ax);
            track = true;
        }
    }
    const uint32_t w0 = __shfl_sync(0xffffffffu, w, 0);
    if (__all_sync(0xffffffffu, w == w0)) {
        if (!__any_sync(0xffffffffu, track)) return;
        for (int ax = 0; ax < 3; ++ax) {
            long long mn = warp_min_ll(lo[ax]), mx = warp_max_ll(hi[ax]);
            if ((threadIdx.x & 31) == 0 && mn <= mx) {
                atomicMin(&a.cext[6 * (size_t)w0 + ax], mn);
                atomicMax(&a.cext[6 * (size_t)w0 + 3 + ax], mx);
            }
        }
    } else if (track) {
        for (int ax = 0; ax < 3; ++ax) {
            atomicMin(&a.cext[6 * (size_t)w + ax], lo[ax]);
            atomicMax(&a.cext[6 * (size_t)w + 3 + ax], hi[ax]);
        }
    }
}

// Key bits each world's grid needs; the widest decides the local key width.
__global__ void __launch_bounds__(kT) k_world_layout(StepArgs a, int fast) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= a.nworlds) return;
    const WorldP& W = a.wp[w];
    const GridSel G = grid_sel(a, W, fast);
    if (G.brute) return;
    const KeyLayout L = world_layout(W, G, a.cext + 6 * (size_t)w);
    atomicMax(&ctl->local_bits, (uint32_t)L.total);
}

// Sort keys of the grid cells; excluded bodies and bodies of brute-force
// worlds get a sentinel that sorts after every real key.
__global__ void __launch_bounds__(kT) k_cell_keys(StepArgs a, int fast) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lb = (int)ctl->local_bits;
    const int total = a.world_bits + lb;
    if (i == 0) {
        ctl->need_bits = max(ctl->need_bits, (uint32_t)(total + 1));
        if (total + 1 > a.key_bits) ctl->abort = 1;
    }
    if (i >= a.n) return;
    const uint32_t w = a.bw[i];
    const WorldP& W = a.wp[w];
    const GridSel G = grid_sel(a, W, fast);
    const D4 p = a.d.pos[i];
    unsigned long long k;
    if (G.brute || excluded(a.d.meta[i], fast)) {
        k = 1ull << total;
    } else {
        const KeyLayout L = key_layout(a, w, G, lb);
        k = compact_key(L, cell_of(W, G, p.x, 0), cell_of(W, G, p.y, 1), cell_of(W, G, p.z, 2));
    }
    a.d.key[0][i] = k;
    a.d.val[0][i] = i;
}

// Number of partners j > i of body i (the sorted unique pair list is the CSR
// of these partner lists).  Partners are always in body i's world.
__global__ void __launch_bounds__(kT) k_pair_count(StepArgs a, int kb, int fast) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    const uint32_t w = a.bw[i];
    const WorldP& W = a.wp[w];
    const GridSel G = grid_sel(a, W, fast);
    if (G.brute || excluded(d.meta[i], fast)) {
        d.bcnt[i] = W.end - 1 - i;
        return;
    }
    const KeyLayout L = key_layout(a, w, G, (int)ctl->local_bits);
    const D4 p = d.pos[i];
    unsigned long long nk[27];
    const int m = neighbour_keys(W, G, L, cell_of(W, G, p.x, 0), cell_of(W, G, p.y, 1), cell_of(W, G, p.z, 2), nk);
    const unsigned long long* keys = d.key[kb];
    const uint32_t* vals = d.val[kb];
    uint32_t cnt = 0;
    for (int t = 0; t < m; ++t) {
        uint32_t lo = lower_bound_u64(keys, 0, a.n, nk[t]);
        uint32_t hi = upper_bound_u64(keys, lo, a.n, nk[t]);
        if (lo == hi) continue;
        uint32_t s = upper_bound_u32(vals, lo, hi, i);
        cnt += hi - s;
    }
    cnt += G.xe - upper_bound_u32(G.xl, G.xb, G.xe, i);
    d.bcnt[i] = cnt;
}

// Candidate partners j > i of grid body i, as up to 28 sorted runs: one per
// distinct neighbour cell (its members with index > i) and, last, the world's
// excluded bodies > i.  Every lane of the warp calls this; the runs land in
// the warp's shared slots lo/len/ex (ex = exclusive offset of each run in the
// concatenated candidate sequence, ex[nr] = total).
struct Runs {
    uint32_t total;
    int nr;
    bool xl_last;      // the last run is the excluded list
};

__device__ __forceinline__ Runs warp_runs(const StepArgs& a, const WorldP& W, const GridSel& G, const KeyLayout& L,
                                          uint32_t i, const D4& p, int kb, uint32_t* lo_s, uint32_t* len_s,
                                          uint32_t* ex_s) {
    const int lane = threadIdx.x & 31;
    const long long cx = cell_of(W, G, p.x, 0), cy = cell_of(W, G, p.y, 1), cz = cell_of(W, G, p.z, 2);
    const unsigned long long* keys = a.d.key[kb];
    const uint32_t* vals = a.d.val[kb];
    // Lane t < 27 takes neighbour offset t (duplicates from wrap aliasing keep
    // their lowest lane); lane 27 takes the excluded list.
    uint32_t rlo = 0, rhi = 0;
    if (lane < 27) {
        const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
        unsigned long long k = neighbour_key(L, wrap_cell(W, G, cx + dx, 0), wrap_cell(W, G, cy + dy, 1),
                                             wrap_cell(W, G, cz + dz, 2));
        const uint32_t grp = __match_any_sync(0x07ffffffu, k);
        if (lane == __ffs(grp) - 1) {
            uint32_t lo = lower_bound_u64(keys, 0, a.n, k);
            uint32_t hi = upper_bound_u64(keys, lo, a.n, k);
            rlo = (lo < hi) ? upper_bound_u32(vals, lo, hi, i) : hi;
            rhi = hi;
        }
    } else if (lane == 27) {
        rlo = upper_bound_u32(G.xl, G.xb, G.xe, i);
        rhi = G.xe;
    }
    // Compact the non-empty runs into shared memory, in lane order.
    const uint32_t len = rhi - rlo;
    const uint32_t nonempty = __ballot_sync(0xffffffffu, len > 0);
    const int r = __popc(nonempty & ((1u << lane) - 1u));
    uint32_t incl = len;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    Runs R;
    R.total = __shfl_sync(0xffffffffu, incl, 31);
    R.nr = __popc(nonempty);
    R.xl_last = (nonempty >> 27) & 1u;
    if (len > 0) {
        lo_s[r] = rlo;
        len_s[r] = len;
        ex_s[r] = incl - len;
    }
    if (lane == 0) ex_s[R.nr] = R.total;
    __syncwarp();
    return R;
}

// Candidate number e of the concatenated runs: its body index, owning run and
// index within that run.
__device__ __forceinline__ uint32_t run_candidate(const Runs& R, const uint32_t* lo_s, const uint32_t* ex_s,
                                                  const uint32_t* vals, const uint32_t* xl, uint32_t e, int& own,
                                                  uint32_t& idx) {
    int lo = 0, hi = R.nr - 1;   // owning run: last r with ex[r] <= e
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ex_s[mid] <= e) lo = mid; else hi = mid - 1;
    }
    own = lo;
    idx = e - ex_s[own];
    const bool own_xl = R.xl_last && own == R.nr - 1;
    return own_xl ? xl[lo_s[own] + idx] : vals[lo_s[own] + idx];
}

// Writes body i's sorted partner list at its CSR offset (the reference-rule
// list of recorded steps).  One warp per body.  Each candidate's output rank is
// its index in its own run plus the number of smaller candidates in the other
// runs (all candidates are distinct bodies).
__global__ void __launch_bounds__(kT) k_pair_emit(StepArgs a, int kb, int fast, uint32_t* out_i, uint32_t* out_j,
                                                  const uint64_t* total_p, uint64_t cap) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    if (*total_p > cap) {
        if (threadIdx.x == 0 && blockIdx.x == 0) ctl->abort = 1;
        return;
    }
    __shared__ uint32_t s_lo[kT / 32][28], s_len[kT / 32][28], s_ex[kT / 32][29];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    const uint32_t w = a.bw[i];
    const WorldP& W = a.wp[w];
    const GridSel G = grid_sel(a, W, fast);
    const uint32_t base = d.boff[i];
    if (G.brute || excluded(d.meta[i], fast)) {
        const uint32_t cnt = W.end - 1 - i;
        for (uint32_t k = lane; k < cnt; k += 32) {
            out_i[base + k] = i;
            out_j[base + k] = i + 1 + k;
        }
        return;
    }
    const KeyLayout L = key_layout(a, w, G, (int)ctl->local_bits);
    const uint32_t* vals = d.val[kb];
    const Runs R = warp_runs(a, W, G, L, i, d.pos[i], kb, s_lo[wid], s_len[wid], s_ex[wid]);
    for (uint32_t e = lane; e < R.total; e += 32) {
        int own;
        uint32_t idx;
        const uint32_t x = run_candidate(R, s_lo[wid], s_ex[wid], vals, G.xl, e, own, idx);
        uint32_t rank = idx;
        for (int q = 0; q < R.nr; ++q) {
            if (q == own) continue;
            const uint32_t ql = s_lo[wid][q], qh = ql + s_len[wid][q];
            const uint32_t* src = (R.xl_last && q == R.nr - 1) ? G.xl : vals;
            rank += lower_bound_u32(src, ql, qh, x) - ql;
        }
        out_i[base + rank] = i;
        out_j[base + rank] = x;
    }
}

// Pair filters (src/world.cpp:513-516) and a conservative bounding-volume cull
// that only removes pairs the narrowphase provably reports as separated.
// CullA holds the first body's operands, loaded once per partner list.
struct CullA {
    V3 x;
    double invM, r;
    uint4 m;
    uint2 nr;
    Q q;
    V3 he;
    Domain dom;
};

__device__ __forceinline__ CullA cull_self(const StepArgs& a, uint32_t i) {
    const DevWorld& d = a.d;
    CullA A;
    const D4 p = d.pos[i];
    A.x = v3of(p);
    A.invM = p.w;
    A.r = d.inert[i].w;
    A.m = d.meta[i];
    A.nr = d.ncrng[i];
    A.q = qof(d.quat[i]);
    A.he = v3of(d.ext[i]);
    A.dom = a.wp[a.bw[i]].dom;
    return A;
}

__device__ __forceinline__ bool cull_keep(const DevWorld& d, const CullA& A, uint32_t j) {
    const D4 pb = d.pos[j];
    const uint4 mb = d.meta[j];
    if (A.invM + pb.w <= 0.0) return false;
    if (!((A.m.w & (1u << (mb.z & 31u))) && (mb.w & (1u << (A.m.z & 31u))))) return false;
    for (uint32_t k = 0; k < A.nr.y; ++k)
        if (d.nc[A.nr.x + k] == j) return false;
    if ((A.m.y | mb.y) & NE_BODY_SENSOR) return false;
    const int sa = (int)A.m.x, sb = (int)mb.x;
    if (sa == SH_PLANE && sb == SH_PLANE) return false;
    if (sa == SH_PLANE || sb == SH_PLANE) return true;
    // Bounding spheres about the centres (nearest image).
    const double rb = d.inert[j].w;
    const V3 dd = min_image(A.dom, mk(pb.x - A.x.x, pb.y - A.x.y, pb.z - A.x.z));
    const double r = (A.r + rb) * (1.0 + 1e-9) + 1e-9;
    if (norm2(dd) > r * r) return false;
    // Box vs bounding sphere: distance from the sphere centre to the box.
    if (sa == SH_BOX || sb == SH_BOX) {
        const bool boxA = (sa == SH_BOX);
        const double rs = boxA ? rb : A.r;
        const V3 rel = boxA ? dd : -dd;     // other centre relative to the box centre
        const Q qb = boxA ? A.q : qof(d.quat[j]);
        const V3 he = boxA ? A.he : v3of(d.ext[j]);
        const V3 l = inv_rotate(qb, rel);
        const double ex = fmax(fabs(l.x) - he.x, 0.0), ey = fmax(fabs(l.y) - he.y, 0.0),
                     ez = fmax(fabs(l.z) - he.z, 0.0);
        const double lim = rs * (1.0 + 1e-9) + 1e-9 * (1.0 + norm(he));
        if (ex * ex + ey * ey + ez * ez > lim * lim) return false;
    }
    return true;
}

// ---- internal grid: cell table, then one pass of filters + cull ------------

constexpr unsigned long long kHashEmpty = ~0ull;

__device__ __forceinline__ uint32_t cell_hash(unsigned long long k, uint32_t mask) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return (uint32_t)k & mask;
}

__global__ void __launch_bounds__(kT) k_hash_clear(StepArgs a) {
    if (a.d.ctl->abort) return;
    const uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h < a.d.hsize) a.d.hkey[h] = kHashEmpty;
}

// Run starts of the sorted cell keys (the run of sentinel keys included, so
// every run has an end), and each body's bounding sphere in sorted order, so
// the members of a cell are contiguous for the cull.
__global__ void __launch_bounds__(kT) k_cell_flags(StepArgs a, int kb) {
    if (a.d.ctl->abort) return;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const DevWorld& d = a.d;
    const unsigned long long* key = d.key[kb];
    d.cflag[k] = (k == 0 || key[k] != key[k - 1]) ? 1u : 0u;
    const uint32_t b = d.val[kb][k];
    const D4 p = d.pos[b];
    d.srec[k] = D4{p.x, p.y, p.z, d.inert[b].w};
}

// cstart of every run, cstart[runs] = n, and the hash entries of the real
// cells (keys below the sentinel 1 << total).
__global__ void __launch_bounds__(kT) k_cell_table(StepArgs a, int kb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const DevWorld& d = a.d;
    const uint32_t r = d.crun[k];
    if (k + 1 == a.n) d.cstart[r + d.cflag[k]] = a.n;
    if (!d.cflag[k]) return;
    d.cstart[r] = k;
    const unsigned long long key = d.key[kb][k];
    const int total = a.world_bits + (int)ctl->local_bits;
    if (key >= (1ull << total)) return;
    const uint32_t mask = d.hsize - 1;
    uint32_t h = cell_hash(key, mask);
    for (uint32_t probe = 0; probe < d.hsize; ++probe) {
        const unsigned long long prev = atomicCAS(&d.hkey[h], kHashEmpty, key);
        if (prev == kHashEmpty) {
            d.hval[h] = r;
            return;
        }
        h = (h + 1) & mask;
    }
}

// Sorted positions [lo, hi) of the bodies in cell `key` (empty if none).
__device__ __forceinline__ void cell_range(const DevWorld& d, unsigned long long key, uint32_t& lo, uint32_t& hi) {
    lo = hi = 0;
    if (key == kNoCell) return;
    const uint32_t mask = d.hsize - 1;
    uint32_t h = cell_hash(key, mask);
    for (uint32_t probe = 0; probe < d.hsize; ++probe) {
        const unsigned long long k = d.hkey[h];
        if (k == key) {
            const uint32_t r = d.hval[h];
            lo = d.cstart[r];
            hi = d.cstart[r + 1];
            return;
        }
        if (k == kHashEmpty) return;
        h = (h + 1) & mask;
    }
}

// warp_runs with the neighbour cells found through the cell table.
__device__ __forceinline__ Runs warp_runs_table(const StepArgs& a, const WorldP& W, const GridSel& G,
                                                const KeyLayout& L, uint32_t i, const D4& p, int kb,
                                                uint32_t* lo_s, uint32_t* len_s, uint32_t* ex_s) {
    const int lane = threadIdx.x & 31;
    const long long cx = cell_of(W, G, p.x, 0), cy = cell_of(W, G, p.y, 1), cz = cell_of(W, G, p.z, 2);
    const uint32_t* vals = a.d.val[kb];
    uint32_t rlo = 0, rhi = 0;
    if (lane < 27) {
        const int dx = lane / 9 - 1, dy = (lane / 3) % 3 - 1, dz = lane % 3 - 1;
        unsigned long long k = neighbour_key(L, wrap_cell(W, G, cx + dx, 0), wrap_cell(W, G, cy + dy, 1),
                                             wrap_cell(W, G, cz + dz, 2));
        const uint32_t grp = __match_any_sync(0x07ffffffu, k);
        if (lane == __ffs(grp) - 1) {
            uint32_t lo, hi;
            cell_range(a.d, k, lo, hi);
            rlo = (lo < hi) ? upper_bound_u32(vals, lo, hi, i) : hi;
            rhi = hi;
        }
    } else if (lane == 27) {
        rlo = upper_bound_u32(G.xl, G.xb, G.xe, i);
        rhi = G.xe;
    }
    const uint32_t len = rhi - rlo;
    const uint32_t nonempty = __ballot_sync(0xffffffffu, len > 0);
    const int r = __popc(nonempty & ((1u << lane) - 1u));
    uint32_t incl = len;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    Runs R;
    R.total = __shfl_sync(0xffffffffu, incl, 31);
    R.nr = __popc(nonempty);
    R.xl_last = (nonempty >> 27) & 1u;
    if (len > 0) {
        lo_s[r] = rlo;
        len_s[r] = len;
        ex_s[r] = incl - len;
    }
    if (lane == 0) ex_s[R.nr] = R.total;
    __syncwarp();
    return R;
}

// Surviving partners of every body (internal grid), in one pass: each
// candidate j > i of body i's partner list is tested once with the filters
// and the cull.  One warp per body.  A body's survivors (at most kSurvBuf;
// usually a handful) are ranked in shared memory and staged, ascending, at an
// offset reserved with one atomic per block; bcnt/bstage record count and
// offset.  A body with more survivors reserves its own space and writes them
// by a slower exact ranking.  ctl->P accumulates the candidates examined.
constexpr uint32_t kSurvBuf = 64;

// The bounding-sphere part of cull_keep for a grid candidate, from its
// sorted record (same arithmetic, so the same decision).
__device__ __forceinline__ bool sphere_pass(const CullA& A, const D4& s) {
    const V3 dd = min_image(A.dom, mk(s.x - A.x.x, s.y - A.x.y, s.z - A.x.z));
    const double r = (A.r + s.w) * (1.0 + 1e-9) + 1e-9;
    return !(norm2(dd) > r * r);
}

__global__ void __launch_bounds__(kT, 5) k_surv_gather(StepArgs a, int kb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    __shared__ uint32_t s_lo[kT / 32][28], s_len[kT / 32][28], s_ex[kT / 32][29];
    __shared__ uint32_t s_buf[kT / 32][kSurvBuf];
    __shared__ uint32_t s_cnt[kT / 32], s_cand[kT / 32];
    __shared__ uint32_t s_base;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const DevWorld& d = a.d;
    const uint32_t* vals = d.val[kb];
    uint32_t cnt = 0, cand = 0;
    bool grid = false;
    Runs R;
    R.total = 0; R.nr = 0; R.xl_last = false;
    CullA A;
    GridSel G;
    uint32_t wend = 0;
    bool split = false;
    if (i < a.n) {
        const uint32_t w = a.bw[i];
        const WorldP& W = a.wp[w];
        G = grid_sel(a, W, 1);
        A = cull_self(a, i);
        wend = W.end;
        if (G.brute || excluded(A.m, 1)) {
            cand = W.end - 1 - i;
            if (cand >= kLongRow) {
                uint32_t slot = 0;
                if (lane == 0) slot = atomicAdd(&ctl->nlong, 1u);
                slot = __shfl_sync(0xffffffffu, slot, 0);
                if (slot < kLongRows) {
                    if (lane == 0) d.lrow[slot] = i;
                    split = true;   // k_long_mask / k_long_place take this list
                }
            }
            for (uint32_t j0 = i + 1; !split && j0 < W.end; j0 += 32) {
                const uint32_t j = j0 + lane;
                const bool k = j < W.end && cull_keep(d, A, j);
                const uint32_t bal = __ballot_sync(0xffffffffu, k);
                const uint32_t slot = cnt + __popc(bal & lt);
                if (k && slot < kSurvBuf) s_buf[wid][slot] = j;
                cnt += __popc(bal);
            }
        } else {
            grid = true;
            const KeyLayout L = key_layout(a, w, G, (int)ctl->local_bits);
            R = warp_runs_table(a, W, G, L, i, d.pos[i], kb, s_lo[wid], s_len[wid], s_ex[wid]);
            cand = R.total;
            for (uint32_t e0 = 0; e0 < R.total; e0 += 32) {
                const uint32_t e = e0 + lane;
                uint32_t x = 0;
                bool k = false;
                if (e < R.total) {
                    int own;
                    uint32_t idx;
                    x = run_candidate(R, s_lo[wid], s_ex[wid], vals, G.xl, e, own, idx);
                    // Grid members (neither is a plane) fail most often on the
                    // bounding spheres: test those from the sorted records first.
                    const bool xl = R.xl_last && own == R.nr - 1;
                    k = (xl || sphere_pass(A, d.srec[s_lo[wid][own] + idx])) && cull_keep(d, A, x);
                }
                const uint32_t bal = __ballot_sync(0xffffffffu, k);
                const uint32_t slot = cnt + __popc(bal & lt);
                if (k && slot < kSurvBuf) s_buf[wid][slot] = x;
                cnt += __popc(bal);
            }
        }
    }
    const bool spill = cnt > kSurvBuf;
    if (lane == 0) {
        s_cnt[wid] = spill ? 0u : cnt;
        s_cand[wid] = cand;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        unsigned long long csum = 0;
        for (int k = 0; k < kT / 32; ++k) { tot += s_cnt[k]; csum += s_cand[k]; }
        s_base = tot ? (uint32_t)atomicAdd((unsigned long long*)&ctl->S_stage, (unsigned long long)tot) : 0u;
        if (csum) atomicAdd((unsigned long long*)&ctl->P, csum);
    }
    __syncthreads();
    if (i >= a.n) return;
    uint32_t off = s_base;
    for (int k = 0; k < wid; ++k) off += s_cnt[k];
    if (!spill) {
        for (uint32_t t = lane; t < cnt; t += 32) {
            const uint32_t x = s_buf[wid][t];
            uint32_t rank = t;   // brute-force and excluded lists are ascending already
            if (grid) {
                rank = 0;
                for (uint32_t u = 0; u < cnt; ++u) rank += (s_buf[wid][u] < x) ? 1u : 0u;
            }
            if ((uint64_t)off + rank < a.Scap) d.stage_j[off + rank] = x;
        }
    } else {
        if (lane == 0) off = (uint32_t)atomicAdd((unsigned long long*)&ctl->S_stage, (unsigned long long)cnt);
        off = __shfl_sync(0xffffffffu, off, 0);
        if (!grid) {
            uint32_t out = 0;
            for (uint32_t j0 = i + 1; j0 < wend && out < cnt; j0 += 32) {
                const uint32_t j = j0 + lane;
                const bool k = j < wend && cull_keep(d, A, j);
                const uint32_t bal = __ballot_sync(0xffffffffu, k);
                const uint32_t slot = out + __popc(bal & lt);
                if (k && slot < cnt && (uint64_t)off + slot < a.Scap) d.stage_j[off + slot] = j;
                out += __popc(bal);
            }
        } else {
            for (uint32_t e = lane; e < R.total; e += 32) {
                int own;
                uint32_t idx;
                const uint32_t x = run_candidate(R, s_lo[wid], s_ex[wid], vals, G.xl, e, own, idx);
                if (!cull_keep(d, A, x)) continue;
                uint32_t rank = 0;
                for (uint32_t u = 0; u < R.total; ++u) {
                    int o2;
                    uint32_t i2;
                    const uint32_t y = run_candidate(R, s_lo[wid], s_ex[wid], vals, G.xl, u, o2, i2);
                    if (y < x && cull_keep(d, A, y)) ++rank;
                }
                if (rank < cnt && (uint64_t)off + rank < a.Scap) d.stage_j[off + rank] = x;
            }
        }
    }
    if (lane == 0 && !split) {
        d.bcnt[i] = cnt;
        d.bstage[i] = off;
    }
}

// Long partner lists (every later body of the world) split over the warps of
// the whole grid: the lists' 32-candidate chunks are numbered through in slot
// order, and each warp takes every nwarps-th chunk and writes its keep bits
// (cull_keep, the test of the one-warp walk) as one mask word.
__global__ void __launch_bounds__(kT) k_long_mask(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t nl = min(ctl->nlong, kLongRows);
    if (nl == 0) return;
    __shared__ uint32_t s_i[kLongRows], s_end[kLongRows], s_pre[kLongRows + 1];
    const DevWorld& d = a.d;
    if (threadIdx.x < nl) {
        const uint32_t i = d.lrow[threadIdx.x];
        s_i[threadIdx.x] = i;
        s_end[threadIdx.x] = a.wp[a.bw[i]].end;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t k = 0; k < nl; ++k) {
            s_pre[k] = acc;
            acc += (s_end[k] - 1 - s_i[k] + 31) / 32;
        }
        s_pre[nl] = acc;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t g = warp; g < s_pre[nl]; g += nwarps) {
        uint32_t lo = 0, hi = nl - 1;   // the slot whose chunks hold g
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (s_pre[mid] <= g) lo = mid; else hi = mid - 1;
        }
        const uint32_t i = s_i[lo], wend = s_end[lo], c = g - s_pre[lo];
        const CullA A = cull_self(a, i);
        const uint32_t j = i + 1 + c * 32 + lane;
        const bool k = j < wend && cull_keep(d, A, j);
        const uint32_t bal = __ballot_sync(0xffffffffu, k);
        if (lane == 0) d.lmask[(size_t)lo * d.lwords + c] = bal;
    }
}

// The survivors of each long list, ascending, at one staging reservation:
// one block per list; a block-wide scan of the mask words' bit counts places
// every survivor.  Sets the list's bcnt / bstage like k_surv_gather.
constexpr int kPlaceT = 512;
__global__ void __launch_bounds__(kPlaceT) k_long_place(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t slot = blockIdx.x;
    if (slot >= min(ctl->nlong, kLongRows)) return;
    __shared__ uint32_t s_w[kPlaceT / 32];
    __shared__ uint32_t s_base, s_tile;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const DevWorld& d = a.d;
    const uint32_t i = d.lrow[slot];
    const uint32_t wend = a.wp[a.bw[i]].end;
    const uint32_t nw = (wend - 1 - i + 31) / 32;
    const uint32_t* mask = d.lmask + (size_t)slot * d.lwords;
    uint32_t cnt = 0;
    for (uint32_t c = threadIdx.x; c < nw; c += kPlaceT) cnt += __popc(mask[c]);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0) s_w[wid] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int k = 0; k < kPlaceT / 32; ++k) tot += s_w[k];
        const uint32_t off = tot ? (uint32_t)atomicAdd((unsigned long long*)&ctl->S_stage, (unsigned long long)tot) : 0u;
        d.bcnt[i] = tot;
        d.bstage[i] = off;
        s_base = off;
        s_tile = 0;
    }
    __syncthreads();
    for (uint32_t c0 = 0; c0 < nw; c0 += kPlaceT) {
        const uint32_t c = c0 + threadIdx.x;
        const uint32_t m = c < nw ? mask[c] : 0u;
        const uint32_t pc = __popc(m);
        uint32_t incl = pc;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_w[wid] = incl;
        __syncthreads();
        uint32_t before = s_tile;
        for (int k = 0; k < wid; ++k) before += s_w[k];
        uint32_t pos = s_base + before + incl - pc;
        for (uint32_t b = m; b; b &= b - 1u) {
            const uint32_t j = i + 1 + c * 32 + (uint32_t)__ffs(b) - 1u;
            if ((uint64_t)pos < a.Scap) d.stage_j[pos] = j;
            ++pos;
        }
        __syncthreads();
        if (threadIdx.x == kPlaceT - 1) s_tile = before + incl;
        __syncthreads();
    }
}

// Staged partner lists -> the CSR survivor list in body order, which is the
// reference's sorted pair list (src/world.cpp:496-499) with culled pairs left
// out.  One warp per body.
__global__ void __launch_bounds__(kT) k_surv_place(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    if (ctl->S > a.Scap) {
        if (threadIdx.x == 0 && blockIdx.x == 0) ctl->abort = 1;
        return;
    }
    const int lane = threadIdx.x & 31;
    const uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    const uint32_t cnt = d.bcnt[i];
    if (cnt == 0) return;
    const uint32_t src = d.bstage[i], dst = d.boff[i];
    for (uint32_t t = lane; t < cnt; t += 32) {
        d.si[dst + t] = i;
        d.sj[dst + t] = d.stage_j[src + t];
    }
}

// ---- narrowphase order -------------------------------------------------------
// In worlds that mix shapes, neighbouring pairs take different narrowphase
// paths (the analytic early returns of detect.hpp:33-77, or GJK/EPA with
// different support functions), and a warp waits for its slowest lane.  There
// the survivors are visited grouped by shape pair: a stable one-pass radix sort
// on the pair's shape code keeps pair order inside each group.  Every pair
// still writes its own slot, so the order changes no result.
__device__ __forceinline__ uint32_t shape_pair_code(int sa, int sb) {
    const int lo = sa < sb ? sa : sb, hi = sa < sb ? sb : sa;
    return (uint32_t)(lo * 8 + hi);   // 0..63
}

// Keys (ccnt, free until the narrowphase) and identity values (stage_j,
// free after the placement) for the sort into sperm.
__global__ void __launch_bounds__(kT) k_pair_class(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ctl->S) return;
    const DevWorld& d = a.d;
    d.ccnt[s] = shape_pair_code((int)d.meta[d.si[s]].x, (int)d.meta[d.sj[s]].x);
    d.stage_j[s] = (uint32_t)s;
}

__device__ __forceinline__ uint64_t narrow_slot(const StepArgs& a, uint64_t t) {
    return a.class_sort ? (uint64_t)a.d.sperm[t] : t;
}

// ---- triangle meshes and compounds (src/world.cpp:53-121) --------------------
// A pair with a mesh or a compound can have any number of contacts: the
// narrowphase counts them, and once the scan has placed every pair,
// k_narrowphase_ext computes them again and writes them at their constraint
// index (ext_cn / ext_cp).  Both passes run the same arithmetic, so they agree.

__device__ __forceinline__ bool is_ext_shape(int s) { return s == SH_MESH || s == SH_COMPOUND; }

// A compound's child as a body of its own (compoundChildWorld, src/body.hpp:358-366).
__device__ __forceinline__ BodyG child_world(const DevWorld& d, const BodyG& parent, uint32_t k) {
    const D4 c0 = d.child[4 * k], c1 = d.child[4 * k + 1], c2 = d.child[4 * k + 2], c3 = d.child[4 * k + 3];
    BodyG c;
    c.x = parent.x + rotate(parent.q, mk(c0.x, c0.y, c0.z));
    c.q = qmul(parent.q, qof(c1));
    c.he = mk(c2.z, c2.w, c3.x);
    c.radius = c2.x;
    c.half_height = c2.y;
    c.verts = nullptr;
    c.nverts = 0;
    c.shape = (int)c0.w;
    return c;
}

// Sink for the contacts of one pair: counts them, and writes them (normal
// b -> a, flipped when `flip`) when `cn` is set, up to `cap`.
struct ExtOut {
    D4 *cn, *cp;
    uint32_t cap, n;
    bool flip;
    __device__ __forceinline__ void add(const Contact& c) {
        if (cn && n < cap) {
            const V3 nrm = flip ? -c.normal : c.normal;
            cn[n] = d4of(nrm, c.overlap);
            cp[n] = d4of(c.point, 0.0);
        }
        ++n;
    }
};

// meshContacts (src/world.cpp:56-85): every triangle of the mesh whose AABB
// meets the other body's bounding cube (BVH walk of src/mesh.hpp:44-57, in
// its order), as a 1e-3-thick prism through the narrowphase; normals point
// mesh -> other.
__device__ void mesh_contacts(const DevWorld& d, const BodyG& other, double other_bound, const BodyG& mb,
                              uint32_t mesh, const Domain& dom, EpaScratch& S, int& fl, ExtOut& out) {
    const uint4 tab = d.mesh_tab[mesh];
    if (tab.x == 0xffffffffu) return;
    const V3 rel = min_image(dom, other.x - mb.x);
    const V3 cl = inv_rotate(mb.q, rel);
    const double rr = other_bound + 0.05;
    const V3 lo = cl - mk(rr, rr, rr), hi = cl + mk(rr, rr, rr);
    const double thick = 1e-3;
    D4 pv[6];
    BodyG tri;
    tri.x = mk(0.0, 0.0, 0.0);
    tri.q = mkq(1.0, 0.0, 0.0, 0.0);
    tri.he = mk(0.0, 0.0, 0.0);
    tri.radius = 1.0;
    tri.half_height = 0.0;
    tri.verts = pv;
    tri.nverts = 6;
    tri.shape = SH_CONVEX;
    int stack[64];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int ni = stack[--sp];
        const D4 nl = d.mnode_lo[tab.x + ni], nh = d.mnode_hi[tab.x + ni];
        if (lo.x > nh.x || hi.x < nl.x || lo.y > nh.y || hi.y < nl.y || lo.z > nh.z || hi.z < nl.z) continue;
        const int4 nd = d.mnode[tab.x + ni];
        if (nd.x >= 0) {
            if (sp < 62) {
                stack[sp++] = nd.x;
                stack[sp++] = nd.y;
            }
            continue;
        }
        for (int t = 0; t < nd.w; ++t) {
            const int ti = d.morder[tab.y + nd.z + t];
            const int4 tv = d.mtri[tab.z + ti];
            const D4 a0 = d.mvert[tab.w + tv.x], a1 = d.mvert[tab.w + tv.y], a2 = d.mvert[tab.w + tv.z];
            const V3 w0 = mb.x + rotate(mb.q, mk(a0.x, a0.y, a0.z));
            const V3 w1 = mb.x + rotate(mb.q, mk(a1.x, a1.y, a1.z));
            const V3 w2 = mb.x + rotate(mb.q, mk(a2.x, a2.y, a2.z));
            V3 n = cross(w1 - w0, w2 - w0);
            const double len = norm(n);
            if (len < 1e-12) continue;   // degenerate triangle
            n = n / len;
            pv[0] = d4of(w0 + n * thick, 0.0);
            pv[1] = d4of(w1 + n * thick, 0.0);
            pv[2] = d4of(w2 + n * thick, 0.0);
            pv[3] = d4of(w0 - n * thick, 0.0);
            pv[4] = d4of(w1 - n * thick, 0.0);
            pv[5] = d4of(w2 - n * thick, 0.0);
            const Contact c = detect_contact(other, tri, dom, S, fl);   // normal tri -> other
            if (c.hit) out.add(c);
        }
    }
}

// gatherContacts (src/world.cpp:88-121) for a pair with a mesh or a compound.
__device__ void ext_contacts(const DevWorld& d, uint32_t i, uint32_t j, const BodyG& A, const BodyG& B,
                             const Domain& dom, EpaScratch& S, int& fl, ExtOut& out) {
    if (B.shape == SH_MESH) {
        out.flip = false;
        mesh_contacts(d, A, d.inert[i].w, B, d.vrng[j].x, dom, S, fl, out);   // mesh(b) -> a
        return;
    }
    if (A.shape == SH_MESH) {
        out.flip = true;                                                     // mesh(a) -> b, reported b -> a
        mesh_contacts(d, B, d.inert[j].w, A, d.vrng[i].x, dom, S, fl, out);
        return;
    }
    out.flip = false;
    const uint2 ra = d.vrng[i], rb = d.vrng[j];
    if (A.shape == SH_COMPOUND && B.shape == SH_COMPOUND) {
        for (uint32_t ka = ra.x; ka < ra.x + ra.y; ++ka) {
            const BodyG ba = child_world(d, A, ka);
            for (uint32_t kb = rb.x; kb < rb.x + rb.y; ++kb) {
                const BodyG bb = child_world(d, B, kb);
                const Contact c = detect_contact(ba, bb, dom, S, fl);
                if (c.hit) out.add(c);
            }
        }
    } else if (A.shape == SH_COMPOUND) {
        for (uint32_t ka = ra.x; ka < ra.x + ra.y; ++ka) {
            const Contact c = detect_contact(child_world(d, A, ka), B, dom, S, fl);
            if (c.hit) out.add(c);
        }
    } else {
        for (uint32_t kb = rb.x; kb < rb.x + rb.y; ++kb) {
            const Contact c = detect_contact(A, child_world(d, B, kb), dom, S, fl);
            if (c.hit) out.add(c);
        }
    }
}

// Contact counts of the mesh and compound pairs alone (the FP32 form, whose
// narrowphase leaves those pairs to the FP64 passes).
__global__ void __launch_bounds__(128) k_narrowphase_ext_count(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ctl->S) return;
    const DevWorld& d = a.d;
    const uint32_t i = d.si[s], j = d.sj[s];
    if (!is_ext_shape((int)d.meta[i].x) && !is_ext_shape((int)d.meta[j].x)) return;
    const BodyG A = load_geom(d, i), B = load_geom(d, j);
    EpaScratch S;
    int fl = 0;
    ExtOut out{nullptr, nullptr, 0, 0, false};
    ext_contacts(d, i, j, A, B, a.wp[a.bw[i]].dom, S, fl, out);
    d.ccnt[s] = out.n;
    if (fl & 1) atomicOr(&ctl->flags, 1u);
    if (fl & 2) atomicAdd((unsigned long long*)&ctl->epa_cap_hits, 1ull);
}

// Second pass over the mesh and compound pairs: their contacts at their
// constraint index.
__global__ void __launch_bounds__(128) k_narrowphase_ext(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    if (ctl->C > a.Ccap) return;   // k_constraint_build raises the abort
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= ctl->S) return;
    const DevWorld& d = a.d;
    const uint32_t cnt = d.ccnt[s];
    if (cnt == 0) return;
    const uint32_t i = d.si[s], j = d.sj[s];
    if (!is_ext_shape((int)d.meta[i].x) && !is_ext_shape((int)d.meta[j].x)) return;
    const BodyG A = load_geom(d, i), B = load_geom(d, j);
    EpaScratch S;
    int fl = 0;
    const uint32_t c0 = d.coff[s];
    ExtOut out{d.ext_cn + c0, d.ext_cp + c0, cnt, 0, false};
    ext_contacts(d, i, j, A, B, a.wp[a.bw[i]].dom, S, fl, out);
}

// gatherContacts() for one surviving pair (src/world.cpp:122-129).
__global__ void __launch_bounds__(128) k_narrowphase(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctl->S) return;
    const uint64_t s = narrow_slot(a, t);
    const DevWorld& d = a.d;
    const uint32_t i = d.si[s], j = d.sj[s];
    const BodyG A = load_geom(d, i), B = load_geom(d, j);
    EpaScratch S;
    int fl = 0;
    const Domain dom = a.wp[a.bw[i]].dom;
    if (is_ext_shape(A.shape) || is_ext_shape(B.shape)) {
        ExtOut out{nullptr, nullptr, 0, 0, false};
        ext_contacts(d, i, j, A, B, dom, S, fl, out);
        d.ccnt[s] = out.n;
        if (fl & 1) atomicOr(&ctl->flags, 1u);
        if (fl & 2) atomicAdd((unsigned long long*)&ctl->epa_cap_hits, 1ull);
        return;
    }
    Contact c = detect_contact(A, B, dom, S, fl);
    uint32_t cnt = 0;
    if (c.hit) {
        if (A.shape == SH_BOX && B.shape == SH_BOX) {
            Manifold m = box_box_manifold(A, B, c.normal, dom, fl);
            for (int k = 0; k < m.count; ++k) {
                d.cn[4 * s + k] = d4of(c.normal, m.depth[k]);
                d.cp[4 * s + k] = d4of(m.point[k], 0.0);
            }
            cnt = (uint32_t)m.count;
        }
        if (cnt == 0) {
            d.cn[4 * s] = d4of(c.normal, c.overlap);
            d.cp[4 * s] = d4of(c.point, 0.0);
            cnt = 1;
        }
    }
    d.ccnt[s] = cnt;
    if (fl & 1) atomicOr(&ctl->flags, 1u);
    if (fl & 2) atomicAdd((unsigned long long*)&ctl->epa_cap_hits, 1ull);
}

__device__ __forceinline__ double combine_mat(int mode, double x, double y) {
    switch (mode) {
        case NE_COMBINE_AVERAGE: return 0.5 * (x + y);
        case NE_COMBINE_MIN: return x < y ? x : y;
        case NE_COMBINE_MAX: return x > y ? x : y;
        case NE_COMBINE_MULTIPLY: return x * y;
        case NE_COMBINE_GEOMETRIC_MEAN: return sqrt((x > 0 ? x : 0) * (y > 0 ? y : 0));
    }
    return 0.5 * (x + y);
}

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
    volatile uint32_t* p = parent;
    while (true) {
        uint32_t px = p[x];
        if (px == x) return x;
        uint32_t gp = p[px];
        if (gp != px) p[x] = gp;   // path halving; gp is an ancestor, so the race is benign
        x = px;
    }
}

// Link the components of a and b; the root is always the smaller index, so
// every component's root is its minimum body index.
__device__ __forceinline__ void uf_union(uint32_t* parent, uint32_t a, uint32_t b) {
    while (true) {
        a = uf_find(parent, a);
        b = uf_find(parent, b);
        if (a == b) return;
        if (a > b) { uint32_t t = a; a = b; b = t; }
        uint32_t old = atomicCAS(&parent[b], b, a);
        if (old == b) return;
        b = old;
    }
}

// effMass(a, b, rA, rB, u) (src/contact.hpp:28-33) from the body arrays.
__device__ __forceinline__ double eff_mass_at(const DevWorld& d, uint32_t i, uint32_t j, const V3& ra, const V3& rb,
                                              const V3& u) {
    const Q qa = qof(d.quat[i]), qb = qof(d.quat[j]);
    const V3 ia = v3of(d.inert[i]), ibv = v3of(d.inert[j]);
    V3 angA = cross(apply_inv_inertia(qa, ia, cross(ra, u)), ra);
    V3 angB = cross(apply_inv_inertia(qb, ibv, cross(rb, u)), rb);
    return d.pos[i].w + d.pos[j].w + dot(angA + angB, u);
}

// Contact constraints of one surviving pair (src/world.cpp:518-553): lever
// arms, restitution bias from the pre-solve velocities, combined material,
// warm-start impulse looked up in the previous step's sorted cache.
__global__ void __launch_bounds__(kT) k_constraint_build(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ctl->C > a.Ccap) {
        if (s == 0) ctl->abort = 1;
        return;
    }
    if (s >= ctl->S) return;
    const DevWorld& d = a.d;
    const uint32_t cnt = d.ccnt[s];
    if (cnt == 0) return;
    const uint32_t i = d.si[s], j = d.sj[s];
    const D4 pa = d.pos[i], pb = d.pos[j];
    const V3 xa = v3of(pa), xb = v3of(pb);
    const V3 va = v3of(d.vel[i]), vb = v3of(d.vel[j]), wa = v3of(d.omg[i]), wb = v3of(d.omg[j]);
    const D4 ma = d.mat[i], mb = d.mat[j];
    const WorldP& W = a.wp[a.bw[i]];
    const double ea = ma.y < 0 ? W.restitution : ma.y, eb = mb.y < 0 ? W.restitution : mb.y;
    const double fa = ma.x < 0 ? W.friction : ma.x, fb = mb.x < 0 ? W.friction : mb.x;
    const double e = combine_mat(W.rcomb, ea, eb);
    const double mu = combine_mat(W.fcomb, fa, fb);
    const uint32_t fla = d.meta[i].y, flb = d.meta[j].y;
    if ((fla & kFlagMutable) && (flb & kFlagMutable)) uf_union(d.parent, i, j);
    const unsigned long long key = ((unsigned long long)i << 32) | (unsigned long long)j;
    const uint32_t c0 = d.coff[s];
    const uint32_t ws = ctl->wsel;
    const uint32_t wn = ctl->wcount[ws];
    uint32_t widx = 0;
    if (a.warm) widx = lower_bound_u64(d.wkey[ws], 0, wn, key);
    const bool ext = is_ext_shape((int)d.meta[i].x) || is_ext_shape((int)d.meta[j].x);
    for (uint32_t k = 0; k < cnt; ++k) {
        const uint32_t c = c0 + k;
        const D4 cn = ext ? d.ext_cn[c] : d.cn[4 * s + k];
        const V3 n = v3of(cn), pt = v3of(ext ? d.ext_cp[c] : d.cp[4 * s + k]);
        const V3 rA = min_image(W.dom, pt - xa);
        const V3 rB = min_image(W.dom, pt - xb);
        const V3 vc = (va + cross(wa, rA)) - (vb + cross(wb, rB));
        const double vn = dot(vc, n);
        const double restBias = (vn < -0.5) ? -e * vn : 0.0;
        double nImp = 0.0;
        if (a.warm && widx + k < wn && d.wkey[ws][widx + k] == key) nImp = d.wimp[ws][widx + k];
        d.ci[c] = i;
        d.cj[c] = j;
        d.cslot[c] = k;
        d.con_n[c] = cn;
        d.con_p[c] = d4of(pt, 0.0);
        d.con_imp[c] = make_double2(nImp, 0.0);
        const double Kn = eff_mass_at(d, i, j, rA, rB, n);
        if (a.f32) {
            // FP32 solver records (built from FP64 operands, then rounded).
            d.f_n[c] = F4{(float)n.x, (float)n.y, (float)n.z, (float)cn.w};
            d.f_ra[c] = F4{(float)rA.x, (float)rA.y, (float)rA.z, (float)restBias};
            d.f_rb[c] = F4{(float)rB.x, (float)rB.y, (float)rB.z, (float)mu};
            d.f_kn[c] = (float)Kn;
        } else {
            d.con_ra[c] = d4of(rA, restBias);
            d.con_rb[c] = d4of(rB, mu);
            d.con_kn[c] = Kn;
        }
        d.wkey[ws ^ 1][c] = key;
    }
}

// Island label of every constraint (root of its first mutable body) and the
// identity order.  Also publishes 2C, the rank-entry count.
__global__ void __launch_bounds__(kT) k_island_label(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t C = ctl->C;
    if (c == 0) ctl->C2 = 2 * C;
    if (c >= C) return;
    const DevWorld& d = a.d;
    const uint32_t i = d.ci[c], j = d.cj[c];
    d.ilab[0][c] = (d.meta[i].y & kFlagMutable) ? uf_find(d.parent, i) : uf_find(d.parent, j);
    d.iord[0][c] = (uint32_t)c;
}

__global__ void __launch_bounds__(kT) k_island_mark(StepArgs a, int ib) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ctl->C) return;
    const uint32_t* lab = a.d.ilab[ib];
    a.d.iflag[k] = (k == 0 || lab[k] != lab[k - 1]) ? 1u : 0u;
}

// Island segments.
__global__ void __launch_bounds__(kT) k_island_start(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t C = ctl->C;
    if (k == 0) {
        ctl->islands = ctl->scan_total;
        a.d.istart[ctl->scan_total] = (uint32_t)C;
    }
    if (k < C && a.d.iflag[k]) a.d.istart[a.d.ioff[k]] = (uint32_t)k;
}

// Per-body rank entries: for every contact position p (island order) and each
// mutable endpoint, key = body, value = 2p + side.  Immovable sides get key n
// and sort last.
__global__ void __launch_bounds__(kT) k_rank_entries(StepArgs a, int ib) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ctl->C) return;
    const DevWorld& d = a.d;
    uint32_t ka = a.n, kb = a.n;
    {
        const uint32_t c = d.iord[ib][p];
        const uint32_t i = d.ci[c], j = d.cj[c];
        if (d.meta[i].y & kFlagMutable) ka = i;
        if (d.meta[j].y & kFlagMutable) kb = j;
    }
    d.rkey[0][2 * p] = ka;
    d.rval[0][2 * p] = (uint32_t)(2 * p);
    d.rkey[0][2 * p + 1] = kb;
    d.rval[0][2 * p + 1] = (uint32_t)(2 * p + 1);
}

// After the stable sort by body: rank = index within the body's run, the run
// start and length are the body's first entry and contact count.
__global__ void __launch_bounds__(kT) k_rank_write(StepArgs a, int rb) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t E = ctl->C2;
    if (e >= E) return;
    const DevWorld& d = a.d;
    const uint32_t* key = d.rkey[rb];
    const uint32_t body = key[e];
    if (body >= a.n) return;
    const uint32_t v = d.rval[rb][e];
    uint32_t lo = 0, hi = (uint32_t)e;   // run start: first index with this key
    while (lo < hi) {
        uint32_t mid = lo + ((hi - lo) >> 1);
        if (key[mid] < body) lo = mid + 1; else hi = mid;
    }
    d.crank[v] = (uint32_t)e - lo;
    if (e == lo) d.bstart[body] = lo;
    if (e + 1 == E || key[e + 1] != body) d.bdeg[body] = (uint32_t)e - lo + 1;
}

struct BodyS {
    V3 v, w;
    Q q;
    V3 invI;
    double invM;
    bool mut;
};

// Mutable solver state (velocities, positions, impulses) goes through
// solve::ld_state/st_state: plain for one-thread islands, L2-coherent for the
// team solver, whose consecutive updates of a body may run on different SMs.
template <bool C>
__device__ __forceinline__ BodyS load_solver_body(const DevWorld& d, uint32_t i) {
    BodyS b;
    b.v = v3of(solve::ld_state<C>(d.vel + i));
    b.w = v3of(solve::ld_state<C>(d.omg + i));
    b.q = qof(d.quat[i]);
    const D4 I = d.inert[i];
    b.invI = v3of(I);
    b.invM = d.pos[i].w;   // constant (the correction rewrites pos with the same w)
    b.mut = (d.meta[i].y & kFlagMutable) != 0;
    return b;
}

// effMass (src/contact.hpp:28-33).
__device__ __forceinline__ double eff_mass(const BodyS& A, const BodyS& B, const V3& ra, const V3& rb,
                                           const V3& u) {
    V3 angA = cross(apply_inv_inertia(A.q, A.invI, cross(ra, u)), ra);
    V3 angB = cross(apply_inv_inertia(B.q, B.invI, cross(rb, u)), rb);
    return A.invM + B.invM + dot(angA + angB, u);
}

__device__ __forceinline__ void apply_pair_impulse(BodyS& A, BodyS& B, const V3& ra, const V3& rb, const V3& J) {
    A.v = A.v + J * A.invM;
    A.w = A.w + apply_inv_inertia(A.q, A.invI, cross(ra, J));
    B.v = B.v - J * B.invM;
    B.w = B.w - apply_inv_inertia(B.q, B.invI, cross(rb, J));
}

template <bool C>
__device__ __forceinline__ void store_solver_body(const DevWorld& d, uint32_t i, const BodyS& b) {
    if (!b.mut) return;   // immovable: +-0 updates leave it unchanged; never written (shared by islands)
    solve::st_state<C>(d.vel + i, d4of(b.v, 0.0));
    solve::st_state<C>(d.omg + i, d4of(b.w, 0.0));
}

// The arithmetic of the three kinds of update on operands already loaded.
// Warm-start application of one contact (src/world.cpp:560-567).
__device__ __forceinline__ void warm_math(BodyS& A, BodyS& B, const D4& cn, const D4& ra4, const D4& rb4,
                                          double nImp) {
    apply_pair_impulse(A, B, v3of(ra4), v3of(rb4), v3of(cn) * nImp);
}

// One sequential-impulse update of one contact (src/world.cpp:575-610).  Kn
// is the effMass along n computed once at constraint build: the reference
// recomputes it every sweep from the same (unchanged) operands, so the value
// is identical.
__device__ __forceinline__ void sweep_math(BodyS& A, BodyS& B, const D4& cn, const D4& ra4, const D4& rb4,
                                           double Kn, double2& imp) {
    const V3 n = v3of(cn), rA = v3of(ra4), rB = v3of(rb4);
    const double restBias = ra4.w, mu = rb4.w;
    const V3 vc = (A.v + cross(A.w, rA)) - (B.v + cross(B.w, rB));
    const double vn = dot(vc, n);
    if (Kn > 1e-18) {
        double dj = (restBias - vn) / Kn;
        const double old = imp.x;
        imp.x = (old + dj > 0.0) ? old + dj : 0.0;
        dj = imp.x - old;
        apply_pair_impulse(A, B, rA, rB, n * dj);
    }
    if (mu > 0.0 && imp.x > 0.0) {
        const V3 vc2 = (A.v + cross(A.w, rA)) - (B.v + cross(B.w, rB));
        const V3 vt = vc2 - n * dot(vc2, n);
        const double vtl = norm(vt);
        if (vtl > 1e-12) {
            const V3 tg = vt / vtl;
            const double Kt = eff_mass(A, B, rA, rB, tg);
            if (Kt > 1e-18) {
                double djt = -vtl / Kt;
                const double maxF = mu * imp.x;
                const double old = imp.y;
                const double sum = old + djt;
                imp.y = (sum < -maxF) ? -maxF : (sum > maxF ? maxF : sum);
                djt = imp.y - old;
                apply_pair_impulse(A, B, rA, rB, tg * djt);
            }
        }
    }
}

// correctPenetration (src/contact.hpp:78-85): the position change of each
// body (false = no change).
__device__ __forceinline__ bool correct_math(const D4& pa, const D4& pb, const D4& cn, double beta, D4& na,
                                             D4& nb) {
    const double invSum = pa.w + pb.w;
    const double overlap = cn.w;
    if (invSum <= 0.0 || overlap <= 0.0) return false;
    const V3 corr = v3of(cn) * (beta * overlap / invSum);
    na = d4of(v3of(pa) + corr * pa.w, pa.w);
    nb = d4of(v3of(pb) - corr * pb.w, pb.w);
    return true;
}

template <bool C>
struct ItemsF64 {
    static __device__ __forceinline__ void warm(const DevWorld& d, uint32_t c) {
        const double nImp = solve::ld_state<C>(d.con_imp + c).x;
        if (nImp == 0.0) return;
        const uint32_t i = d.ci[c], j = d.cj[c];
        BodyS A = load_solver_body<C>(d, i), B = load_solver_body<C>(d, j);
        warm_math(A, B, d.con_n[c], d.con_ra[c], d.con_rb[c], nImp);
        store_solver_body<C>(d, i, A);
        store_solver_body<C>(d, j, B);
    }

    static __device__ __forceinline__ void sweep(const DevWorld& d, uint32_t c) {
        const uint32_t i = d.ci[c], j = d.cj[c];
        BodyS A = load_solver_body<C>(d, i), B = load_solver_body<C>(d, j);
        double2 imp = solve::ld_state<C>(d.con_imp + c);
        sweep_math(A, B, d.con_n[c], d.con_ra[c], d.con_rb[c], d.con_kn[c], imp);
        solve::st_state<C>(d.con_imp + c, imp);
        store_solver_body<C>(d, i, A);
        store_solver_body<C>(d, j, B);
    }

    // correctPenetration and the warm-cache store value.
    static __device__ __forceinline__ void correct(const DevWorld& d, uint32_t c, double beta, double* wimp_out) {
        const uint32_t i = d.ci[c], j = d.cj[c];
        const D4 pa = solve::ld_state<C>(d.pos + i), pb = solve::ld_state<C>(d.pos + j);
        D4 na, nb;
        if (correct_math(pa, pb, d.con_n[c], beta, na, nb)) {
            if (d.meta[i].y & kFlagMutable) solve::st_state<C>(d.pos + i, na);
            if (d.meta[j].y & kFlagMutable) solve::st_state<C>(d.pos + j, nb);
        }
        if (wimp_out) wimp_out[c] = solve::ld_state<C>(d.con_imp + c).x;
    }

};

__global__ void __launch_bounds__(128) k_island_list(StepArgs a) { solve::island_list(a); }

__global__ void __launch_bounds__(128) k_island_solve(StepArgs a, int ib) {
    solve::island_solve_small<ItemsF64<false>>(a, ib);
}

__global__ void __launch_bounds__(solve::kPlanThreads) k_big_plan(StepArgs a, uint32_t G) { solve::big_plan(a, G); }

__global__ void __launch_bounds__(256) k_big_init(StepArgs a, int ib) { solve::big_init(a, ib); }

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_big(StepArgs a, int ib, int rb) {
    solve::island_solve_team<ItemsF64<true>>(a, ib, rb);
}

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_local(StepArgs a, int ib, int rb) {
    solve::island_solve_local<ItemsF64<false>>(a, ib, rb);
}

__global__ void __launch_bounds__(256) k_big_rec(StepArgs a, int ib, int rb) { solve::big_rec(a, ib, rb); }

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_shared(StepArgs a) {
    solve::island_solve_shared<ItemsF64<false>>(a);
}

// wrapPositions() / applyWalls() (src/world.cpp:698-702, 635-657).
__global__ void __launch_bounds__(kT) k_boundary(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    D4 p = d.pos[i];
    if (!(p.w > 0.0)) return;
    const WorldP& W = a.wp[a.bw[i]];
    if (W.dom.periodic) {
        V3 x = wrap(W.dom, v3of(p));
        d.pos[i] = d4of(x, p.w);
        return;
    }
    if (W.open_boundary) return;
    BodyG b = load_geom(d, i);
    D4 v4 = d.vel[i];
    double px[3] = {p.x, p.y, p.z};
    double pv[3] = {v4.x, v4.y, v4.z};
    const double h = W.dom.half;
    for (int axis = 0; axis < 3; ++axis) {
        for (int sgn = -1; sgn <= 1; sgn += 2) {
            V3 outward = mk(axis == 0 ? double(sgn) : 0.0, axis == 1 ? double(sgn) : 0.0,
                            axis == 2 ? double(sgn) : 0.0);
            b.x = mk(px[0], px[1], px[2]);
            V3 sp = support_world(b, outward);
            double coord = (axis == 0 ? sp.x : axis == 1 ? sp.y : sp.z) * sgn;
            double pen = coord - h;
            if (pen > 0.0) {
                px[axis] -= double(sgn) * pen;
                if (pv[axis] * sgn > 0.0) pv[axis] = -W.restitution * pv[axis];
            }
        }
    }
    d.pos[i] = d4of(mk(px[0], px[1], px[2]), p.w);
    d.vel[i] = d4of(mk(pv[0], pv[1], pv[2]), 0.0);
}

__global__ void k_step_end(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) {
        ctl->halt = 1;
        return;
    }
    if (a.warm) {
        const uint32_t nw = ctl->wsel ^ 1;
        ctl->wcount[nw] = (uint32_t)ctl->C;
        ctl->wsel = nw;
    }
    ctl->steps_done += 1;
    ctl->acc_flags |= ctl->flags;
    ctl->acc_timeout |= ctl->solve_timeout;
    ctl->need_max = max(ctl->need_max, ctl->need_bits);
    ctl->acc_epa += ctl->epa_cap_hits;
    if (ctl->solve_timeout) ctl->halt = 1;   // a failed solve ends a replayed batch
}

__global__ void k_batch_begin(Ctl* ctl) {
    ctl->halt = 0;
    ctl->steps_done = 0;
    ctl->acc_flags = 0;
    ctl->acc_timeout = 0;
    ctl->need_max = 0;
    ctl->acc_epa = 0;
}

inline uint32_t blocks_for(uint64_t n, int t) { return (uint32_t)((n + t - 1) / t); }

// Host-layout state block (the C-ABI's interleaved arrays, back to back):
// x[3n] | q[4n] | v[3n] | w[3n] | force[3n] | torque[3n].  mask bit k selects
// array k.  Unpacking keeps each record's fourth word (invMass in pos).
__global__ void __launch_bounds__(kT) k_unpack_state(DevWorld d, uint32_t n, const double* __restrict__ io,
                                                     uint32_t mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = n;
    if (mask & 1u) {
        const double* x = io + 3 * (size_t)i;
        d.pos[i] = D4{x[0], x[1], x[2], d.pos[i].w};
    }
    if (mask & 2u) {
        const double* q = io + 3 * N + 4 * (size_t)i;
        d.quat[i] = D4{q[0], q[1], q[2], q[3]};
    }
    if (mask & 4u) {
        const double* v = io + 7 * N + 3 * (size_t)i;
        d.vel[i] = D4{v[0], v[1], v[2], 0.0};
    }
    if (mask & 8u) {
        const double* w = io + 10 * N + 3 * (size_t)i;
        d.omg[i] = D4{w[0], w[1], w[2], 0.0};
    }
}

__global__ void __launch_bounds__(kT) k_pack_state(DevWorld d, uint32_t n, double* __restrict__ io, uint32_t mask) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t N = n;
    const D4* src[6] = {d.pos, d.quat, d.vel, d.omg, d.frc, d.trq};
    const size_t off[6] = {0, 3 * N, 7 * N, 10 * N, 13 * N, 16 * N};
    for (int k = 0; k < 6; ++k) {
        if (!(mask & (1u << k))) continue;
        const D4 r = src[k][i];
        if (k == 1) {
            double* o = io + off[k] + 4 * (size_t)i;
            o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = r.w;
        } else {
            double* o = io + off[k] + 3 * (size_t)i;
            o[0] = r.x; o[1] = r.y; o[2] = r.z;
        }
    }
}

}  // namespace

void launch_unpack_state(const DevWorld& d, uint32_t n, const double* io, uint32_t mask, cudaStream_t st) {
    if (n) k_unpack_state<<<blocks_for(n, kT), kT, 0, st>>>(d, n, io, mask);
}

void launch_pack_state(const DevWorld& d, uint32_t n, double* io, uint32_t mask, cudaStream_t st) {
    if (n) k_pack_state<<<blocks_for(n, kT), kT, 0, st>>>(d, n, io, mask);
}

// Teams and dataflow state of the big islands (both precisions).
void launch_big_prep(const StepArgs& a, int ib, cudaStream_t st, uint64_t* launches) {
    k_big_plan<<<1, solve::kPlanThreads, 0, st>>>(a, (uint32_t)(a.num_sms * a.big_ctas_per_sm));
    k_big_init<<<a.num_sms * 2, 256, 0, st>>>(a, ib);
    *launches += 2;
}

void launch_batch_begin(Ctl* ctl, cudaStream_t st) { k_batch_begin<<<1, 1, 0, st>>>(ctl); }

void launch_big_rec(const StepArgs& a, int ib, int rb, cudaStream_t st, uint64_t* launches) {
    k_big_rec<<<a.num_sms * 8, 256, 0, st>>>(a, ib, rb);
    ++*launches;
}

void init_kernel_attrs() {
    cudaFuncSetAttribute(k_island_solve_shared, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLocalCap);
    init_kernel_attrs_f32();
}

// Enqueue one step.  The host reads ctl afterwards to learn whether it must
// be re-run with larger buffers.
void launch_step(const StepArgs& a0, cudaStream_t st, uint64_t* launches, cudaEvent_t* ev, const SideStream* side) {
    StepArgs a = a0;
    const DevWorld& d = a.d;
    Ctl* ctl = d.ctl;
    uint64_t& L = *launches;
    auto mark = [&](int k) {
        if (ev) cudaEventRecord(ev[k], st);
    };
    mark(0);
    k_step_begin<<<1, 1, 0, st>>>(ctl, a.sticky); ++L;
    k_integrate<<<blocks_for(a.n, kT), kT, 0, st>>>(a); ++L;

    mark(1);
    // Broadphase: cell keys -> stable sort -> per-body partner counts -> CSR.
    // Pass 0 (recorded steps only) builds the reference-rule pair list; pass 1
    // builds the internal candidate list the cull consumes.
    for (int fast = a.record ? 0 : 1; fast <= 1; ++fast) {
        int kb = 0;
        if (a.any_grid) {
            k_ext_reset<<<blocks_for(a.nworlds, kT), kT, 0, st>>>(a); ++L;
            k_extents<<<blocks_for(a.n, kT), kT, 0, st>>>(a, fast); ++L;
            k_world_layout<<<blocks_for(a.nworlds, kT), kT, 0, st>>>(a, fast); ++L;
            k_cell_keys<<<blocks_for(a.n, kT), kT, 0, st>>>(a, fast); ++L;
            unsigned long long* keys[2] = {d.key[0], d.key[1]};
            uint32_t* vals[2] = {d.val[0], d.val[1]};
            kb = radix_sort_u64(keys, vals, a.n, a.key_bits, d.hist, d.tsum, ctl, st, launches);
        }
        if (!fast) {
            k_pair_count<<<blocks_for(a.n, kT), kT, 0, st>>>(a, kb, 0); ++L;
            scan_u32(d.bcnt, d.boff, a.n, d.tsum, &ctl->P_ref, ctl, st, launches);
            k_pair_emit<<<blocks_for((uint64_t)a.n * 32, kT), kT, 0, st>>>(a, kb, 0, d.rec_i, d.rec_j, &ctl->P_ref,
                                                                          a.Rcap); ++L;
            continue;
        }
        // Internal grid: cell table, then the filters and the cull inside
        // the partner lists.
        if (a.any_grid) {
            k_hash_clear<<<blocks_for(d.hsize, kT), kT, 0, st>>>(a); ++L;
            k_cell_flags<<<blocks_for(a.n, kT), kT, 0, st>>>(a, kb); ++L;
            scan_u32(d.cflag, d.crun, a.n, d.tsum, &ctl->ncells, ctl, st, launches);
            k_cell_table<<<blocks_for(a.n, kT), kT, 0, st>>>(a, kb); ++L;
        }
        mark(2);
        k_surv_gather<<<blocks_for((uint64_t)a.n * 32, kT), kT, 0, st>>>(a, kb); ++L;
        {
            // one warp per 32 candidates of the longest possible list, at most 2 blocks per SM
            const uint32_t lb = (uint32_t)std::min<uint64_t>(((uint64_t)a.n + 32 * (kT / 32) - 1) / (32 * (kT / 32)), 296);
            k_long_mask<<<lb ? lb : 1, kT, 0, st>>>(a); ++L;
            k_long_place<<<kLongRows, kPlaceT, 0, st>>>(a); ++L;
        }
        scan_u32(d.bcnt, d.boff, a.n, d.tsum, &ctl->S, ctl, st, launches);
        k_surv_place<<<blocks_for((uint64_t)a.n * 32, kT), kT, 0, st>>>(a); ++L;
    }
    if (a.class_sort) {
        k_pair_class<<<blocks_for(a.Scap, kT), kT, 0, st>>>(a); ++L;
        // 6-bit keys: one pass, so the values end in buffer 1 (sperm).
        uint32_t* pk[2] = {d.ccnt, d.coff};
        uint32_t* pv[2] = {d.stage_j, d.sperm};
        radix_sort_u32(pk, pv, (uint32_t)a.Scap, 6, d.hist, d.tsum, ctl, st, launches, &ctl->S);
    }
    mark(3);
    if (a.f32) {
        launch_narrowphase_f32(a, st, launches);
        if (a.any_ext) {
            k_narrowphase_ext_count<<<blocks_for(a.Scap, 128), 128, 0, st>>>(a); ++L;
        }
    } else {
        k_narrowphase<<<blocks_for(a.Scap, 128), 128, 0, st>>>(a); ++L;
    }
    mark(4);
    scan_u32(d.ccnt, d.coff, (uint32_t)a.Scap, d.tsum, &ctl->C, ctl, st, launches, &ctl->S);
    if (a.any_ext) {
        k_narrowphase_ext<<<blocks_for(a.Scap, 128), 128, 0, st>>>(a); ++L;
    }
    k_constraint_build<<<blocks_for(a.Scap, kT), kT, 0, st>>>(a); ++L;

    mark(5);
    // Islands: label, stable sort by label, segment starts.
    k_island_label<<<blocks_for(a.Ccap, kT), kT, 0, st>>>(a); ++L;
    int lbits = 1;
    while ((1ull << lbits) <= (unsigned long long)a.n) ++lbits;
    uint32_t* labs[2] = {d.ilab[0], d.ilab[1]};
    uint32_t* ords[2] = {d.iord[0], d.iord[1]};
    const int ib = radix_sort_u32(labs, ords, (uint32_t)a.Ccap, lbits, d.hist, d.tsum, ctl, st, launches, &ctl->C);
    k_island_mark<<<blocks_for(a.Ccap, kT), kT, 0, st>>>(a, ib); ++L;
    scan_u32(d.iflag, d.ioff, (uint32_t)a.Ccap, d.tsum, &ctl->scan_total, ctl, st, launches, &ctl->C);
    k_island_start<<<blocks_for(a.Ccap, kT), kT, 0, st>>>(a); ++L;
    k_island_list<<<blocks_for(a.Ccap, 128), 128, 0, st>>>(a); ++L;
    // Small islands (one thread each) on the side stream, beside the rank
    // sort and the big-island solvers.
    cudaStream_t ss = st;
    if (side && side->st2) {
        cudaEventRecord(side->fork, st);
        cudaStreamWaitEvent(side->st2, side->fork, 0);
        ss = side->st2;
    }
    if (a.f32) {
        launch_solve_small_f32(a, ib, ss, launches);
    } else {
        k_island_solve<<<blocks_for(a.Ccap, 128), 128, 0, ss>>>(a, ib); ++L;
    }
    // Per-body update ranks for the dataflow solver.
    k_rank_entries<<<blocks_for(a.Ccap, kT), kT, 0, st>>>(a, ib); ++L;
    uint32_t* rks[2] = {d.rkey[0], d.rkey[1]};
    uint32_t* rvs[2] = {d.rval[0], d.rval[1]};
    const int rb = radix_sort_u32(rks, rvs, (uint32_t)(2 * a.Ccap), lbits, d.hist, d.tsum, ctl, st, launches,
                                  &ctl->C2);
    k_rank_write<<<blocks_for(2 * a.Ccap, kT), kT, 0, st>>>(a, rb); ++L;
    mark(6);
    if (a.f32) {
        launch_solve_big_f32(a, ib, rb, st, launches);
    } else {
        if (a.big_team_max == 1) {
            launch_big_rec(a, ib, rb, st, launches);
            k_island_solve_shared<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, a.local_cap, st>>>(a); ++L;
            k_island_solve_local<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, 0, st>>>(a, ib, rb); ++L;
        } else {
            launch_big_prep(a, ib, st, launches);
            k_island_solve_big<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, 0, st>>>(a, ib, rb); ++L;
        }
    }
    if (ss != st) {
        cudaEventRecord(side->join, ss);
        cudaStreamWaitEvent(st, side->join, 0);
    }
    if (a.f32) launch_writeback_f32(a, st, launches);
    mark(7);
    k_boundary<<<blocks_for(a.n, kT), kT, 0, st>>>(a); ++L;
    k_step_end<<<1, 1, 0, st>>>(a); ++L;
    mark(8);
}

}  // namespace neb
