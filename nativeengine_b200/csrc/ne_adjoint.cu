// ne_adjoint.cu -- stepBackward on the device: one CTA per world runs the
// per-world step program and its adjoint (ne_adjoint.cuh), its threads sharing
// the bodies, the pairs and the islands of the world.
//
// Per world: (1) the state and the warm-cache entries of the world are read
// from the device world; (2) the trajectory is stepped forward, keeping the
// state and warm cache every K steps; (3) segments are taken in reverse: the
// K steps of a segment are recomputed from its checkpoint, keeping each
// step's input, and the adjoint of each step is applied from the last to the
// first.  Memory per world: ceil(T/K) + K states and warm caches, one step's
// contacts and tape (phases 0-8 of every contact).  The world itself is only
// read.
#include "ne_adjoint.cuh"

namespace neb {

namespace {

using adj::St;

__device__ __forceinline__ St load_state(const DevWorld& d, uint32_t i) {
    St s;
    const D4 p = d.pos[i], q = d.quat[i], v = d.vel[i], w = d.omg[i], f = d.frc[i], t = d.trq[i];
    s.x = mk(p.x, p.y, p.z);
    s.q = mkq(q.x, q.y, q.z, q.w);
    s.v = mk(v.x, v.y, v.z);
    s.w = mk(w.x, w.y, w.z);
    s.f = mk(f.x, f.y, f.z);
    s.t = mk(t.x, t.y, t.z);
    return s;
}

struct WarmSlot {
    unsigned long long* k;
    double* v;
    uint32_t* n;
};

__device__ __forceinline__ WarmSlot warm_slot(const AdjArgs& a, uint32_t slot, uint32_t w) {
    WarmSlot s;
    const size_t off = (size_t)slot * a.CT + a.coff[w];
    s.k = a.WK + off;
    s.v = a.WI + off;
    s.n = a.WN + (size_t)slot * a.nworlds + w;
    return s;
}

__device__ __forceinline__ void copy_warm(const WarmSlot& dst, const WarmSlot& src, const adj::Team& t) {
    const uint32_t n = *src.n;
    for (uint32_t k = t.lane; k < n; k += t.size) { dst.k[k] = src.k[k]; dst.v[k] = src.v[k]; }
    t.sync();
    if (t.lane == 0) *dst.n = n;
    t.sync();
}

// Threads per world: the lanes share the world's bodies, pairs, islands and
// contacts; 64 keeps every world of a 512-world batch resident at once.
constexpr int kTeamThreads = 64;

// One CTA per world.
__global__ void __launch_bounds__(kTeamThreads) k_adj_world(AdjArgs a) {
    __shared__ uint32_t s_team[adj::kTeamScratch];
    const uint32_t w = blockIdx.x;
    if (w >= a.nworlds) return;   // whole blocks only
    const adj::Team t{(int)threadIdx.x, (int)blockDim.x, s_team};
    const DevWorld& d = a.d;
    const WorldP& W = a.wp[w];
    const uint32_t b0 = a.wbegin[w], b1 = a.wbegin[w + 1], nb = b1 - b0;
    const uint32_t cap = a.cap[w];
    const int warm = a.warm;
    if (t.lane == 0) a.err[w] = 0;
    if (nb > kAdjMaxBodies || !adj::backward_supported(d, W, b0, b1)) {
        if (t.lane == 0) a.err[w] = adj::kErrUnsupported;
        return;
    }
    adj::WScr s;
    s.b0 = b0;
    s.nb = nb;
    s.cap = cap;
    s.s = a.S + b0;
    s.s0 = a.S0 + b0;
    s.s1 = a.S1 + b0;
    s.uf = a.UF + b0;
    s.con = a.CON + a.coff[w];
    s.ncon = 0;
    s.tape = nullptr;
    s.err = 0;
    adj::Cb* cbs = a.CBS + a.coff[w];
    double* tape = a.TAPE + (size_t)9 * adj::kTapeRec * a.coff[w];
    St* sb = a.SB + b0;
    adj::Pb* pb = a.PB + b0;
    double* wob = a.WOB + a.coff[w];
    double* wib = a.WIB + a.coff[w];
    int err = 0;

    // Initial state and the world's entries of the warm cache (keys i<<32|j
    // with b0 <= i < b1 form one sorted run of the device cache).
    for (uint32_t b = t.lane; b < nb; b += t.size) s.s[b] = load_state(d, b0 + b);
    WarmSlot cur[2] = {warm_slot(a, 0, w), warm_slot(a, 1, w)};
    {
        const unsigned long long lo = (unsigned long long)b0 << 32, hi = (unsigned long long)b1 << 32;
        const uint32_t i0 = adj::lower_bound_key(a.wk0, a.nw0, lo), i1 = adj::lower_bound_key(a.wk0, a.nw0, hi);
        if (i1 - i0 > cap) {
            if (t.lane == 0) a.err[w] = adj::kErrCapacity;
            return;
        }
        for (uint32_t k = i0 + t.lane; k < i1; k += t.size) {
            cur[0].k[k - i0] = a.wk0[k];
            cur[0].v[k - i0] = a.wi0[k];
        }
        t.sync();
        if (t.lane == 0) {
            *cur[0].n = i1 - i0;
            *cur[1].n = 0;
        }
        t.sync();
    }
    int rd = 0;
    auto step_fwd = [&]() {
        s.wk_in = cur[rd].k;
        s.wi_in = cur[rd].v;
        s.nw_in = *cur[rd].n;
        s.wk_out = cur[rd ^ 1].k;
        s.wi_out = cur[rd ^ 1].v;
        s.tape = nullptr;
        adj::fwd_step(d, W, warm, s, t);
        if (warm) {
            t.sync();
            if (t.lane == 0) *cur[rd ^ 1].n = s.nw_out;
            t.sync();
            rd ^= 1;
        }
    };
    auto save = [&](St* dst, const WarmSlot& wdst) {
        for (uint32_t b = t.lane; b < nb; b += t.size) dst[b] = s.s[b];
        copy_warm(wdst, cur[rd], t);
    };
    auto load = [&](const St* src, const WarmSlot& wsrc) {
        for (uint32_t b = t.lane; b < nb; b += t.size) s.s[b] = src[b];
        copy_warm(cur[rd], wsrc, t);
    };

    // Forward pass with checkpoints every K steps.
    for (uint32_t step = 0; step < a.nsteps; ++step) {
        if (step % a.K == 0) save(a.CKS + (size_t)(step / a.K) * a.n + b0, warm_slot(a, 2 + step / a.K, w));
        step_fwd();
        if (s.err & (adj::kErrCapacity | adj::kErrUnsupported)) {
            if (t.lane == 0) a.err[w] = s.err;
            return;
        }
        err |= s.err;
    }

    // Adjoint of the final state.
    for (uint32_t b = t.lane; b < nb; b += t.size) {
        sb[b] = adj::st_zero();
        const size_t g = 3 * (size_t)(b0 + b);
        if (a.xbar) sb[b].x = mk(a.xbar[g], a.xbar[g + 1], a.xbar[g + 2]);
        if (a.vbar) sb[b].v = mk(a.vbar[g], a.vbar[g + 1], a.vbar[g + 2]);
        pb[b].invM = 0.0;
        pb[b].invI = mk(0.0, 0.0, 0.0);
    }
    t.sync();
    double mub = 0.0, eb = 0.0;
    bool have_wob = false;
    const uint32_t nseg = (a.nsteps + a.K - 1) / a.K;
    for (uint32_t seg = nseg; seg-- > 0;) {
        const uint32_t t0 = seg * a.K, t1 = min(a.nsteps, t0 + a.K);
        rd = 0;
        load(a.CKS + (size_t)seg * a.n + b0, warm_slot(a, 2 + seg, w));
        for (uint32_t step = t0; step < t1; ++step) {
            save(a.SEGS + (size_t)(step - t0) * a.n + b0, warm_slot(a, 2 + a.nck + (step - t0), w));
            step_fwd();
        }
        for (uint32_t step = t1; step-- > t0;) {
            rd = 0;
            load(a.SEGS + (size_t)(step - t0) * a.n + b0, warm_slot(a, 2 + a.nck + (step - t0), w));
            s.wk_in = cur[0].k;
            s.wi_in = cur[0].v;
            s.nw_in = *cur[0].n;
            s.wk_out = cur[1].k;
            s.wi_out = cur[1].v;
            s.tape = tape;
            s.err = 0;
            for (uint32_t k = t.lane; k < s.nw_in; k += t.size) wib[k] = 0.0;
            t.sync();
            adj::bwd_step(d, W, warm, s, sb, have_wob ? wob : nullptr, wib, pb, cbs, mub, eb, t);
            if (s.err & (adj::kErrCapacity | adj::kErrUnsupported)) {
                if (t.lane == 0) a.err[w] = s.err;
                return;
            }
            err |= s.err;
            t.sync();
            for (uint32_t k = t.lane; k < s.nw_in; k += t.size) wob[k] = wib[k];
            t.sync();
            have_wob = true;
        }
    }

    // Outputs.
    for (uint32_t b = t.lane; b < nb; b += t.size) {
        const St& g = sb[b];
        const size_t i = b0 + b;
        if (a.gx) { a.gx[3 * i] = g.x.x; a.gx[3 * i + 1] = g.x.y; a.gx[3 * i + 2] = g.x.z; }
        if (a.gq) { a.gq[4 * i] = g.q.w; a.gq[4 * i + 1] = g.q.x; a.gq[4 * i + 2] = g.q.y; a.gq[4 * i + 3] = g.q.z; }
        if (a.gv) { a.gv[3 * i] = g.v.x; a.gv[3 * i + 1] = g.v.y; a.gv[3 * i + 2] = g.v.z; }
        if (a.gw) { a.gw[3 * i] = g.w.x; a.gw[3 * i + 1] = g.w.y; a.gw[3 * i + 2] = g.w.z; }
        a.ginvm[i] = pb[b].invM;
        a.ginvi[3 * i] = pb[b].invI.x;
        a.ginvi[3 * i + 1] = pb[b].invI.y;
        a.ginvi[3 * i + 2] = pb[b].invI.z;
    }
    if (t.lane == 0) {
        a.gmu[w] = mub;
        a.ge[w] = eb;
        a.err[w] = err;
    }
}

}  // namespace

void launch_adjoint(const AdjArgs& a, cudaStream_t st) {
    k_adj_world<<<a.nworlds, kTeamThreads, 0, st>>>(a);
}

}  // namespace neb
