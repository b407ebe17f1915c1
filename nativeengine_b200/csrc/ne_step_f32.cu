// ne_step_f32.cu -- the batched FP32 form's narrowphase and contact solve.
//
// Same stages, same contact order and the same update sequence as the FP64
// kernels in ne_step.cu; only the arithmetic precision differs:
//
//   narrowphase   the pair is moved into a frame centred on the body with the
//                 smaller bounding radius (offset = FP64 minimum image, then
//                 rounded), so FP32 coordinates stay of the order of the
//                 bodies' size even in a large or periodic world.  Support
//                 mappings, the analytic pairs and the box-box clipping run
//                 in FP32; GJK's simplex and EPA's polytope arithmetic (their
//                 containment and termination tests) run in FP64 over the
//                 FP32 support points (ne_geom.cuh).  Contacts
//                 are stored in the FP64 contact arrays (point = origin +
//                 FP32 offset, in FP64).
//   solve         body velocities, lever arms, restitution bias, friction and
//                 effective masses in FP32 (records written by the FP64
//                 constraint build); the accumulated normal impulse nImp,
//                 which is the warm-start cache, is accumulated in FP64;
//                 position correction is an FP32 displacement added to the
//                 FP64 pose.  Velocities go back to the FP64 state as
//                 v64 += (v32_final - v32_initial), so a body the solve does
//                 not touch keeps its FP64 velocity bit for bit.
//
// This translation unit is compiled with FMA contraction enabled (the FP64
// path is compiled without it, for bit parity with the reference).
#include "ne_solve.cuh"

namespace neb {

namespace {

constexpr int kT = 256;

__device__ __forceinline__ V3 v3d(const D4& a) { return mk(a.x, a.y, a.z); }
__device__ __forceinline__ V3f v3f(const F4& a) { return mk3<float>(a.x, a.y, a.z); }
__device__ __forceinline__ Qf qf(const F4& a) { return mkq4<float>(a.x, a.y, a.z, a.w); }
__device__ __forceinline__ D4 d4of(const V3& v, double w) { D4 r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }
__device__ __forceinline__ F4 f4of(const V3f& v, float w) { F4 r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = w; return r; }

inline uint32_t blocks_for(uint64_t n, int t) { return (uint32_t)((n + t - 1) / t); }

__device__ __forceinline__ BodyGT<float> load_geom_f32(const DevWorld& d, uint32_t i, const V3f& x) {
    const F4 e = d.f_e[i];
    const uint4 m = d.meta[i];
    const uint2 vr = d.vrng[i];
    BodyGT<float> b;
    b.x = x;
    b.q = qf(d.f_q[i]);
    b.he = v3f(e);
    b.radius = e.w;
    b.half_height = d.f_I[i].w;
    b.verts = d.f_verts + vr.x;
    b.nverts = (int)vr.y;
    b.shape = (int)m.x;
    return b;
}

// gatherContacts() for one surviving pair (src/world.cpp:122-129), FP32.
__global__ void __launch_bounds__(128) k_narrowphase_f32(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ctl->S) return;
    const uint64_t s = a.class_sort ? (uint64_t)a.d.sperm[t] : t;   // narrowphase order (ne_step.cu)
    const DevWorld& d = a.d;
    const uint32_t i = d.si[s], j = d.sj[s];
    // Triangle meshes and compounds: their contacts come from the FP64
    // count and write passes (k_narrowphase_ext_count, k_narrowphase_ext).
    const int shi = (int)d.meta[i].x, shj = (int)d.meta[j].x;
    if (shi == SH_MESH || shi == SH_COMPOUND || shj == SH_MESH || shj == SH_COMPOUND) return;
    const Domain dom = a.wp[a.bw[i]].dom;
    const V3 xi = v3d(d.pos[i]), xj = v3d(d.pos[j]);
    const V3 dij = min_image(dom, xj - xi);
    const bool origin_j = d.inert[j].w < d.inert[i].w;
    const V3f zero = mk3<float>(0.0f, 0.0f, 0.0f);
    const V3f ri = origin_j ? cvt<float>(-dij) : zero;
    const V3f rj = origin_j ? zero : cvt<float>(dij);
    const V3 xo = origin_j ? xj : xi;
    const BodyGT<float> A = load_geom_f32(d, i, ri), B = load_geom_f32(d, j, rj);
    const Domain local = {dom.half, 0};   // the frame is already a minimum image
    EpaScratchT<float> S;
    int fl = 0;
    ContactT<float> c = detect_contact(A, B, local, S, fl);
    uint32_t cnt = 0;
    if (c.hit) {
        const V3 n = cvt<double>(c.normal);
        if (A.shape == SH_BOX && B.shape == SH_BOX) {
            ManifoldT<float> m = box_box_manifold(A, B, c.normal, local, fl);
            for (int k = 0; k < m.count; ++k) {
                d.cn[4 * s + k] = d4of(n, (double)m.depth[k]);
                d.cp[4 * s + k] = d4of(xo + cvt<double>(m.point[k]), 0.0);
            }
            cnt = (uint32_t)m.count;
        }
        if (cnt == 0) {
            d.cn[4 * s] = d4of(n, (double)c.overlap);
            d.cp[4 * s] = d4of(xo + cvt<double>(c.point), 0.0);
            cnt = 1;
        }
    }
    d.ccnt[s] = cnt;
    if (fl & 1) atomicOr(&ctl->flags, 1u);
    if (fl & 2) atomicAdd((unsigned long long*)&ctl->epa_cap_hits, 1ull);
}

struct BodyF {
    V3f v, w;
    Qf q;
    V3f invI;
    float invM;
    bool mut;
};

template <bool C>
__device__ __forceinline__ BodyF load_body_f32(const DevWorld& d, uint32_t i) {
    BodyF b;
    const F4 v = solve::ld_state<C>(d.f_v + i);
    b.v = v3f(v);
    b.invM = v.w;
    b.w = v3f(solve::ld_state<C>(d.f_w + i));
    b.q = qf(d.f_q[i]);
    b.invI = v3f(d.f_I[i]);
    b.mut = (d.meta[i].y & kFlagMutable) != 0;
    return b;
}

template <bool C>
__device__ __forceinline__ void store_body_f32(const DevWorld& d, uint32_t i, const BodyF& b) {
    if (!b.mut) return;   // immovable: shared by islands, never written
    solve::st_state<C>(d.f_v + i, f4of(b.v, b.invM));
    solve::st_state<C>(d.f_w + i, f4of(b.w, 0.0f));
}

// effMass (src/contact.hpp:28-33).
__device__ __forceinline__ float eff_mass_f32(const BodyF& A, const BodyF& B, const V3f& ra, const V3f& rb,
                                              const V3f& u) {
    V3f angA = cross(apply_inv_inertia(A.q, A.invI, cross(ra, u)), ra);
    V3f angB = cross(apply_inv_inertia(B.q, B.invI, cross(rb, u)), rb);
    return A.invM + B.invM + dot(angA + angB, u);
}

__device__ __forceinline__ void apply_pair_impulse_f32(BodyF& A, BodyF& B, const V3f& ra, const V3f& rb,
                                                       const V3f& J) {
    A.v = A.v + J * A.invM;
    A.w = A.w + apply_inv_inertia(A.q, A.invI, cross(ra, J));
    B.v = B.v - J * B.invM;
    B.w = B.w - apply_inv_inertia(B.q, B.invI, cross(rb, J));
}

// The arithmetic of the three kinds of update on operands already loaded.
// Warm-start application (src/world.cpp:560-567).
__device__ __forceinline__ void warm_math_f32(BodyF& A, BodyF& B, const F4& n4, const F4& ra4, const F4& rb4,
                                              double nImp) {
    apply_pair_impulse_f32(A, B, v3f(ra4), v3f(rb4), v3f(n4) * (float)nImp);
}

// One sequential-impulse update (src/world.cpp:575-610).  nImp accumulates
// in FP64; the velocity change it implies is FP32.
__device__ __forceinline__ void sweep_math_f32(BodyF& A, BodyF& B, const F4& n4, const F4& ra4, const F4& rb4,
                                               float Kn, double2& imp) {
    const V3f n = v3f(n4), rA = v3f(ra4), rB = v3f(rb4);
    const float restBias = ra4.w, mu = rb4.w;
    const V3f vc = (A.v + cross(A.w, rA)) - (B.v + cross(B.w, rB));
    const float vn = dot(vc, n);
    if (Kn > 1e-18f) {
        const float dj = (restBias - vn) / Kn;
        const double old = imp.x;
        const double sum = old + (double)dj;
        imp.x = (sum > 0.0) ? sum : 0.0;
        apply_pair_impulse_f32(A, B, rA, rB, n * (float)(imp.x - old));
    }
    if (mu > 0.0f && imp.x > 0.0) {
        const V3f vc2 = (A.v + cross(A.w, rA)) - (B.v + cross(B.w, rB));
        const V3f vt = vc2 - n * dot(vc2, n);
        const float vtl = norm(vt);
        if (vtl > 1e-12f) {
            const V3f tg = vt / vtl;
            const float Kt = eff_mass_f32(A, B, rA, rB, tg);
            if (Kt > 1e-18f) {
                const float djt = -vtl / Kt;
                const float maxF = mu * (float)imp.x;
                const float old = (float)imp.y;
                const float sum = old + djt;
                const float nt = (sum < -maxF) ? -maxF : (sum > maxF ? maxF : sum);
                imp.y = (double)nt;
                apply_pair_impulse_f32(A, B, rA, rB, tg * (nt - old));
            }
        }
    }
}

// correctPenetration (src/contact.hpp:78-85): FP32 displacement, FP64 pose.
__device__ __forceinline__ bool correct_math_f32(const D4& pa, const D4& pb, const F4& n4, double beta, D4& na,
                                                 D4& nb) {
    const float invSum = (float)pa.w + (float)pb.w;
    const float overlap = n4.w;
    if (invSum <= 0.0f || overlap <= 0.0f) return false;
    const V3f corr = v3f(n4) * ((float)beta * overlap / invSum);
    na = d4of(v3d(pa) + cvt<double>(corr * (float)pa.w), pa.w);
    nb = d4of(v3d(pb) - cvt<double>(corr * (float)pb.w), pb.w);
    return true;
}

template <bool C>
struct ItemsF32 {
    static __device__ __forceinline__ void warm(const DevWorld& d, uint32_t c) {
        const double nImp = solve::ld_state<C>(d.con_imp + c).x;
        if (nImp == 0.0) return;
        const uint32_t i = d.ci[c], j = d.cj[c];
        BodyF A = load_body_f32<C>(d, i), B = load_body_f32<C>(d, j);
        warm_math_f32(A, B, d.f_n[c], d.f_ra[c], d.f_rb[c], nImp);
        store_body_f32<C>(d, i, A);
        store_body_f32<C>(d, j, B);
    }

    static __device__ __forceinline__ void sweep(const DevWorld& d, uint32_t c) {
        const uint32_t i = d.ci[c], j = d.cj[c];
        BodyF A = load_body_f32<C>(d, i), B = load_body_f32<C>(d, j);
        double2 imp = solve::ld_state<C>(d.con_imp + c);
        sweep_math_f32(A, B, d.f_n[c], d.f_ra[c], d.f_rb[c], d.f_kn[c], imp);
        solve::st_state<C>(d.con_imp + c, imp);
        store_body_f32<C>(d, i, A);
        store_body_f32<C>(d, j, B);
    }

    static __device__ __forceinline__ void correct(const DevWorld& d, uint32_t c, double beta, double* wout) {
        const uint32_t i = d.ci[c], j = d.cj[c];
        const D4 pa = solve::ld_state<C>(d.pos + i), pb = solve::ld_state<C>(d.pos + j);
        D4 na, nb;
        if (correct_math_f32(pa, pb, d.f_n[c], beta, na, nb)) {
            if (d.meta[i].y & kFlagMutable) solve::st_state<C>(d.pos + i, na);
            if (d.meta[j].y & kFlagMutable) solve::st_state<C>(d.pos + j, nb);
        }
        if (wout) wout[c] = solve::ld_state<C>(d.con_imp + c).x;
    }
};

__global__ void __launch_bounds__(128) k_island_solve_f32(StepArgs a, int ib) {
    solve::island_solve_small<ItemsF32<false>>(a, ib);
}

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_big_f32(StepArgs a, int ib, int rb) {
    solve::island_solve_team<ItemsF32<true>>(a, ib, rb);
}

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_local_f32(StepArgs a, int ib, int rb) {
    solve::island_solve_local<ItemsF32<false>>(a, ib, rb);
}

__global__ void __launch_bounds__(solve::kMaxBigThreads) k_island_solve_shared_f32(StepArgs a) {
    solve::island_solve_shared<ItemsF32<false>>(a);
}

// Solver velocities back into the FP64 state: v64 += v32 - fl(v64).
__global__ void __launch_bounds__(kT) k_writeback_f32(StepArgs a) {
    Ctl* ctl = a.d.ctl;
    if (ctl->abort) return;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const DevWorld& d = a.d;
    if (!(d.meta[i].y & kFlagMutable)) return;
    const D4 v = d.vel[i], w = d.omg[i];
    const F4 fv = d.f_v[i], fw = d.f_w[i];
    const V3f dv = v3f(fv) - cvt<float>(v3d(v));
    const V3f dw = v3f(fw) - cvt<float>(v3d(w));
    if (dv.x != 0.0f || dv.y != 0.0f || dv.z != 0.0f) d.vel[i] = d4of(v3d(v) + cvt<double>(dv), v.w);
    if (dw.x != 0.0f || dw.y != 0.0f || dw.z != 0.0f) d.omg[i] = d4of(v3d(w) + cvt<double>(dw), w.w);
}

__global__ void __launch_bounds__(kT) k_convert_verts(const D4* src, F4* dst, uint32_t count) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const D4 v = src[k];
    dst[k] = F4{(float)v.x, (float)v.y, (float)v.z, 0.0f};
}

}  // namespace

void launch_narrowphase_f32(const StepArgs& a, cudaStream_t st, uint64_t* launches) {
    k_narrowphase_f32<<<blocks_for(a.Scap, 128), 128, 0, st>>>(a);
    ++*launches;
}

void launch_solve_small_f32(const StepArgs& a, int ib, cudaStream_t st, uint64_t* launches) {
    k_island_solve_f32<<<blocks_for(a.Ccap, 128), 128, 0, st>>>(a, ib);
    ++*launches;
}

void launch_solve_big_f32(const StepArgs& a, int ib, int rb, cudaStream_t st, uint64_t* launches) {
    if (a.big_team_max == 1) {
        launch_big_rec(a, ib, rb, st, launches);
        k_island_solve_shared_f32<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, a.local_cap, st>>>(a);
        k_island_solve_local_f32<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, 0, st>>>(a, ib, rb);
        ++*launches;
    } else {
        launch_big_prep(a, ib, st, launches);
        k_island_solve_big_f32<<<a.num_sms * a.big_ctas_per_sm, a.big_threads, 0, st>>>(a, ib, rb);
    }
    ++*launches;
}

void launch_writeback_f32(const StepArgs& a, cudaStream_t st, uint64_t* launches) {
    k_writeback_f32<<<blocks_for(a.n, kT), kT, 0, st>>>(a);
    ++*launches;
}

void init_kernel_attrs_f32() {
    cudaFuncSetAttribute(k_island_solve_shared_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLocalCap);
}

void convert_verts_f32(const D4* src, F4* dst, uint32_t count, cudaStream_t st) {
    if (count) k_convert_verts<<<blocks_for(count, kT), kT, 0, st>>>(src, dst, count);
}

}  // namespace neb
