// Test-only host build of the per-world step program and its adjoint
// (nativeengine_b200/csrc/ne_adjoint.cuh).  The library ships these functions
// only as device code (ne_adjoint.cu); compiling the same __host__ __device__
// source with g++ lets the CPU test suite check the forward bit for bit
// against the oracle and the gradients against finite differences.  Nothing
// in the library loads this file.
//
// Build (tests/test_adjoint_cpu.py):
//   g++ -std=c++17 -O2 -ffp-contract=off -fPIC -shared -I include
//       -I nativeengine_b200/csrc tests/cpp/adjoint_host.cpp -o <tmp>/libadj_host.so
#include <cstring>
#include <vector>

#include "ne_adjoint.cuh"

using namespace neb;

namespace {

// Host image of the device records of one world (what ne_world_upload builds).
struct HostWorld {
    std::vector<D4> pos, quat, vel, omg, frc, trq, inert, geom, ext, mat, verts;
    std::vector<uint4> meta;
    std::vector<uint2> vrng, ncrng;
    std::vector<uint32_t> nc;
    DevWorld d{};
    WorldP W{};
    int warm = 1;
    uint32_t n = 0;
};

void build(HostWorld& h, const NeWorldParams* p, const NeBodyArrays* b) {
    const uint32_t n = b->n;
    h.n = n;
    auto v3 = [&](const double* a, uint32_t i, double w) { return D4{a[3 * i], a[3 * i + 1], a[3 * i + 2], w}; };
    h.verts.assign(b->n_verts ? b->n_verts : 1, D4{0, 0, 0, 0});
    for (uint32_t k = 0; k < b->n_verts; ++k) h.verts[k] = v3(b->verts, k, 0.0);
    h.pos.resize(n); h.quat.resize(n); h.vel.resize(n); h.omg.resize(n); h.frc.resize(n); h.trq.resize(n);
    h.inert.resize(n); h.geom.resize(n); h.ext.resize(n); h.mat.resize(n); h.meta.resize(n);
    h.vrng.resize(n); h.ncrng.resize(n);
    h.nc.assign(b->n_nocollide ? b->n_nocollide : 1, 0);
    for (uint32_t k = 0; k < b->n_nocollide; ++k) h.nc[k] = b->nocollide[k];
    for (uint32_t i = 0; i < n; ++i) {
        h.pos[i] = v3(b->x, i, b->inv_mass[i]);
        h.quat[i] = D4{b->q[4 * i], b->q[4 * i + 1], b->q[4 * i + 2], b->q[4 * i + 3]};
        h.vel[i] = v3(b->v, i, 0.0);
        h.omg[i] = v3(b->w, i, 0.0);
        h.frc[i] = b->force ? v3(b->force, i, 0.0) : D4{0, 0, 0, 0};
        h.trq[i] = b->torque ? v3(b->torque, i, 0.0) : D4{0, 0, 0, 0};
        const int s = b->shape[i];
        const V3 he = mk(b->half_extents[3 * i], b->half_extents[3 * i + 1], b->half_extents[3 * i + 2]);
        const D4* vp = (s == NE_SHAPE_CONVEX) ? h.verts.data() + b->vert_offset[i] : h.verts.data();
        const int nv = (s == NE_SHAPE_CONVEX) ? (int)b->vert_count[i] : 0;
        const double br = bounding_radius(s, b->radius[i], b->half_height[i], he, vp, nv);
        h.inert[i] = v3(b->inv_inertia, i, br);
        h.geom[i] = D4{b->radius[i], b->half_height[i], b->gravity_scale[i], 0.0};
        h.ext[i] = v3(b->half_extents, i, 0.0);
        h.mat[i] = D4{b->friction[i], b->restitution[i], b->linear_damping[i], b->angular_damping[i]};
        uint32_t fl = b->flags[i] & 0xFFFFu;
        const bool mut = b->inv_mass[i] > 0.0 || b->inv_inertia[3 * i] != 0.0 || b->inv_inertia[3 * i + 1] != 0.0 ||
                         b->inv_inertia[3 * i + 2] != 0.0;
        if (mut) fl |= kFlagMutable;
        h.meta[i] = make_uint4((uint32_t)s, fl, b->layer[i], b->mask[i]);
        h.vrng[i] = (s == NE_SHAPE_CONVEX) ? make_uint2(b->vert_offset[i], b->vert_count[i]) : make_uint2(0, 0);
        h.ncrng[i] = (b->nocollide_count && b->nocollide_count[i])
                         ? make_uint2(b->nocollide_offset[i], b->nocollide_count[i]) : make_uint2(0, 0);
    }
    DevWorld& d = h.d;
    d.pos = h.pos.data(); d.quat = h.quat.data(); d.vel = h.vel.data(); d.omg = h.omg.data();
    d.frc = h.frc.data(); d.trq = h.trq.data(); d.inert = h.inert.data(); d.geom = h.geom.data();
    d.ext = h.ext.data(); d.mat = h.mat.data(); d.meta = h.meta.data(); d.vrng = h.vrng.data();
    d.verts = h.verts.data(); d.ncrng = h.ncrng.data(); d.nc = h.nc.data();
    WorldP& W = h.W;
    W.dom.half = p->half;
    W.dom.periodic = p->periodic;
    W.dt = p->dt;
    W.restitution = p->restitution;
    W.friction = p->friction;
    W.beta = p->contact_beta;
    W.g = mk(p->gravity[0], p->gravity[1], p->gravity[2]);
    W.rcomb = p->restitution_combine;
    W.fcomb = p->friction_combine;
    W.open_boundary = p->open_boundary;
    W.begin = 0;
    W.end = n;
    h.warm = p->warm_start ? 1 : 0;
}

struct Run {
    std::vector<adj::St> s, s0, s1;
    std::vector<uint32_t> uf;
    std::vector<adj::Con> con;
    std::vector<double> tape;
    std::vector<unsigned long long> wk[2];
    std::vector<double> wi[2];
    uint32_t nw[2] = {0, 0};
    adj::WScr w{};
    uint32_t cap = 0;

    void init(const HostWorld& h, uint32_t capacity) {
        cap = capacity;
        s.resize(h.n); s0.resize(h.n); s1.resize(h.n); uf.resize(h.n);
        for (uint32_t i = 0; i < h.n; ++i) {
            adj::St& t = s[i];
            t.x = mk(h.pos[i].x, h.pos[i].y, h.pos[i].z);
            t.q = mkq(h.quat[i].x, h.quat[i].y, h.quat[i].z, h.quat[i].w);
            t.v = mk(h.vel[i].x, h.vel[i].y, h.vel[i].z);
            t.w = mk(h.omg[i].x, h.omg[i].y, h.omg[i].z);
            t.f = mk(h.frc[i].x, h.frc[i].y, h.frc[i].z);
            t.t = mk(h.trq[i].x, h.trq[i].y, h.trq[i].z);
        }
        con.resize(cap);
        tape.resize((size_t)9 * cap * adj::kTapeRec);
        for (int k = 0; k < 2; ++k) { wk[k].assign(cap, 0); wi[k].assign(cap, 0.0); }
        w.b0 = 0; w.nb = h.n; w.cap = cap;
        w.s = s.data(); w.s0 = s0.data(); w.s1 = s1.data(); w.con = con.data(); w.tape = tape.data();
        w.uf = uf.data();
    }

    // One forward step reading warm cache `rd`, writing the other.
    int step(const HostWorld& h, int rd, bool with_tape) {
        w.wk_in = wk[rd].data(); w.wi_in = wi[rd].data(); w.nw_in = nw[rd];
        w.wk_out = wk[rd ^ 1].data(); w.wi_out = wi[rd ^ 1].data();
        w.tape = with_tape ? tape.data() : nullptr;
        w.err = 0;
        adj::fwd_step(h.d, h.W, h.warm, w, adj::Team{0, 1});
        nw[rd ^ 1] = w.nw_out;
        return w.err;
    }
};

}  // namespace

extern "C" {

// nsteps forward from the given bodies; state out in the C-ABI layout.
int adjh_forward(const NeWorldParams* p, const NeBodyArrays* b, int nsteps, uint32_t cap, double* x, double* q,
                 double* v, double* w) {
    HostWorld h;
    build(h, p, b);
    Run r;
    r.init(h, cap);
    int rd = 0;
    for (int k = 0; k < nsteps; ++k) {
        if (int e = r.step(h, rd, false)) return e;
        if (h.warm) rd ^= 1;
    }
    for (uint32_t i = 0; i < h.n; ++i) {
        const adj::St& s = r.s[i];
        x[3 * i] = s.x.x; x[3 * i + 1] = s.x.y; x[3 * i + 2] = s.x.z;
        q[4 * i] = s.q.w; q[4 * i + 1] = s.q.x; q[4 * i + 2] = s.q.y; q[4 * i + 3] = s.q.z;
        v[3 * i] = s.v.x; v[3 * i + 1] = s.v.y; v[3 * i + 2] = s.v.z;
        w[3 * i] = s.w.x; w[3 * i + 1] = s.w.y; w[3 * i + 2] = s.w.z;
    }
    return 0;
}

// Gradient of L(x_T, v_T) through nsteps steps, given dL/dx_T and dL/dv_T
// ([3n] each, either may be NULL).  Outputs [3n] dL/dx0, dL/dv0, dL/dw0,
// [4n] dL/dq0, [n] dL/dinvMass, [3n] dL/dinvInertia, and dL/d world friction,
// dL/d world restitution.  Every pre-step state is kept (no checkpointing).
int adjh_grad(const NeWorldParams* p, const NeBodyArrays* b, int nsteps, uint32_t cap, const double* xb,
              const double* vb, double* gx, double* gq, double* gv, double* gw, double* ginvm, double* ginvi,
              double* gmu, double* ge) {
    HostWorld h;
    build(h, p, b);
    Run r;
    r.init(h, cap);
    const uint32_t n = h.n;
    std::vector<std::vector<adj::St>> pre(nsteps);
    std::vector<std::vector<unsigned long long>> wkp(nsteps + 1);
    std::vector<std::vector<double>> wip(nsteps + 1);
    int rd = 0;
    wkp[0] = std::vector<unsigned long long>(r.wk[0].begin(), r.wk[0].begin() + r.nw[0]);
    wip[0] = std::vector<double>(r.wi[0].begin(), r.wi[0].begin() + r.nw[0]);
    for (int k = 0; k < nsteps; ++k) {
        pre[k] = r.s;
        if (int e = r.step(h, rd, false)) return e;
        if (h.warm) rd ^= 1;
        wkp[k + 1] = std::vector<unsigned long long>(r.wk[rd].begin(), r.wk[rd].begin() + r.nw[rd]);
        wip[k + 1] = std::vector<double>(r.wi[rd].begin(), r.wi[rd].begin() + r.nw[rd]);
    }
    std::vector<adj::St> sb(n, adj::st_zero());
    for (uint32_t i = 0; i < n; ++i) {
        if (xb) sb[i].x = mk(xb[3 * i], xb[3 * i + 1], xb[3 * i + 2]);
        if (vb) sb[i].v = mk(vb[3 * i], vb[3 * i + 1], vb[3 * i + 2]);
    }
    std::vector<adj::Pb> pb(n);
    for (auto& e : pb) { e.invM = 0.0; e.invI = mk(0.0, 0.0, 0.0); }
    std::vector<adj::Cb> cbs(cap);
    std::vector<double> wob, wib;
    double mub = 0.0, eb = 0.0;
    for (int k = nsteps - 1; k >= 0; --k) {
        r.s = pre[k];
        r.w.s = r.s.data();
        // warm cache read by step k
        r.wk[0].assign(wkp[k].begin(), wkp[k].end());
        r.wi[0].assign(wip[k].begin(), wip[k].end());
        r.wk[0].resize(cap); r.wi[0].resize(cap);
        r.nw[0] = (uint32_t)wkp[k].size();
        r.w.wk_in = r.wk[0].data(); r.w.wi_in = r.wi[0].data(); r.w.nw_in = r.nw[0];
        r.w.wk_out = r.wk[1].data(); r.w.wi_out = r.wi[1].data();
        r.w.tape = r.tape.data();
        r.w.err = 0;
        wib.assign(cap, 0.0);
        adj::bwd_step(h.d, h.W, h.warm, r.w, sb.data(), wob.empty() ? nullptr : wob.data(), wib.data(), pb.data(),
                      cbs.data(), mub, eb, adj::Team{0, 1});
        if (r.w.err & (adj::kErrCapacity | adj::kErrUnsupported)) return r.w.err;
        wob = wib;   // the warm impulses read by step k were stored by step k - 1
    }
    for (uint32_t i = 0; i < n; ++i) {
        const adj::St& g = sb[i];
        gx[3 * i] = g.x.x; gx[3 * i + 1] = g.x.y; gx[3 * i + 2] = g.x.z;
        gq[4 * i] = g.q.w; gq[4 * i + 1] = g.q.x; gq[4 * i + 2] = g.q.y; gq[4 * i + 3] = g.q.z;
        gv[3 * i] = g.v.x; gv[3 * i + 1] = g.v.y; gv[3 * i + 2] = g.v.z;
        gw[3 * i] = g.w.x; gw[3 * i + 1] = g.w.y; gw[3 * i + 2] = g.w.z;
        ginvm[i] = pb[i].invM;
        ginvi[3 * i] = pb[i].invI.x; ginvi[3 * i + 1] = pb[i].invI.y; ginvi[3 * i + 2] = pb[i].invI.z;
    }
    *gmu = mub;
    *ge = eb;
    return 0;
}

}  // extern "C"
