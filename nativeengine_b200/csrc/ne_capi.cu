// ne_capi.cu -- the extern "C" boundary (include/ne_cuda.h): world lifecycle,
// host <-> HBM packing of the body arrays, and the step loop with its
// capacity retry.
//
// Capacities (pairs, surviving pairs, contacts) are data dependent.  Each step
// is enqueued with the current capacities; the kernels never write past them
// but raise ctl->abort and report the totals they needed.  The host then
// restores the pre-step snapshot that k_integrate took, grows the buffers and
// runs the step again -- so growth never changes the result, and steady-state
// steps cost one small device->host read of the control block.
#include <algorithm>
#include <type_traits>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ne_adjoint.cuh"
#include "ne_step.cuh"

namespace {

thread_local std::string g_last_error;

int set_err(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define NE_CUDA_TRY(expr)                                                                         \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return set_err(NE_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));     \
    } while (0)

template <typename T>
int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return set_err(NE_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return NE_OK;
}

template <typename T>
void dfree(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

inline size_t grow_to(uint64_t need) { return (size_t)(need + need / 2 + 4096); }

}  // namespace

namespace neb {
// Lets other translation units of the library report through ne_last_error().
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace neb

struct NeWorld {
    NeWorldParams p{};
    int device = 0;
    cudaStream_t stream = nullptr;
    neb::SideStream side{};               // small-island solve beside the big-island solvers
    cudaEvent_t dl_ev[6] = {};            // per-array completion of a state download
    uint32_t n = 0;
    neb::DevWorld d{};
    neb::Ctl* h_ctl = nullptr;   // pinned mirror of d.ctl
    // worlds of the batch (a single ne::World is a batch of one)
    uint32_t nworlds = 1;
    std::vector<NeWorldParams> wparams;   // [nworlds]
    std::vector<uint32_t> wbegin;         // [nworlds + 1] body ranges
    std::vector<double> h_bound;          // bounding radius per body (grid constants)
    std::vector<int> h_shape;
    std::vector<neb::WorldP> h_wp;
    neb::WorldP* d_wp = nullptr;
    uint32_t* d_bw = nullptr;             // world of each body
    long long* d_cext = nullptr;          // per-world cell extents
    int world_bits = 0;
    int any_grid = 0;
    std::vector<uint8_t> h_large;         // body flagged large (internal grid)
    uint32_t record = 0;                  // NE_RECORD_* flags
    int precision = NE_PRECISION_F64;
    uint32_t big_threads = 384;           // big-island solver launch shape
    uint32_t big_ctas_per_sm = 1;
    uint32_t big_team_max = 1;
    bool shape_chosen = false;            // set by the caller or the autotuner (else per upload)
    bool has_ext = false;                 // some body is a triangle mesh or a compound
    bool class_sort = false;              // some world holds two or more non-plane shapes
    size_t nverts = 0;                    // convex vertex pool entries on the device
    uint64_t Rcap = 0;                    // capacity of the recorded pair list
    int key_bits = 64;
    int num_sms = 148;
    // capacities (entries)
    uint64_t Scap = 0, Ccap = 0;
    size_t nverts_alloc = 0, nnc_alloc = 0, nplanes_alloc = 0;
    std::vector<double> h_invmass;   // for upload_state packing
    std::vector<neb::D4> stage;      // host packing buffer (uploads)
    double* pinned = nullptr;        // page-locked staging for per-step state traffic (host layout)
    size_t pinned_cap = 0;           // doubles
    NeStepStats stats{};
    uint64_t launches = 0;
    bool has_bodies = false;
    // CUDA graph of one step, replayed for batches of steps; valid while
    // make_args() returns the arguments it was captured with.
    bool graph_on = true;
    cudaGraphExec_t gexec = nullptr;
    neb::StepArgs gargs{};
    uint64_t g_launches = 0;              // kernels in the captured step
    // stage timing
    bool profile = false;
    cudaEvent_t ev[NE_NUM_STAGES + 1] = {};
    double stage_ms[NE_NUM_STAGES] = {};
    uint64_t stage_steps = 0;
};

namespace {

void free_body_arrays(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.pos); dfree(d.quat); dfree(d.vel); dfree(d.omg); dfree(d.frc); dfree(d.trq);
    dfree(d.inert); dfree(d.geom); dfree(d.ext); dfree(d.mat); dfree(d.meta); dfree(d.vrng); dfree(d.ncrng);
    dfree(d.s_pos); dfree(d.s_quat); dfree(d.s_vel); dfree(d.s_omg); dfree(d.s_frc); dfree(d.s_trq);
    dfree(d.key[0]); dfree(d.key[1]); dfree(d.val[0]); dfree(d.val[1]);
    dfree(d.bcnt); dfree(d.boff); dfree(d.parent); dfree(d.bdeg); dfree(d.bstart);
    dfree(d.cflag); dfree(d.crun); dfree(d.cstart); dfree(d.hkey); dfree(d.hval); dfree(d.bstage); dfree(d.srec);
    dfree(d.lrow); dfree(d.lmask);
    d.hsize = 0;
    d.lwords = 0;
    dfree(d.f_v); dfree(d.f_w); dfree(d.f_q); dfree(d.f_I); dfree(d.f_e); dfree(d.f_verts);
}

// FP32 copies of the body state and the convex vertex pool (FP32 form only).
int alloc_f32_bodies(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.f_v); dfree(d.f_w); dfree(d.f_q); dfree(d.f_I); dfree(d.f_e); dfree(d.f_verts);
    const size_t m = w->n ? w->n : 1;
    int rc;
    if ((rc = dalloc(&d.f_v, m)) || (rc = dalloc(&d.f_w, m)) || (rc = dalloc(&d.f_q, m)) ||
        (rc = dalloc(&d.f_I, m)) || (rc = dalloc(&d.f_e, m)) || (rc = dalloc(&d.f_verts, w->nverts ? w->nverts : 1)))
        return rc;
    neb::convert_verts_f32(d.verts, d.f_verts, (uint32_t)w->nverts, w->stream);
    NE_CUDA_TRY(cudaGetLastError());
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    return NE_OK;
}

void free_f32_cons(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.f_n); dfree(d.f_ra); dfree(d.f_rb); dfree(d.f_kn);
}

int alloc_f32_cons(NeWorld* w, uint64_t cap) {
    neb::DevWorld& d = w->d;
    free_f32_cons(w);
    int rc;
    if ((rc = dalloc(&d.f_n, cap)) || (rc = dalloc(&d.f_ra, cap)) || (rc = dalloc(&d.f_rb, cap)) ||
        (rc = dalloc(&d.f_kn, cap)))
        return rc;
    return NE_OK;
}

int alloc_rec(NeWorld* w, uint64_t cap) {
    neb::DevWorld& d = w->d;
    dfree(d.rec_i);
    dfree(d.rec_j);
    int rc;
    if ((rc = dalloc(&d.rec_i, cap)) || (rc = dalloc(&d.rec_j, cap))) return rc;
    w->Rcap = cap;
    return NE_OK;
}

void free_surv_arrays(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.si); dfree(d.sj); dfree(d.stage_j); dfree(d.ccnt); dfree(d.coff); dfree(d.cn); dfree(d.cp);
    dfree(d.sperm);
}

void free_con_arrays(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.ci); dfree(d.cj); dfree(d.cslot); dfree(d.con_n); dfree(d.con_ra); dfree(d.con_rb); dfree(d.con_p);
    dfree(d.con_imp); dfree(d.ilab[0]); dfree(d.ilab[1]); dfree(d.iord[0]); dfree(d.iord[1]); dfree(d.iflag);
    dfree(d.ioff); dfree(d.istart); dfree(d.big); dfree(d.con_kn);
    dfree(d.rkey[0]); dfree(d.rkey[1]); dfree(d.rval[0]); dfree(d.rval[1]); dfree(d.crank);
    dfree(d.bcnt10); dfree(d.bq10); dfree(d.bctl); dfree(d.bteam); dfree(d.brec); dfree(d.bigs);
    dfree(d.ext_cn); dfree(d.ext_cp);
    free_f32_cons(w);
}

int alloc_scratch(NeWorld* w) {
    neb::DevWorld& d = w->d;
    dfree(d.hist);
    dfree(d.tsum);
    uint64_t sortn = std::max<uint64_t>(std::max<uint64_t>(w->n, 2 * w->Ccap), w->Scap);
    size_t hw = neb::radix_hist_words((uint32_t)sortn);
    uint64_t scann = std::max<uint64_t>(w->Scap, std::max<uint64_t>(hw, sortn));
    int rc;
    if ((rc = dalloc(&d.hist, hw)) != NE_OK) return rc;
    const size_t tw = neb::scan_tsum_words((uint32_t)scann) + 8;
    if ((rc = dalloc(&d.tsum, tw)) != NE_OK) return rc;
    NE_CUDA_TRY(cudaMemset(d.tsum, 0, tw * sizeof(uint32_t)));   // scan tile states start empty
    return NE_OK;
}

int alloc_surv(NeWorld* w, uint64_t cap) {
    free_surv_arrays(w);
    neb::DevWorld& d = w->d;
    int rc;
    if ((rc = dalloc(&d.si, cap)) || (rc = dalloc(&d.sj, cap)) || (rc = dalloc(&d.stage_j, cap)) ||
        (rc = dalloc(&d.ccnt, cap)) ||
        (rc = dalloc(&d.coff, cap)) || (rc = dalloc(&d.sperm, cap)) ||
        (rc = dalloc(&d.cn, 4 * cap)) || (rc = dalloc(&d.cp, 4 * cap)))
        return rc;
    w->Scap = cap;
    return NE_OK;
}

// Contact-sized arrays.  The warm cache survives a resize: the buffer holding
// the previous step is copied into the new allocation.
int alloc_cons(NeWorld* w, uint64_t cap) {
    neb::DevWorld& d = w->d;
    free_con_arrays(w);
    int rc;
    if ((rc = dalloc(&d.ci, cap)) || (rc = dalloc(&d.cj, cap)) || (rc = dalloc(&d.cslot, cap)) ||
        (rc = dalloc(&d.con_n, cap)) || (rc = dalloc(&d.con_ra, cap)) || (rc = dalloc(&d.con_rb, cap)) ||
        (rc = dalloc(&d.con_p, cap)) || (rc = dalloc(&d.con_imp, cap)) || (rc = dalloc(&d.ilab[0], cap)) ||
        (rc = dalloc(&d.ilab[1], cap)) || (rc = dalloc(&d.iord[0], cap)) || (rc = dalloc(&d.iord[1], cap)) ||
        (rc = dalloc(&d.iflag, cap)) || (rc = dalloc(&d.ioff, cap)) || (rc = dalloc(&d.istart, cap + 1)) ||
        (rc = dalloc(&d.big, cap)) || (rc = dalloc(&d.con_kn, cap)) || (rc = dalloc(&d.rkey[0], 2 * cap)) ||
        (rc = dalloc(&d.rkey[1], 2 * cap)) || (rc = dalloc(&d.rval[0], 2 * cap)) ||
        (rc = dalloc(&d.rval[1], 2 * cap)) || (rc = dalloc(&d.crank, 2 * cap)) ||
        (rc = dalloc(&d.bcnt10, 10 * cap)) || (rc = dalloc(&d.bq10, 10 * cap)) ||
        (rc = dalloc(&d.bctl, cap / neb::kBigIsland + 1)) || (rc = dalloc(&d.bteam, cap / neb::kBigIsland + 2)) ||
        (rc = dalloc(&d.brec, 2 * cap)) || (rc = dalloc(&d.bigs, cap / neb::kBigIsland + 1)) ||
        (rc = dalloc(&d.ext_cn, cap)) || (rc = dalloc(&d.ext_cp, cap)))
        return rc;
    if (w->precision == NE_PRECISION_F32 && (rc = alloc_f32_cons(w, cap))) return rc;
    unsigned long long* nk[2] = {nullptr, nullptr};
    double* ni[2] = {nullptr, nullptr};
    for (int b = 0; b < 2; ++b) {
        if ((rc = dalloc(&nk[b], cap)) || (rc = dalloc(&ni[b], cap))) return rc;
    }
    if (d.wkey[0]) {
        NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
        NE_CUDA_TRY(cudaMemcpy(w->h_ctl, d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost));
        const uint32_t ws = w->h_ctl->wsel;
        const uint64_t cnt = std::min<uint64_t>(w->h_ctl->wcount[ws], cap);
        if (cnt) {
            NE_CUDA_TRY(cudaMemcpy(nk[ws], d.wkey[ws], cnt * sizeof(unsigned long long), cudaMemcpyDeviceToDevice));
            NE_CUDA_TRY(cudaMemcpy(ni[ws], d.wimp[ws], cnt * sizeof(double), cudaMemcpyDeviceToDevice));
        }
    }
    for (int b = 0; b < 2; ++b) {
        dfree(d.wkey[b]);
        dfree(d.wimp[b]);
        d.wkey[b] = nk[b];
        d.wimp[b] = ni[b];
    }
    w->Ccap = cap;
    return NE_OK;
}

neb::StepArgs make_args(const NeWorld* w) {
    neb::StepArgs a;
    std::memset(&a, 0, sizeof a);   // padding too: captured arguments are compared bytewise
    a.d = w->d;
    a.n = w->n;
    a.nworlds = w->nworlds;
    a.world_bits = w->world_bits;
    a.wp = w->d_wp;
    a.bw = w->d_bw;
    a.cext = w->d_cext;
    a.key_bits = w->key_bits;
    a.any_grid = w->any_grid;
    a.warm = w->wparams.empty() ? (w->p.warm_start ? 1 : 0) : (w->wparams[0].warm_start ? 1 : 0);
    a.record = (w->record & NE_RECORD_PAIRS) ? 1 : 0;
    a.f32 = w->precision == NE_PRECISION_F32 ? 1 : 0;
    a.big_threads = (int)w->big_threads;
    a.big_ctas_per_sm = (int)w->big_ctas_per_sm;
    a.big_team_max = (int)w->big_team_max;
    a.Scap = w->Scap;
    a.Ccap = w->Ccap;
    a.Rcap = w->Rcap;
    a.num_sms = w->num_sms;
    a.local_cap = neb::kLocalCap;
    a.any_ext = w->has_ext ? 1 : 0;
    a.class_sort = w->class_sort ? 1 : 0;
    return a;
}

int check_params(const NeWorldParams* p) {
    if (!p) return set_err(NE_ERR_ARG, "params is NULL");
    if (p->restitution_combine < 0 || p->restitution_combine > 4 || p->friction_combine < 0 || p->friction_combine > 4)
        return set_err(NE_ERR_ARG, "combine mode out of range");
    if (p->sleep_enabled) return set_err(NE_ERR_UNSUPPORTED, "sleeping is not on the device path");
    if (p->n_distance_joints || p->n_joints) return set_err(NE_ERR_UNSUPPORTED, "joints are not on the device path");
    return NE_OK;
}

// Per-world constants of World::broadphasePairs() (src/world.cpp:427-457):
// cell = 2 * max bounding radius over the world's grid bodies, brute force
// below 64 bodies, periodic cell counts nc = max(1, floor(L / cell)); the
// range of the world's planes in the (ascending) plane list; and the bits the
// cell-key sort needs when every grid world is periodic.
int derive_worlds(NeWorld* w, const std::vector<uint32_t>& planes) {
    const uint32_t nw = w->nworlds;
    std::vector<uint32_t> xlist;
    for (uint32_t i = 0; i < w->n; ++i)
        if (w->h_shape[i] == NE_SHAPE_PLANE || w->h_shape[i] == NE_SHAPE_MESH || w->h_large[i]) xlist.push_back(i);
    size_t xk = 0;
    w->h_wp.assign(nw, neb::WorldP{});
    w->any_grid = 0;
    int local_bits = 0;
    bool all_periodic = true;
    size_t pk = 0;
    for (uint32_t k = 0; k < nw; ++k) {
        const NeWorldParams& p = w->wparams[k];
        neb::WorldP& W = w->h_wp[k];
        W.dom.half = p.half;
        W.dom.periodic = p.periodic ? 1 : 0;
        W.dt = p.dt;
        W.restitution = p.restitution;
        W.friction = p.friction;
        W.beta = p.contact_beta;
        W.g = neb::mk(p.gravity[0], p.gravity[1], p.gravity[2]);
        W.rcomb = p.restitution_combine;
        W.fcomb = p.friction_combine;
        W.open_boundary = p.open_boundary ? 1 : 0;
        W.begin = w->wbegin[k];
        W.end = w->wbegin[k + 1];
        double maxR = 0.0;
        for (uint32_t i = W.begin; i < W.end; ++i) {
            if (w->h_shape[i] == NE_SHAPE_PLANE || w->h_shape[i] == NE_SHAPE_MESH) continue;
            maxR = (maxR < w->h_bound[i]) ? w->h_bound[i] : maxR;
        }
        W.cell = 2.0 * maxR;
        W.brute = (p.force_brute_force || (W.end - W.begin) < 64 || W.cell < 1e-9) ? 1 : 0;
        W.nc[0] = W.nc[1] = W.nc[2] = 1;
        if (p.periodic && !W.brute) {
            const double L = 2.0 * p.half;
            for (int a = 0; a < 3; ++a) {
                long long m = (long long)(int)std::floor(L / W.cell);
                W.nc[a] = m < 1 ? 1 : m;
            }
        }
        while (pk < planes.size() && planes[pk] < W.begin) ++pk;
        W.plane_begin = (uint32_t)pk;
        while (pk < planes.size() && planes[pk] < W.end) ++pk;
        W.plane_end = (uint32_t)pk;
        // Internal grid: large bodies are paired with everyone (like planes),
        // so the cell only has to cover the remaining bodies.  The cell exceeds
        // every bounding-sphere distance the cull keeps ((ra + rb)(1 + 1e-9) +
        // 1e-9), so each pair the cull can keep is still a candidate and the
        // surviving pairs -- hence contacts and results -- are those of the
        // reference's grid.
        double maxS = 0.0;
        for (uint32_t i = W.begin; i < W.end; ++i) {
            if (w->h_shape[i] == NE_SHAPE_PLANE || w->h_shape[i] == NE_SHAPE_MESH || w->h_large[i]) continue;
            maxS = (maxS < w->h_bound[i]) ? w->h_bound[i] : maxS;
        }
        W.fcell = 2.0 * maxS * (1.0 + 1e-8) + 1e-8;
        W.fbrute = (W.brute || maxS <= 0.0) ? 1 : 0;
        W.fnc[0] = W.fnc[1] = W.fnc[2] = 1;
        if (p.periodic && !W.fbrute) {
            const double L = 2.0 * p.half;
            for (int a = 0; a < 3; ++a) {
                long long m = (long long)std::floor(L / W.fcell);
                W.fnc[a] = m < 1 ? 1 : m;
            }
        }
        while (xk < xlist.size() && xlist[xk] < W.begin) ++xk;
        W.xl_begin = (uint32_t)xk;
        while (xk < xlist.size() && xlist[xk] < W.end) ++xk;
        W.xl_end = (uint32_t)xk;
        if (!W.fbrute && p.periodic) {
            int bits = 0;
            for (int a = 0; a < 3; ++a) {
                long long m = W.fnc[a];
                int b = 0;
                if (m > (1ll << 21)) b = 21;
                else while ((1ll << b) < m) ++b;
                bits += b;
            }
            local_bits = std::max(local_bits, bits);
        }
        if (!W.brute || !W.fbrute) {
            w->any_grid = 1;
            if (!p.periodic) all_periodic = false;
            int bits = 0;
            for (int a = 0; a < 3; ++a) {
                long long m = W.nc[a];
                int b = 0;
                if (m > (1ll << 21)) b = 21;
                else while ((1ll << b) < m) ++b;
                bits += b;
            }
            local_bits = std::max(local_bits, bits);
        }
    }
    w->world_bits = 0;
    while ((1u << w->world_bits) < nw) ++w->world_bits;
    w->key_bits = all_periodic ? ((w->world_bits + local_bits + 1 + 7) / 8) * 8 : 64;
    if (w->key_bits > 64) return set_err(NE_ERR_CAPACITY, "cell keys of this batch need more than 64 bits");
    neb::DevWorld& d = w->d;
    (void)d;
    dfree(w->d_wp);
    dfree(w->d_cext);
    int rc;
    if ((rc = dalloc(&w->d_wp, nw)) || (rc = dalloc(&w->d_cext, 6 * (size_t)nw))) return rc;
    NE_CUDA_TRY(cudaMemcpy(w->d_wp, w->h_wp.data(), nw * sizeof(neb::WorldP), cudaMemcpyHostToDevice));
    dfree(w->d.xlist);
    if ((rc = dalloc(&w->d.xlist, xlist.size() ? xlist.size() : 1))) return rc;
    if (!xlist.empty())
        NE_CUDA_TRY(cudaMemcpy(w->d.xlist, xlist.data(), xlist.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return NE_OK;
}

}  // namespace

extern "C" {

void ne_world_params_default(NeWorldParams* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->half = 12.0;
    p->periodic = 0;
    p->open_boundary = 0;
    p->dt = 1.0 / 120.0;
    p->restitution = 1.0;
    p->friction = 0.0;
    p->contact_beta = 0.2;
    p->restitution_combine = NE_COMBINE_MAX;
    p->friction_combine = NE_COMBINE_GEOMETRIC_MEAN;
    p->warm_start = 1;
    p->force_brute_force = 0;
    p->capture_contacts = 0;
    p->sleep_enabled = 0;
    p->sleep_lin_vel = 0.05;
    p->sleep_ang_vel = 0.05;
    p->sleep_time = 0.5;
    p->wake_vel = 0.5;
}

const char* ne_status_string(int s) {
    switch (s) {
        case NE_OK: return "ok";
        case NE_ERR_ARG: return "invalid argument";
        case NE_ERR_CUDA: return "CUDA error";
        case NE_ERR_CAPACITY: return "device capacity exceeded";
        case NE_ERR_UNSUPPORTED: return "feature not supported on the device path";
        case NE_ERR_TIMEOUT: return "device wait timed out";
        case NE_ERR_NUMERIC: return "narrowphase budget exceeded";
        case NE_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char* ne_last_error(void) { return g_last_error.c_str(); }

int ne_world_create(const NeWorldParams* params, NeWorld** out) {
    if (!out) return set_err(NE_ERR_ARG, "out is NULL");
    *out = nullptr;
    int rc = check_params(params);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(NE_ERR_NO_DEVICE, "no CUDA device");
    NeWorld* w = new NeWorld();
    w->p = *params;
    NE_CUDA_TRY(cudaGetDevice(&w->device));
    NE_CUDA_TRY(cudaDeviceGetAttribute(&w->num_sms, cudaDevAttrMultiProcessorCount, w->device));
    NE_CUDA_TRY(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    NE_CUDA_TRY(cudaStreamCreateWithFlags(&w->side.st2, cudaStreamNonBlocking));
    NE_CUDA_TRY(cudaEventCreateWithFlags(&w->side.fork, cudaEventDisableTiming));
    NE_CUDA_TRY(cudaEventCreateWithFlags(&w->side.join, cudaEventDisableTiming));
    for (int k = 0; k < 6; ++k) NE_CUDA_TRY(cudaEventCreateWithFlags(&w->dl_ev[k], cudaEventDisableTiming));
    neb::init_kernel_attrs();
    NE_CUDA_TRY(cudaGetLastError());
    NE_CUDA_TRY(cudaMallocHost((void**)&w->h_ctl, sizeof(neb::Ctl)));
    if ((rc = dalloc(&w->d.ctl, 1))) { ne_world_destroy(w); return rc; }
    std::memset(w->h_ctl, 0, sizeof(neb::Ctl));
    NE_CUDA_TRY(cudaMemcpy(w->d.ctl, w->h_ctl, sizeof(neb::Ctl), cudaMemcpyHostToDevice));
    *out = w;
    return NE_OK;
}

int ne_world_destroy(NeWorld* w) {
    if (!w) return NE_OK;
    if (w->stream) cudaStreamSynchronize(w->stream);
    free_body_arrays(w);
    free_surv_arrays(w);
    free_con_arrays(w);
    neb::DevWorld& d = w->d;
    dfree(d.verts); dfree(d.nc); dfree(d.planes); dfree(d.io);
    dfree(d.child); dfree(d.mesh_tab); dfree(d.mnode_lo); dfree(d.mnode_hi); dfree(d.mnode); dfree(d.morder);
    dfree(d.mtri); dfree(d.mvert);
    for (int b = 0; b < 2; ++b) { dfree(d.wkey[b]); dfree(d.wimp[b]); }
    dfree(d.hist); dfree(d.tsum); dfree(d.ctl);
    dfree(w->d_wp); dfree(w->d_bw); dfree(w->d_cext); dfree(d.xlist); dfree(d.rec_i); dfree(d.rec_j);
    if (w->h_ctl) cudaFreeHost(w->h_ctl);
    if (w->pinned) cudaFreeHost(w->pinned);
    for (int k = 0; k <= NE_NUM_STAGES; ++k)
        if (w->ev[k]) cudaEventDestroy(w->ev[k]);
    if (w->gexec) cudaGraphExecDestroy(w->gexec);
    if (w->side.st2) cudaStreamSynchronize(w->side.st2);
    if (w->side.fork) cudaEventDestroy(w->side.fork);
    if (w->side.join) cudaEventDestroy(w->side.join);
    for (int k = 0; k < 6; ++k)
        if (w->dl_ev[k]) cudaEventDestroy(w->dl_ev[k]);
    if (w->side.st2) cudaStreamDestroy(w->side.st2);
    if (w->stream) cudaStreamDestroy(w->stream);
    delete w;
    return NE_OK;
}

int ne_world_set_params(NeWorld* w, const NeWorldParams* params) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    int rc = check_params(params);
    if (rc) return rc;
    if (w->nworlds > 1) return set_err(NE_ERR_ARG, "a batch takes its parameters from ne_world_upload_batch");
    w->p = *params;
    if (w->has_bodies) {
        w->wparams.assign(1, *params);
        std::vector<uint32_t> planes;
        for (uint32_t i = 0; i < w->n; ++i)
            if (w->h_shape[i] == NE_SHAPE_PLANE || w->h_shape[i] == NE_SHAPE_MESH) planes.push_back(i);
        if ((rc = derive_worlds(w, planes))) return rc;
    }
    return NE_OK;
}

}  // extern "C"

namespace {

// Every index a BVH walk or a triangle reads stays inside its arrays.
int check_mesh(const NeMeshData& m) {
    if (m.n_tris && (!m.verts || !m.tris || !m.order)) return set_err(NE_ERR_ARG, "mesh arrays are NULL");
    if (m.n_nodes && (!m.node_lo || !m.node_hi || !m.node_left || !m.node_right || !m.node_start || !m.node_count))
        return set_err(NE_ERR_ARG, "mesh BVH arrays are NULL");
    for (uint32_t t = 0; t < 3 * m.n_tris; ++t)
        if (m.tris[t] < 0 || (uint32_t)m.tris[t] >= m.n_verts) return set_err(NE_ERR_ARG, "mesh vertex index out of range");
    for (uint32_t t = 0; t < m.n_tris; ++t)
        if (m.order[t] < 0 || (uint32_t)m.order[t] >= m.n_tris) return set_err(NE_ERR_ARG, "mesh triangle order out of range");
    for (uint32_t k = 0; k < m.n_nodes; ++k) {
        const int l = m.node_left[k], r = m.node_right[k];
        if (l < 0) {
            if (m.node_start[k] < 0 || m.node_count[k] < 0 ||
                (uint64_t)m.node_start[k] + (uint64_t)m.node_count[k] > m.n_tris)
                return set_err(NE_ERR_ARG, "mesh BVH leaf range out of bounds");
        } else if ((uint32_t)l >= m.n_nodes || r < 0 || (uint32_t)r >= m.n_nodes) {
            return set_err(NE_ERR_ARG, "mesh BVH child index out of range");
        }
    }
    return NE_OK;
}

// Compound children and meshes on the device.  Children: four records each,
// (localPos, shape), localRot (w,x,y,z), (radius, halfHeight, he.x, he.y),
// (he.z, 0, 0, 0).  Meshes: one table row per mesh (node, order, triangle and
// vertex offsets) over concatenated node, order, triangle and vertex arrays.
int upload_children_meshes(NeWorld* w, const NeBodyArrays* b) {
    neb::DevWorld& d = w->d;
    int rc;
    const uint32_t nc = b->child_shape ? b->n_children : 0;
    std::vector<neb::D4> ch(4 * (size_t)(nc ? nc : 1), neb::D4{0, 0, 0, 0});
    for (uint32_t k = 0; k < nc; ++k) {
        const double* lp = b->child_pos + 3 * (size_t)k;
        const double* lr = b->child_rot + 4 * (size_t)k;
        const double* he = b->child_half_extents + 3 * (size_t)k;
        ch[4 * k + 0] = neb::D4{lp[0], lp[1], lp[2], (double)b->child_shape[k]};
        ch[4 * k + 1] = neb::D4{lr[0], lr[1], lr[2], lr[3]};
        ch[4 * k + 2] = neb::D4{b->child_radius[k], b->child_half_height[k], he[0], he[1]};
        ch[4 * k + 3] = neb::D4{he[2], 0.0, 0.0, 0.0};
    }
    dfree(d.child);
    if ((rc = dalloc(&d.child, ch.size()))) return rc;
    NE_CUDA_TRY(cudaMemcpy(d.child, ch.data(), ch.size() * sizeof(neb::D4), cudaMemcpyHostToDevice));

    const uint32_t nm = b->meshes ? b->n_meshes : 0;
    std::vector<uint4> tab(nm ? nm : 1, make_uint4(0, 0, 0, 0));
    std::vector<neb::D4> lo, hi, vs;
    std::vector<int4> nodes, tris;
    std::vector<int> order;
    for (uint32_t k = 0; k < nm; ++k) {
        const NeMeshData& m = b->meshes[k];
        if ((rc = check_mesh(m))) return rc;
        tab[k] = make_uint4((uint32_t)nodes.size(), (uint32_t)order.size(), (uint32_t)tris.size(), (uint32_t)vs.size());
        for (uint32_t t = 0; t < m.n_nodes; ++t) {
            lo.push_back(neb::D4{m.node_lo[3 * t], m.node_lo[3 * t + 1], m.node_lo[3 * t + 2], 0.0});
            hi.push_back(neb::D4{m.node_hi[3 * t], m.node_hi[3 * t + 1], m.node_hi[3 * t + 2], 0.0});
            nodes.push_back(make_int4(m.node_left[t], m.node_right[t], m.node_start[t], m.node_count[t]));
        }
        for (uint32_t t = 0; t < m.n_tris; ++t) {
            order.push_back(m.order[t]);
            tris.push_back(make_int4(m.tris[3 * t], m.tris[3 * t + 1], m.tris[3 * t + 2], 0));
        }
        for (uint32_t v = 0; v < m.n_verts; ++v)
            vs.push_back(neb::D4{m.verts[3 * v], m.verts[3 * v + 1], m.verts[3 * v + 2], 0.0});
        if (!m.n_nodes) tab[k].x = 0xffffffffu;   // empty mesh: no walk
    }
    auto put = [&](auto*& dst, const auto& src) -> int {
        using T = typename std::decay_t<decltype(src)>::value_type;
        dfree(dst);
        const size_t cnt = src.empty() ? 1 : src.size();
        int r = dalloc(&dst, cnt);
        if (r) return r;
        if (!src.empty()) {
            cudaError_t e = cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return set_err(NE_ERR_CUDA, cudaGetErrorString(e));
        }
        return NE_OK;
    };
    if ((rc = put(d.mesh_tab, tab)) || (rc = put(d.mnode_lo, lo)) || (rc = put(d.mnode_hi, hi)) ||
        (rc = put(d.mnode, nodes)) || (rc = put(d.morder, order)) || (rc = put(d.mtri, tris)) ||
        (rc = put(d.mvert, vs)))
        return rc;
    return NE_OK;
}

// Bounding radius of a compound (src/body.hpp:147-155).
double compound_bound(const NeBodyArrays* b, uint32_t i) {
    double m = 0.0;
    for (uint32_t k = b->child_offset[i]; k < b->child_offset[i] + b->child_count[i]; ++k) {
        const int cs = b->child_shape[k];
        const double* he = b->child_half_extents + 3 * (size_t)k;
        const double* lp = b->child_pos + 3 * (size_t)k;
        const double cr = (cs == NE_SHAPE_SPHERE) ? b->child_radius[k]
                        : (cs == NE_SHAPE_BOX) ? std::sqrt(he[0] * he[0] + he[1] * he[1] + he[2] * he[2])
                                               : b->child_half_height[k] + b->child_radius[k];
        const double r = std::sqrt(lp[0] * lp[0] + lp[1] * lp[1] + lp[2] * lp[2]) + cr;
        m = std::max(m, r);
    }
    return m;
}

int upload_impl(NeWorld* w, const NeWorldParams* params, uint32_t nworlds, const uint32_t* wbegin,
                const NeBodyArrays* b) {
    const uint32_t n = b->n;
    if (nworlds == 0) return set_err(NE_ERR_ARG, "a batch needs at least one world");
    if (wbegin[0] != 0 || wbegin[nworlds] != n) return set_err(NE_ERR_ARG, "world ranges must cover [0, n)");
    for (uint32_t k = 0; k < nworlds; ++k) {
        if (wbegin[k + 1] < wbegin[k]) return set_err(NE_ERR_ARG, "world ranges must be ascending");
        int rc = check_params(&params[k]);
        if (rc) return rc;
        if ((params[k].warm_start != 0) != (params[0].warm_start != 0))
            return set_err(NE_ERR_ARG, "all worlds of a batch share one warm_start setting");
    }
    if (n > (1u << 24)) return set_err(NE_ERR_CAPACITY, "more than 2^24 bodies");
    if (n && (!b->x || !b->q || !b->v || !b->w || !b->inv_mass || !b->inv_inertia || !b->shape || !b->radius ||
              !b->half_height || !b->half_extents || !b->friction || !b->restitution || !b->linear_damping ||
              !b->angular_damping || !b->gravity_scale || !b->layer || !b->mask || !b->flags))
        return set_err(NE_ERR_ARG, "a required body array is NULL");
    for (uint32_t i = 0; i < n; ++i) {
        const int s = b->shape[i];
        if (s < 0 || s > NE_SHAPE_COMPOUND) return set_err(NE_ERR_ARG, "shape tag out of range");
        if (s == NE_SHAPE_COMPOUND) {
            if (!b->child_offset || !b->child_count || !b->child_shape || !b->child_pos || !b->child_rot ||
                !b->child_radius || !b->child_half_height || !b->child_half_extents)
                return set_err(NE_ERR_ARG, "compound body without child arrays");
            if ((uint64_t)b->child_offset[i] + b->child_count[i] > b->n_children)
                return set_err(NE_ERR_ARG, "compound child range out of bounds");
            for (uint32_t k = b->child_offset[i]; k < b->child_offset[i] + b->child_count[i]; ++k) {
                const int cs = b->child_shape[k];
                if (cs != NE_SHAPE_SPHERE && cs != NE_SHAPE_BOX && cs != NE_SHAPE_CYLINDER && cs != NE_SHAPE_CAPSULE)
                    return set_err(NE_ERR_ARG, "compound children are spheres, boxes, cylinders or capsules");
            }
        }
        if (s == NE_SHAPE_MESH) {
            if (!b->mesh_index || !b->meshes || b->mesh_index[i] >= b->n_meshes)
                return set_err(NE_ERR_ARG, "mesh body without a valid mesh");
        }
        if (s == NE_SHAPE_CONVEX) {
            if (!b->verts || !b->vert_offset || !b->vert_count) return set_err(NE_ERR_ARG, "convex body without vertices");
            if ((uint64_t)b->vert_offset[i] + b->vert_count[i] > b->n_verts)
                return set_err(NE_ERR_ARG, "convex vertex range out of bounds");
        }
        if ((b->flags[i] & NE_BODY_CCD) && b->inv_mass[i] > 0.0 && !(b->flags[i] & NE_BODY_SLEEPING))
            return set_err(NE_ERR_UNSUPPORTED, "continuous collision is not on the device path");
        if (b->nocollide_count && b->nocollide_count[i]) {
            if (!b->nocollide || !b->nocollide_offset ||
                (uint64_t)b->nocollide_offset[i] + b->nocollide_count[i] > b->n_nocollide)
                return set_err(NE_ERR_ARG, "noCollide range out of bounds");
        }
    }
    NE_CUDA_TRY(cudaSetDevice(w->device));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    int rc;
    neb::DevWorld& d = w->d;
    if (n != w->n || !d.pos) {
        free_body_arrays(w);
        w->n = n;
        const size_t m = n ? n : 1;
        if ((rc = dalloc(&d.pos, m)) || (rc = dalloc(&d.quat, m)) || (rc = dalloc(&d.vel, m)) ||
            (rc = dalloc(&d.omg, m)) || (rc = dalloc(&d.frc, m)) || (rc = dalloc(&d.trq, m)) ||
            (rc = dalloc(&d.inert, m)) || (rc = dalloc(&d.geom, m)) || (rc = dalloc(&d.ext, m)) ||
            (rc = dalloc(&d.mat, m)) || (rc = dalloc(&d.meta, m)) || (rc = dalloc(&d.vrng, m)) ||
            (rc = dalloc(&d.ncrng, m)) || (rc = dalloc(&d.s_pos, m)) || (rc = dalloc(&d.s_quat, m)) ||
            (rc = dalloc(&d.s_vel, m)) || (rc = dalloc(&d.s_omg, m)) || (rc = dalloc(&d.s_frc, m)) ||
            (rc = dalloc(&d.s_trq, m)) || (rc = dalloc(&d.key[0], m)) || (rc = dalloc(&d.key[1], m)) ||
            (rc = dalloc(&d.val[0], m)) || (rc = dalloc(&d.val[1], m)) || (rc = dalloc(&d.bcnt, m)) ||
            (rc = dalloc(&d.boff, m)) || (rc = dalloc(&d.parent, m)) || (rc = dalloc(&d.bdeg, m)) ||
            (rc = dalloc(&d.bstart, m)) || (rc = dalloc(&d.cflag, m)) || (rc = dalloc(&d.crun, m)) ||
            (rc = dalloc(&d.cstart, m + 1)) || (rc = dalloc(&d.bstage, m)) || (rc = dalloc(&d.srec, m)))
            return rc;
        // Cell hash table: a power of two >= 2n slots (load factor <= 1/2).
        uint32_t hs = 64;
        while (hs < 2 * m) hs <<= 1;
        if ((rc = dalloc(&d.hkey, hs)) || (rc = dalloc(&d.hval, hs))) return rc;
        d.hsize = hs;
        const size_t lw = (m + 31) / 32 + 1;
        if ((rc = dalloc(&d.lrow, neb::kLongRows)) || (rc = dalloc(&d.lmask, neb::kLongRows * lw))) return rc;
        d.lwords = (uint32_t)lw;
    }
    // Pack the host arrays into the 32-byte device records.
    std::vector<neb::D4>& st = w->stage;
    st.assign(n ? n : 1, neb::D4{0, 0, 0, 0});
    auto put = [&](neb::D4* dst) -> int {
        if (!n) return NE_OK;
        cudaError_t e = cudaMemcpy(dst, st.data(), n * sizeof(neb::D4), cudaMemcpyHostToDevice);
        return e == cudaSuccess ? NE_OK : set_err(NE_ERR_CUDA, cudaGetErrorString(e));
    };
    auto v3 = [&](const double* a, uint32_t i, double wv) { return neb::D4{a[3 * i], a[3 * i + 1], a[3 * i + 2], wv}; };
    w->h_invmass.assign(b->inv_mass, b->inv_mass + n);
    for (uint32_t i = 0; i < n; ++i) st[i] = v3(b->x, i, b->inv_mass[i]);
    if ((rc = put(d.pos))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = neb::D4{b->q[4 * i], b->q[4 * i + 1], b->q[4 * i + 2], b->q[4 * i + 3]};
    if ((rc = put(d.quat))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = v3(b->v, i, 0.0);
    if ((rc = put(d.vel))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = v3(b->w, i, 0.0);
    if ((rc = put(d.omg))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = b->force ? v3(b->force, i, 0.0) : neb::D4{0, 0, 0, 0};
    if ((rc = put(d.frc))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = b->torque ? v3(b->torque, i, 0.0) : neb::D4{0, 0, 0, 0};
    if ((rc = put(d.trq))) return rc;

    // Convex vertex pool (needed for bounding radii below).
    std::vector<neb::D4> verts(b->n_verts ? b->n_verts : 1);
    for (uint32_t k = 0; k < b->n_verts; ++k) verts[k] = v3(b->verts, k, 0.0);
    dfree(d.verts);
    if ((rc = dalloc(&d.verts, verts.size()))) return rc;
    NE_CUDA_TRY(cudaMemcpy(d.verts, verts.data(), verts.size() * sizeof(neb::D4), cudaMemcpyHostToDevice));
    w->nverts = b->n_verts;
    if (w->precision == NE_PRECISION_F32 && (rc = alloc_f32_bodies(w))) return rc;
    if ((rc = upload_children_meshes(w, b))) return rc;
    w->has_ext = false;
    for (uint32_t i = 0; i < n; ++i)
        if (b->shape[i] == NE_SHAPE_MESH || b->shape[i] == NE_SHAPE_COMPOUND) w->has_ext = true;
    // A world of one shape (and planes) gives one kind of narrowphase work;
    // several shapes mix analytic and GJK/EPA pairs in one warp.
    w->class_sort = false;
    for (uint32_t k = 0; k < nworlds && !w->class_sort; ++k) {
        int first = -1;
        for (uint32_t i = wbegin[k]; i < wbegin[k + 1]; ++i) {
            if (b->shape[i] == NE_SHAPE_PLANE) continue;
            if (first < 0) first = b->shape[i];
            else if (b->shape[i] != first) { w->class_sort = true; break; }
        }
    }

    std::vector<double> boundR(n);
    std::vector<int> shapes(n);
    std::vector<uint32_t> planes;
    for (uint32_t i = 0; i < n; ++i) {
        const int s = b->shape[i];
        shapes[i] = s;
        const neb::V3 he = neb::mk(b->half_extents[3 * i], b->half_extents[3 * i + 1], b->half_extents[3 * i + 2]);
        const neb::D4* vp = (s == NE_SHAPE_CONVEX) ? verts.data() + b->vert_offset[i] : verts.data();
        const int nv = (s == NE_SHAPE_CONVEX) ? (int)b->vert_count[i] : 0;
        boundR[i] = (s == NE_SHAPE_COMPOUND) ? compound_bound(b, i)
                                             : neb::bounding_radius(s, b->radius[i], b->half_height[i], he, vp, nv);
        if (s == NE_SHAPE_PLANE || s == NE_SHAPE_MESH) planes.push_back(i);
        st[i] = v3(b->inv_inertia, i, boundR[i]);
    }
    if ((rc = put(d.inert))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = neb::D4{b->radius[i], b->half_height[i], b->gravity_scale[i], 0.0};
    if ((rc = put(d.geom))) return rc;
    for (uint32_t i = 0; i < n; ++i) st[i] = v3(b->half_extents, i, 0.0);
    if ((rc = put(d.ext))) return rc;
    for (uint32_t i = 0; i < n; ++i)
        st[i] = neb::D4{b->friction[i], b->restitution[i], b->linear_damping[i], b->angular_damping[i]};
    if ((rc = put(d.mat))) return rc;

    // Large bodies: bounding radius above 4x the world's 90th-percentile
    // radius, unless that would flag more than 5% of the world (then none).
    w->h_large.assign(n ? n : 1, 0);
    for (uint32_t k = 0; k < nworlds; ++k) {
        std::vector<double> r;
        for (uint32_t i = wbegin[k]; i < wbegin[k + 1]; ++i)
            if (shapes[i] != NE_SHAPE_PLANE && shapes[i] != NE_SHAPE_MESH) r.push_back(boundR[i]);
        if (r.size() < 8) continue;
        std::vector<double> sr = r;
        std::sort(sr.begin(), sr.end());
        const double split = 4.0 * sr[(size_t)(0.9 * (double)(sr.size() - 1))];
        size_t nlarge = 0;
        for (double x : r) nlarge += x > split;
        if (nlarge == 0 || nlarge > std::max<size_t>(4, r.size() / 20)) continue;
        for (uint32_t i = wbegin[k]; i < wbegin[k + 1]; ++i)
            if (shapes[i] != NE_SHAPE_PLANE && shapes[i] != NE_SHAPE_MESH && boundR[i] > split) w->h_large[i] = 1;
    }
    std::vector<uint4> meta(n ? n : 1);
    std::vector<uint2> vr(n ? n : 1), ncr(n ? n : 1);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t fl = b->flags[i] & 0xFFFFu;
        const bool mut = b->inv_mass[i] > 0.0 || b->inv_inertia[3 * i] != 0.0 || b->inv_inertia[3 * i + 1] != 0.0 ||
                         b->inv_inertia[3 * i + 2] != 0.0;
        if (mut) fl |= neb::kFlagMutable;
        if (w->h_large[i]) fl |= neb::kFlagLarge;
        meta[i] = make_uint4((uint32_t)b->shape[i], fl, b->layer[i], b->mask[i]);
        vr[i] = (b->shape[i] == NE_SHAPE_CONVEX)     ? make_uint2(b->vert_offset[i], b->vert_count[i])
                : (b->shape[i] == NE_SHAPE_COMPOUND) ? make_uint2(b->child_offset[i], b->child_count[i])
                : (b->shape[i] == NE_SHAPE_MESH)     ? make_uint2(b->mesh_index[i], 0)
                                                     : make_uint2(0, 0);
        ncr[i] = (b->nocollide_count && b->nocollide_count[i])
                     ? make_uint2(b->nocollide_offset[i], b->nocollide_count[i])
                     : make_uint2(0, 0);
    }
    if (n) {
        NE_CUDA_TRY(cudaMemcpy(d.meta, meta.data(), n * sizeof(uint4), cudaMemcpyHostToDevice));
        NE_CUDA_TRY(cudaMemcpy(d.vrng, vr.data(), n * sizeof(uint2), cudaMemcpyHostToDevice));
        NE_CUDA_TRY(cudaMemcpy(d.ncrng, ncr.data(), n * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    dfree(d.nc);
    if ((rc = dalloc(&d.nc, b->n_nocollide ? b->n_nocollide : 1))) return rc;
    if (b->n_nocollide && b->nocollide)
        NE_CUDA_TRY(cudaMemcpy(d.nc, b->nocollide, b->n_nocollide * sizeof(uint32_t), cudaMemcpyHostToDevice));
    dfree(d.planes);
    if ((rc = dalloc(&d.planes, planes.size() ? planes.size() : 1))) return rc;
    if (!planes.empty())
        NE_CUDA_TRY(cudaMemcpy(d.planes, planes.data(), planes.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));

    w->nworlds = nworlds;
    w->wparams.assign(params, params + nworlds);
    // Default solver shape until the caller sets or tunes one: one island
    // per SM in one wide CTA for a single world (its big island is a long
    // dependency chain), several narrower CTAs per SM for a batch (many
    // islands of a few hundred to a few thousand contacts).
    if (!w->shape_chosen) {
        w->big_threads = nworlds > 1 ? 128 : 384;
        w->big_ctas_per_sm = nworlds > 1 ? 3 : 1;
        w->big_team_max = 1;
    }
    w->wbegin.assign(wbegin, wbegin + nworlds + 1);
    w->h_bound = boundR;
    w->h_shape = shapes;
    std::vector<uint32_t> bw(n ? n : 1, 0);
    for (uint32_t k = 0; k < nworlds; ++k)
        for (uint32_t i = wbegin[k]; i < wbegin[k + 1]; ++i) bw[i] = k;
    dfree(w->d_bw);
    if ((rc = dalloc(&w->d_bw, bw.size()))) return rc;
    NE_CUDA_TRY(cudaMemcpy(w->d_bw, bw.data(), bw.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if ((rc = derive_worlds(w, planes))) return rc;

    // Initial capacities; they grow on demand (see ne_world_step).
    if (!w->Scap) {
        // Typical contact-rich scenes: ~4 surviving pairs and ~5 contacts per
        // body; larger needs grow (a re-run step).
        if ((rc = alloc_surv(w, std::max<uint64_t>(6ull * n, 1024)))) return rc;
        if ((rc = alloc_cons(w, std::max<uint64_t>(8ull * n, 1024)))) return rc;
    }
    if ((rc = alloc_scratch(w))) return rc;
    w->has_bodies = true;
    std::memset(&w->stats, 0, sizeof(w->stats));
    return NE_OK;
}

// Copies the pre-step snapshot k_integrate took back into the state: undoes
// the integration of a step that aborted.
int restore_pre_step(NeWorld* w) {
    const size_t bytes = (size_t)w->n * sizeof(neb::D4);
    neb::DevWorld& d = w->d;
    NE_CUDA_TRY(cudaMemcpyAsync(d.pos, d.s_pos, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaMemcpyAsync(d.quat, d.s_quat, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaMemcpyAsync(d.vel, d.s_vel, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaMemcpyAsync(d.omg, d.s_omg, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaMemcpyAsync(d.frc, d.s_frc, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaMemcpyAsync(d.trq, d.s_trq, bytes, cudaMemcpyDeviceToDevice, w->stream));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    return NE_OK;
}

// Grows what an aborted step (its counts in c) overflowed.
int grow_for(NeWorld* w, const neb::Ctl& c) {
    int rc = NE_OK;
    bool grew = false;
    if ((int)c.need_bits > w->key_bits) {
        w->key_bits = (((int)c.need_bits + 7) / 8) * 8;
        grew = true;
    }
    if (c.P_ref > w->Rcap && (w->record & NE_RECORD_PAIRS)) {
        if (c.P_ref > 0x7fffffffull) return set_err(NE_ERR_CAPACITY, "more than 2^31 recorded pairs");
        if ((rc = alloc_rec(w, grow_to(c.P_ref)))) return rc;
        grew = true;
    } else if (c.S > w->Scap) {
        if (c.S > 0x7fffffffull) return set_err(NE_ERR_CAPACITY, "more than 2^31 surviving pairs");
        if ((rc = alloc_surv(w, grow_to(c.S)))) return rc;
        grew = true;
    } else if (c.C > w->Ccap) {
        if (c.C > 0x7fffffffull) return set_err(NE_ERR_CAPACITY, "more than 2^31 contacts");
        if ((rc = alloc_cons(w, grow_to(c.C)))) return rc;
        grew = true;
    }
    if (!grew) return set_err(NE_ERR_CAPACITY, "step aborted without a growable cause");
    if ((rc = alloc_scratch(w))) return rc;
    ++w->stats.retries;
    return NE_OK;
}

// Counters of the last completed step (c holds its ctl block).
void take_step_counts(NeWorld* w, const neb::Ctl& c) {
    w->stats.pairs = (w->record & NE_RECORD_PAIRS) ? c.P_ref : c.P;
    w->stats.candidates = c.P;
    w->stats.survivors = c.S;
    w->stats.contacts = c.C;
    w->stats.islands = c.islands;
    w->stats.max_island = c.max_island;
}

// One step, launched kernel by kernel, re-run after growth until it fits.
int step_eager(NeWorld* w, int* status) {
    for (int attempt = 0;; ++attempt) {
        if (attempt > 16) return set_err(NE_ERR_CAPACITY, "step did not fit after repeated growth");
        neb::StepArgs a = make_args(w);
        neb::launch_step(a, w->stream, &w->launches, w->profile ? w->ev : nullptr, &w->side);
        NE_CUDA_TRY(cudaGetLastError());
        NE_CUDA_TRY(cudaMemcpyAsync(w->h_ctl, w->d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost, w->stream));
        NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
        const neb::Ctl& c = *w->h_ctl;
        if (!c.abort) break;
        int rc;
        if ((rc = restore_pre_step(w)) || (rc = grow_for(w, *w->h_ctl))) return rc;
    }
    const neb::Ctl& c = *w->h_ctl;
    if (w->profile) {
        for (int k = 0; k < NE_NUM_STAGES; ++k) {
            float ms = 0.f;
            NE_CUDA_TRY(cudaEventElapsedTime(&ms, w->ev[k], w->ev[k + 1]));
            w->stage_ms[k] += ms;
        }
        ++w->stage_steps;
    }
    // Shrink the cell-key sort to the bits this step needed.
    if (w->any_grid) {
        int kb = (((int)c.need_bits + 7) / 8) * 8;
        if (kb >= 8) w->key_bits = kb;
    }
    take_step_counts(w, c);
    w->stats.epa_cap_hits += c.epa_cap_hits;
    w->stats.steps += 1;
    if (c.solve_timeout) return set_err(NE_ERR_TIMEOUT, "a dataflow-solver dependency wait ran out");
    if (c.flags & 1u) *status = set_err(NE_ERR_NUMERIC, "an EPA or clipping budget was exceeded");
    return NE_OK;
}

// Steps per replayed batch: the host reads the control block once per batch.
constexpr uint32_t kGraphBatch = 64;

// Stage timing records events between kernels and recording builds a second
// pair list into a host-sized buffer: both step kernel by kernel.
bool graph_usable(const NeWorld* w) { return w->graph_on && !w->profile && !(w->record & NE_RECORD_PAIRS); }

// Up to min(want, kGraphBatch) steps by replaying the captured step (captured
// again first if the arguments changed).  *done = steps completed; *halted =
// the next step overflowed a buffer, its pre-step state has been restored
// and the buffer grown.
int step_graph_batch(NeWorld* w, uint32_t want, uint32_t* done, bool* halted, int* status) {
    neb::StepArgs a = make_args(w);
    a.sticky = 1;
    if (!w->gexec || std::memcmp(&a, &w->gargs, sizeof a) != 0) {
        if (w->gexec) {
            NE_CUDA_TRY(cudaGraphExecDestroy(w->gexec));
            w->gexec = nullptr;
        }
        uint64_t L = 0;
        cudaGraph_t g = nullptr;
        NE_CUDA_TRY(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
        neb::launch_step(a, w->stream, &L, nullptr, &w->side);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(w->stream, &g);
        if (le != cudaSuccess || ce != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return set_err(NE_ERR_CUDA, cudaGetErrorString(le != cudaSuccess ? le : ce));
        }
        const cudaError_t ie = cudaGraphInstantiate(&w->gexec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            w->gexec = nullptr;
            return set_err(NE_ERR_CUDA, cudaGetErrorString(ie));
        }
        w->gargs = a;
        w->g_launches = L;
        ++w->stats.graph_captures;
    }
    const uint32_t G = std::min(want, kGraphBatch);
    neb::launch_batch_begin(w->d.ctl, w->stream);
    ++w->launches;
    for (uint32_t k = 0; k < G; ++k) NE_CUDA_TRY(cudaGraphLaunch(w->gexec, w->stream));
    w->launches += (uint64_t)G * w->g_launches;
    NE_CUDA_TRY(cudaMemcpyAsync(w->h_ctl, w->d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost, w->stream));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    const neb::Ctl& c = *w->h_ctl;
    *done = c.steps_done;
    *halted = c.halt != 0;
    w->stats.steps += c.steps_done;
    w->stats.graph_steps += c.steps_done;
    w->stats.epa_cap_hits += c.acc_epa;
    if (!*halted) {
        take_step_counts(w, c);
        if (w->any_grid) {
            const int kb = (((int)c.need_max + 7) / 8) * 8;
            if (kb >= 8 && kb < w->key_bits) w->key_bits = kb;
        }
    }
    if (c.acc_timeout) return set_err(NE_ERR_TIMEOUT, "a dataflow-solver dependency wait ran out");
    if (c.acc_flags & 1u) *status = set_err(NE_ERR_NUMERIC, "an EPA or clipping budget was exceeded");
    if (*halted) {
        int rc;
        if ((rc = restore_pre_step(w)) || (rc = grow_for(w, *w->h_ctl))) return rc;
    }
    return NE_OK;
}

}  // namespace

extern "C" {

int ne_world_upload(NeWorld* w, const NeBodyArrays* b) {
    if (!w || !b) return set_err(NE_ERR_ARG, "NULL argument");
    const uint32_t range[2] = {0, b->n};
    return upload_impl(w, &w->p, 1, range, b);
}

int ne_world_upload_batch(NeWorld* w, const NeWorldParams* params, uint32_t nworlds, const uint32_t* world_begin,
                          const NeBodyArrays* b) {
    if (!w || !b || !params || !world_begin) return set_err(NE_ERR_ARG, "NULL argument");
    int rc = upload_impl(w, params, nworlds, world_begin, b);
    if (rc == NE_OK) w->p = params[0];
    return rc;
}

// Pinned host staging for per-step state traffic: 6 records per body
// (pos, quat, vel, omg, frc, trq), so each transfer is one async copy per
// array straight from page-locked memory.
// Page-locked host staging and a device block, both in the C-ABI's host
// layout (x[3n] | q[4n] | v[3n] | w[3n] | force[3n] | torque[3n]): a state
// transfer is one copy each way, and kernels scatter / gather the records.
static int ensure_io(NeWorld* w) {
    const size_t need = (size_t)19 * (w->n ? w->n : 1);   // doubles
    if (w->pinned_cap >= need && w->d.io) return NE_OK;
    if (w->pinned) cudaFreeHost(w->pinned);
    w->pinned = nullptr;
    w->pinned_cap = 0;
    dfree(w->d.io);
    NE_CUDA_TRY(cudaMallocHost((void**)&w->pinned, need * sizeof(double)));
    w->pinned_cap = need;
    int rc;
    if ((rc = dalloc(&w->d.io, need))) return rc;
    return NE_OK;
}

// memcpy split over up to 16 threads (at least 1 MiB each): one thread does
// not saturate the host memory bandwidth for the ~100 MB a large batch moves
// per step.
static void par_copy(void* dst, const void* src, size_t bytes) {
    const size_t kChunk = (size_t)1 << 20;
    const size_t hw = std::max<size_t>(1, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<size_t>(std::min<size_t>(16, hw), bytes / kChunk);
    if (nt < 2) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (bytes + nt - 1) / nt;
    for (unsigned t = 0; t < nt; ++t) {
        const size_t b0 = t * per, b1 = std::min(bytes, b0 + per);
        if (b0 >= b1) break;
        th.emplace_back([=] { std::memcpy((char*)dst + b0, (const char*)src + b0, b1 - b0); });
    }
    for (auto& t : th) t.join();
}

int ne_world_upload_state(NeWorld* w, const double* x, const double* q, const double* v, const double* wv) {
    if (!w || !w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    const uint32_t n = w->n;
    if (!n) return NE_OK;
    int rc;
    if ((rc = ensure_io(w))) return rc;
    NE_CUDA_TRY(cudaSetDevice(w->device));
    double* st = w->pinned;
    const size_t N = n;
    const double* src[4] = {x, q, v, wv};
    const size_t off[4] = {0, 3 * N, 7 * N, 10 * N};
    const size_t len[4] = {3 * N, 4 * N, 3 * N, 3 * N};
    uint32_t mask = 0;
    // Array by array: the transfer of one overlaps the staging copy of the next.
    for (int k = 0; k < 4; ++k) {
        if (!src[k]) continue;
        par_copy(st + off[k], src[k], len[k] * sizeof(double));
        NE_CUDA_TRY(cudaMemcpyAsync(w->d.io + off[k], st + off[k], len[k] * sizeof(double),
                                    cudaMemcpyHostToDevice, w->stream));
        mask |= 1u << k;
    }
    if (!mask) return NE_OK;
    neb::launch_unpack_state(w->d, n, w->d.io, mask, w->stream);
    NE_CUDA_TRY(cudaGetLastError());
    // The staging buffer is reused by the next call: wait for the copy.
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    return NE_OK;
}

int ne_world_download(NeWorld* w, NeBodyArrays* out) {
    if (!w || !out) return set_err(NE_ERR_ARG, "NULL argument");
    if (!w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    const uint32_t n = std::min(w->n, out->n);
    if (!n) return NE_OK;
    int rc;
    if ((rc = ensure_io(w))) return rc;
    NE_CUDA_TRY(cudaSetDevice(w->device));
    const size_t N = w->n;
    double* dst[6] = {out->x, out->q, out->v, out->w, out->force, out->torque};
    const size_t off[6] = {0, 3 * N, 7 * N, 10 * N, 13 * N, 16 * N};
    const size_t per[6] = {3, 4, 3, 3, 3, 3};
    uint32_t mask = 0;
    for (int k = 0; k < 6; ++k)
        if (dst[k]) mask |= 1u << k;
    if (!mask) return NE_OK;
    neb::launch_pack_state(w->d, w->n, w->d.io, mask, w->stream);
    NE_CUDA_TRY(cudaGetLastError());
    double* st = w->pinned;
    // Array by array: the copy out of one overlaps the transfer of the next.
    for (int k = 0; k < 6; ++k) {
        if (!dst[k]) continue;
        NE_CUDA_TRY(cudaMemcpyAsync(st + off[k], w->d.io + off[k], per[k] * N * sizeof(double),
                                    cudaMemcpyDeviceToHost, w->stream));
        NE_CUDA_TRY(cudaEventRecord(w->dl_ev[k], w->stream));
    }
    for (int k = 0; k < 6; ++k) {
        if (!dst[k]) continue;
        NE_CUDA_TRY(cudaEventSynchronize(w->dl_ev[k]));
        par_copy(dst[k], st + off[k], per[k] * (size_t)n * sizeof(double));
    }
    return NE_OK;
}

int ne_world_step(NeWorld* w, uint32_t nsteps) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    if (!w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    w->launches = 0;
    int status = NE_OK;
    if (w->n == 0) { w->stats.steps += nsteps; return NE_OK; }
    uint32_t s = 0;
    while (s < nsteps) {
        int rc;
        if (graph_usable(w)) {
            uint32_t done = 0;
            bool halted = false;
            if ((rc = step_graph_batch(w, nsteps - s, &done, &halted, &status))) return rc;
            s += done;
            if (!halted) continue;
            // The batch stopped at a step that overflowed a buffer: that
            // step's pre-step state is back in place and the buffer has
            // grown; it is taken once more outside the graph.
        }
        if ((rc = step_eager(w, &status))) return rc;
        ++s;
    }
    return status;
}

int ne_world_reset_warm_cache(NeWorld* w) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    NE_CUDA_TRY(cudaMemcpy(w->h_ctl, w->d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost));
    w->h_ctl->wcount[0] = w->h_ctl->wcount[1] = 0;
    NE_CUDA_TRY(cudaMemcpy(w->d.ctl, w->h_ctl, sizeof(neb::Ctl), cudaMemcpyHostToDevice));
    return NE_OK;
}

int ne_world_stats(const NeWorld* w, NeStepStats* out) {
    if (!w || !out) return set_err(NE_ERR_ARG, "NULL argument");
    *out = w->stats;
    return NE_OK;
}

int ne_world_pairs(NeWorld* w, uint32_t* pi, uint32_t* pj, uint64_t cap, uint64_t* count) {
    if (!w || !count) return set_err(NE_ERR_ARG, "NULL argument");
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    if (!(w->record & NE_RECORD_PAIRS))
        return set_err(NE_ERR_ARG, "pair recording is off (ne_world_set_record(world, NE_RECORD_PAIRS))");
    const uint64_t P = w->stats.pairs;
    *count = P;
    const uint64_t m = std::min(P, cap);
    if (m && pi) NE_CUDA_TRY(cudaMemcpy(pi, w->d.rec_i, m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (m && pj) NE_CUDA_TRY(cudaMemcpy(pj, w->d.rec_j, m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return NE_OK;
}

int ne_world_contacts(NeWorld* w, NeContactArrays* out, uint64_t cap, uint64_t* count) {
    if (!w || !out || !count) return set_err(NE_ERR_ARG, "NULL argument");
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    const uint64_t C = w->stats.contacts;
    *count = C;
    const uint64_t m = std::min(C, cap);
    if (!m) return NE_OK;
    neb::DevWorld& d = w->d;
    if (out->i) NE_CUDA_TRY(cudaMemcpy(out->i, d.ci, m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (out->j) NE_CUDA_TRY(cudaMemcpy(out->j, d.cj, m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (out->slot) NE_CUDA_TRY(cudaMemcpy(out->slot, d.cslot, m * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    std::vector<neb::D4> t(m);
    if (out->point) {
        NE_CUDA_TRY(cudaMemcpy(t.data(), d.con_p, m * sizeof(neb::D4), cudaMemcpyDeviceToHost));
        for (uint64_t k = 0; k < m; ++k) { out->point[3 * k] = t[k].x; out->point[3 * k + 1] = t[k].y; out->point[3 * k + 2] = t[k].z; }
    }
    if (out->normal || out->depth) {
        NE_CUDA_TRY(cudaMemcpy(t.data(), d.con_n, m * sizeof(neb::D4), cudaMemcpyDeviceToHost));
        for (uint64_t k = 0; k < m; ++k) {
            if (out->normal) { out->normal[3 * k] = t[k].x; out->normal[3 * k + 1] = t[k].y; out->normal[3 * k + 2] = t[k].z; }
            if (out->depth) out->depth[k] = t[k].w;
        }
    }
    if (out->n_imp || out->t_imp) {
        std::vector<double2> imp(m);
        NE_CUDA_TRY(cudaMemcpy(imp.data(), d.con_imp, m * sizeof(double2), cudaMemcpyDeviceToHost));
        for (uint64_t k = 0; k < m; ++k) {
            if (out->n_imp) out->n_imp[k] = imp[k].x;
            if (out->t_imp) out->t_imp[k] = imp[k].y;
        }
    }
    return NE_OK;
}

int ne_world_islands(NeWorld* w, uint32_t* label, uint32_t n) {
    if (!w || !label) return set_err(NE_ERR_ARG, "NULL argument");
    if (n > w->n) return set_err(NE_ERR_ARG, "n exceeds the body count");
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    std::vector<uint32_t> parent(w->n);
    if (w->n) NE_CUDA_TRY(cudaMemcpy(parent.data(), w->d.parent, w->n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t x = i;
        for (uint32_t guard = 0; parent[x] != x && guard < w->n; ++guard) x = parent[x];
        label[i] = x;
    }
    return NE_OK;
}

int ne_world_set_precision(NeWorld* w, int precision) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    if (precision != NE_PRECISION_F64 && precision != NE_PRECISION_F32)
        return set_err(NE_ERR_ARG, "precision must be NE_PRECISION_F64 or NE_PRECISION_F32");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    if (precision == w->precision) return NE_OK;
    w->precision = precision;
    int rc;
    if (precision == NE_PRECISION_F32) {
        if (w->d.pos && (rc = alloc_f32_bodies(w))) return rc;
        if (w->Ccap && (rc = alloc_f32_cons(w, w->Ccap))) return rc;
    } else {
        neb::DevWorld& d = w->d;
        dfree(d.f_v); dfree(d.f_w); dfree(d.f_q); dfree(d.f_I); dfree(d.f_e); dfree(d.f_verts);
        free_f32_cons(w);
    }
    return NE_OK;
}

int ne_world_set_solver_shape(NeWorld* w, const NeSolverShape* s) {
    if (!w || !s) return set_err(NE_ERR_ARG, "NULL argument");
    if (s->threads < 64 || s->threads > 512 || s->threads % 32 != 0)
        return set_err(NE_ERR_ARG, "solver threads must be a multiple of 32 in 64..512");
    if (s->ctas_per_sm < 1 || s->ctas_per_sm > 4) return set_err(NE_ERR_ARG, "solver ctas_per_sm must be 1..4");
    if (s->team_max < 1 || s->team_max > 64) return set_err(NE_ERR_ARG, "solver team_max must be 1..64");
    w->big_threads = s->threads;
    w->big_ctas_per_sm = s->ctas_per_sm;
    w->big_team_max = s->team_max;
    w->shape_chosen = true;
    return NE_OK;
}

int ne_world_get_solver_shape(const NeWorld* w, NeSolverShape* s) {
    if (!w || !s) return set_err(NE_ERR_ARG, "NULL argument");
    s->threads = w->big_threads;
    s->ctas_per_sm = w->big_ctas_per_sm;
    s->team_max = w->big_team_max;
    return NE_OK;
}

// Device copy of the state a step changes: the six body arrays and the warm
// cache (the buffer holding the last step's impulses).
struct Saved {
    neb::D4* body[6] = {};
    unsigned long long* wkey = nullptr;
    double* wimp = nullptr;
    uint32_t wsel = 0, wcount = 0;
    NeStepStats stats{};
};

static void saved_free(Saved& s) {
    for (auto*& p : s.body) dfree(p);
    dfree(s.wkey);
    dfree(s.wimp);
}

static int save_state(NeWorld* w, Saved& s) {
    neb::DevWorld& d = w->d;
    neb::D4* src[6] = {d.pos, d.quat, d.vel, d.omg, d.frc, d.trq};
    const size_t m = w->n ? w->n : 1;
    int rc;
    for (int k = 0; k < 6; ++k) {
        if ((rc = dalloc(&s.body[k], m))) return rc;
        NE_CUDA_TRY(cudaMemcpy(s.body[k], src[k], m * sizeof(neb::D4), cudaMemcpyDeviceToDevice));
    }
    NE_CUDA_TRY(cudaMemcpy(w->h_ctl, d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost));
    s.wsel = w->h_ctl->wsel;
    s.wcount = w->h_ctl->wcount[s.wsel];
    const size_t c = s.wcount ? s.wcount : 1;
    if ((rc = dalloc(&s.wkey, c)) || (rc = dalloc(&s.wimp, c))) return rc;
    if (s.wcount) {
        NE_CUDA_TRY(cudaMemcpy(s.wkey, d.wkey[s.wsel], s.wcount * sizeof(unsigned long long), cudaMemcpyDeviceToDevice));
        NE_CUDA_TRY(cudaMemcpy(s.wimp, d.wimp[s.wsel], s.wcount * sizeof(double), cudaMemcpyDeviceToDevice));
    }
    s.stats = w->stats;
    return NE_OK;
}

static int restore_state(NeWorld* w, const Saved& s) {
    neb::DevWorld& d = w->d;
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    neb::D4* dst[6] = {d.pos, d.quat, d.vel, d.omg, d.frc, d.trq};
    const size_t m = w->n ? w->n : 1;
    for (int k = 0; k < 6; ++k)
        NE_CUDA_TRY(cudaMemcpy(dst[k], s.body[k], m * sizeof(neb::D4), cudaMemcpyDeviceToDevice));
    // The warm buffers may have been reallocated (grown) meanwhile; the
    // saved entries always fit.
    if (s.wcount) {
        NE_CUDA_TRY(cudaMemcpy(d.wkey[s.wsel], s.wkey, s.wcount * sizeof(unsigned long long), cudaMemcpyDeviceToDevice));
        NE_CUDA_TRY(cudaMemcpy(d.wimp[s.wsel], s.wimp, s.wcount * sizeof(double), cudaMemcpyDeviceToDevice));
    }
    NE_CUDA_TRY(cudaMemcpy(w->h_ctl, d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost));
    w->h_ctl->wsel = s.wsel;
    w->h_ctl->wcount[s.wsel] = s.wcount;
    NE_CUDA_TRY(cudaMemcpy(d.ctl, w->h_ctl, sizeof(neb::Ctl), cudaMemcpyHostToDevice));
    w->stats = s.stats;
    return NE_OK;
}

}  // extern "C"

struct NeCheckpoint {
    const NeWorld* owner = nullptr;
    uint32_t n = 0;
    Saved s;
};

extern "C" {

int ne_world_checkpoint(NeWorld* w, NeCheckpoint** out) {
    if (!w || !out) return set_err(NE_ERR_ARG, "NULL argument");
    *out = nullptr;
    if (!w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    NeCheckpoint* ck = new NeCheckpoint;
    ck->owner = w;
    ck->n = w->n;
    int rc = save_state(w, ck->s);
    if (rc != NE_OK) {
        saved_free(ck->s);
        delete ck;
        return rc;
    }
    *out = ck;
    return NE_OK;
}

int ne_world_restore(NeWorld* w, const NeCheckpoint* ck) {
    if (!w || !ck) return set_err(NE_ERR_ARG, "NULL argument");
    if (ck->owner != w) return set_err(NE_ERR_ARG, "checkpoint belongs to another world");
    if (ck->n != w->n) return set_err(NE_ERR_ARG, "body count changed since the checkpoint");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    return restore_state(w, ck->s);
}

int ne_checkpoint_destroy(NeCheckpoint* ck) {
    if (!ck) return NE_OK;
    saved_free(ck->s);
    delete ck;
    return NE_OK;
}

}  // extern "C"

namespace {

// Device scratch of one stepBackward call, freed as a whole.
struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    int get(T** out, size_t count) {
        *out = nullptr;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
        if (e != cudaSuccess) return set_err(NE_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        ptrs.push_back(p);
        *out = static_cast<T*>(p);
        return NE_OK;
    }
};

// One attempt at stepBackward with contact capacity cap_factor * bodies + 64
// per world; *world_err receives the OR of the per-world error bits.
int step_backward_once(NeWorld* w, uint32_t nsteps, uint32_t K, const NeStateGrad* fin, NeParamGrad* out,
                       uint32_t cap_factor, int* world_err) {
    const uint32_t n = w->n, nw = w->nworlds;
    const uint32_t nck = (nsteps + K - 1) / K;
    std::vector<uint32_t> coff(nw), cap(nw);
    uint64_t CT = 0;
    for (uint32_t k = 0; k < nw; ++k) {
        const uint32_t nb = w->wbegin[k + 1] - w->wbegin[k];
        cap[k] = cap_factor * nb + 64;
        coff[k] = (uint32_t)CT;
        CT += cap[k];
    }
    if (CT > 0x7fffffffull) return set_err(NE_ERR_CAPACITY, "stepBackward contact scratch exceeds 2^31 entries");
    Scratch sc;
    neb::AdjArgs a{};
    a.d = w->d;
    a.wp = w->d_wp;
    a.nworlds = nw;
    a.n = n;
    a.warm = w->wparams.empty() ? (w->p.warm_start ? 1 : 0) : (w->wparams[0].warm_start ? 1 : 0);
    a.nsteps = nsteps;
    a.K = K;
    a.nck = nck;
    a.CT = (uint32_t)CT;
    NE_CUDA_TRY(cudaMemcpy(w->h_ctl, w->d.ctl, sizeof(neb::Ctl), cudaMemcpyDeviceToHost));
    const uint32_t ws = w->h_ctl->wsel;
    a.wk0 = w->d.wkey[ws];
    a.wi0 = w->d.wimp[ws];
    a.nw0 = a.warm ? w->h_ctl->wcount[ws] : 0;
    int rc;
    uint32_t *d_wbegin, *d_coff, *d_cap;
    const size_t nslot = 2 + (size_t)nck + K;
    if ((rc = sc.get(&d_wbegin, nw + 1)) || (rc = sc.get(&d_coff, nw)) || (rc = sc.get(&d_cap, nw)) ||
        (rc = sc.get(&a.S, n)) || (rc = sc.get(&a.S0, n)) || (rc = sc.get(&a.S1, n)) || (rc = sc.get(&a.SB, n)) ||
        (rc = sc.get(&a.UF, n)) ||
        (rc = sc.get(&a.CKS, (size_t)nck * n)) || (rc = sc.get(&a.SEGS, (size_t)K * n)) ||
        (rc = sc.get(&a.PB, n)) || (rc = sc.get(&a.CON, CT)) || (rc = sc.get(&a.CBS, CT)) ||
        (rc = sc.get(&a.TAPE, (size_t)9 * neb::adj::kTapeRec * CT)) || (rc = sc.get(&a.WK, nslot * CT)) ||
        (rc = sc.get(&a.WI, nslot * CT)) || (rc = sc.get(&a.WN, nslot * nw)) || (rc = sc.get(&a.WOB, CT)) ||
        (rc = sc.get(&a.WIB, CT)) || (rc = sc.get(&a.gx, 3 * (size_t)n)) || (rc = sc.get(&a.gq, 4 * (size_t)n)) ||
        (rc = sc.get(&a.gv, 3 * (size_t)n)) || (rc = sc.get(&a.gw, 3 * (size_t)n)) ||
        (rc = sc.get(&a.ginvm, n)) || (rc = sc.get(&a.ginvi, 3 * (size_t)n)) || (rc = sc.get(&a.gmu, nw)) ||
        (rc = sc.get(&a.ge, nw)) || (rc = sc.get(&a.err, nw)))
        return rc;
    NE_CUDA_TRY(cudaMemcpy(d_wbegin, w->wbegin.data(), (nw + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    NE_CUDA_TRY(cudaMemcpy(d_coff, coff.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice));
    NE_CUDA_TRY(cudaMemcpy(d_cap, cap.data(), nw * sizeof(uint32_t), cudaMemcpyHostToDevice));
    a.wbegin = d_wbegin;
    a.coff = d_coff;
    a.cap = d_cap;
    double *xb = nullptr, *vb = nullptr;
    if (fin && fin->x) {
        if ((rc = sc.get(&xb, 3 * (size_t)n))) return rc;
        NE_CUDA_TRY(cudaMemcpy(xb, fin->x, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (fin && fin->v) {
        if ((rc = sc.get(&vb, 3 * (size_t)n))) return rc;
        NE_CUDA_TRY(cudaMemcpy(vb, fin->v, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice));
    }
    a.xbar = xb;
    a.vbar = vb;
    neb::launch_adjoint(a, w->stream);
    NE_CUDA_TRY(cudaGetLastError());
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    std::vector<int> err(nw);
    NE_CUDA_TRY(cudaMemcpy(err.data(), a.err, nw * sizeof(int), cudaMemcpyDeviceToHost));
    *world_err = 0;
    for (int e : err) *world_err |= e;
    if (*world_err & (neb::adj::kErrCapacity | neb::adj::kErrUnsupported)) return NE_OK;
    if (!out) return NE_OK;
    auto fetch = [&](double* dst, const double* src, size_t count) -> int {
        if (!dst) return NE_OK;
        cudaError_t e = cudaMemcpy(dst, src, count * sizeof(double), cudaMemcpyDeviceToHost);
        return e == cudaSuccess ? NE_OK : set_err(NE_ERR_CUDA, cudaGetErrorString(e));
    };
    if ((rc = fetch(out->x, a.gx, 3 * (size_t)n)) || (rc = fetch(out->q, a.gq, 4 * (size_t)n)) ||
        (rc = fetch(out->v, a.gv, 3 * (size_t)n)) || (rc = fetch(out->w, a.gw, 3 * (size_t)n)) ||
        (rc = fetch(out->friction, a.gmu, nw)) || (rc = fetch(out->restitution, a.ge, nw)))
        return rc;
    std::vector<double> gim(n), gii(3 * (size_t)n);
    NE_CUDA_TRY(cudaMemcpy(gim.data(), a.ginvm, n * sizeof(double), cudaMemcpyDeviceToHost));
    NE_CUDA_TRY(cudaMemcpy(gii.data(), a.ginvi, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (out->inv_mass) std::memcpy(out->inv_mass, gim.data(), n * sizeof(double));
    if (out->inv_inertia) std::memcpy(out->inv_inertia, gii.data(), 3 * (size_t)n * sizeof(double));
    if (out->mass) {
        // mass m: invMass = 1/m, invInertia = invInertia_0 * m_0 / m (shape fixed), so
        // dL/dm = -(dL/dinvMass * invMass + dL/dinvInertia . invInertia) * invMass.
        std::vector<neb::D4> pos(n), inert(n);
        NE_CUDA_TRY(cudaMemcpy(pos.data(), w->d.pos, n * sizeof(neb::D4), cudaMemcpyDeviceToHost));
        NE_CUDA_TRY(cudaMemcpy(inert.data(), w->d.inert, n * sizeof(neb::D4), cudaMemcpyDeviceToHost));
        for (uint32_t i = 0; i < n; ++i) {
            const double im = pos[i].w;
            out->mass[i] = (im > 0.0) ? -(gim[i] * im + gii[3 * i] * inert[i].x + gii[3 * i + 1] * inert[i].y +
                                          gii[3 * i + 2] * inert[i].z) * im
                                      : 0.0;
        }
    }
    return NE_OK;
}

}  // namespace

extern "C" {

int ne_world_step_backward(NeWorld* w, uint32_t nsteps, uint32_t checkpoint_every, const NeStateGrad* final_grad,
                           NeParamGrad* out) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    if (!w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    if (nsteps == 0) return set_err(NE_ERR_ARG, "nsteps must be at least 1");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    const uint32_t K = (checkpoint_every == 0 || checkpoint_every > nsteps) ? nsteps : checkpoint_every;
    for (uint32_t factor = 8; factor <= 256; factor *= 2) {
        int werr = 0;
        int rc = step_backward_once(w, nsteps, K, final_grad, out, factor, &werr);
        if (rc != NE_OK) return rc;
        if (werr & neb::adj::kErrUnsupported)
            return set_err(NE_ERR_UNSUPPORTED, "stepBackward supports open or periodic worlds of planes, boxes and "
                                               "convex hulls (spheres with spheres and planes), <= 1024 bodies");
        if (werr & neb::adj::kErrCapacity) continue;
        if (werr & neb::adj::kErrNumeric)
            return set_err(NE_ERR_NUMERIC, "an EPA or clipping budget was exceeded in the recomputed trajectory");
        return NE_OK;
    }
    return set_err(NE_ERR_CAPACITY, "stepBackward contact scratch did not fit");
}

int ne_world_autotune(NeWorld* w, uint32_t steps, NeSolverShape* chosen) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    if (!w->has_bodies) return set_err(NE_ERR_ARG, "world has no bodies");
    NE_CUDA_TRY(cudaSetDevice(w->device));
    NE_CUDA_TRY(cudaStreamSynchronize(w->stream));
    if (steps == 0) steps = 1;
    static const NeSolverShape cand[] = {{512, 1, 1}, {384, 1, 1}, {256, 1, 1}, {256, 2, 1}, {128, 1, 1},
                                         {128, 2, 1}, {128, 3, 1}, {64, 3, 1}, {256, 1, 4}, {256, 1, 16},
                                         {128, 2, 8}};
    const bool prof = w->profile;
    w->profile = false;
    // Candidates change the launch shape, so each would re-capture the step
    // graph inside its timing: time them kernel by kernel instead.
    const bool graph = w->graph_on;
    w->graph_on = false;
    Saved s;
    int rc = save_state(w, s);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NeSolverShape best = {w->big_threads, w->big_ctas_per_sm, w->big_team_max};
    float best_ms = -1.0f;
    if (rc == NE_OK && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
        rc = set_err(NE_ERR_CUDA, "cudaEventCreate failed");
    // One untimed pass first, so buffer growth does not land in a timing.
    if (rc == NE_OK && (rc = ne_world_step(w, steps)) == NE_OK) rc = restore_state(w, s);
    for (const NeSolverShape& c : cand) {
        if (rc != NE_OK) break;
        w->big_threads = c.threads;
        w->big_ctas_per_sm = c.ctas_per_sm;
        w->big_team_max = c.team_max;
        cudaEventRecord(e0, w->stream);
        if ((rc = ne_world_step(w, steps)) != NE_OK) break;
        cudaEventRecord(e1, w->stream);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best_ms < 0.0f || ms < best_ms) { best_ms = ms; best = c; }
        rc = restore_state(w, s);
    }
    if (rc != NE_OK) restore_state(w, s);
    w->big_threads = best.threads;
    w->big_ctas_per_sm = best.ctas_per_sm;
    w->big_team_max = best.team_max;
    if (rc == NE_OK) w->shape_chosen = true;
    w->profile = prof;
    w->graph_on = graph;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    saved_free(s);
    if (rc == NE_OK && chosen) *chosen = best;
    return rc;
}

int ne_world_set_record(NeWorld* w, uint32_t flags) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    w->record = flags;
    if ((flags & NE_RECORD_PAIRS) && !w->d.rec_i) {
        int rc = alloc_rec(w, std::max<uint64_t>(16ull * w->n, 4096));
        if (rc) return rc;
    }
    return NE_OK;
}

int ne_world_profile(NeWorld* w, int enable) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    if (enable && !w->ev[0])
        for (int k = 0; k <= NE_NUM_STAGES; ++k) NE_CUDA_TRY(cudaEventCreate(&w->ev[k]));
    w->profile = enable != 0;
    for (int k = 0; k < NE_NUM_STAGES; ++k) w->stage_ms[k] = 0.0;
    w->stage_steps = 0;
    return NE_OK;
}

int ne_world_stage_times(NeWorld* w, double* ms, uint64_t* steps) {
    if (!w || !ms) return set_err(NE_ERR_ARG, "NULL argument");
    for (int k = 0; k < NE_NUM_STAGES; ++k) ms[k] = w->stage_ms[k];
    if (steps) *steps = w->stage_steps;
    return NE_OK;
}

const char* ne_stage_name(int k) {
    static const char* names[NE_NUM_STAGES] = {"integrate", "broadphase", "cull", "narrowphase",
                                               "constraints", "islands", "solve", "boundary"};
    return (k >= 0 && k < NE_NUM_STAGES) ? names[k] : "?";
}

int ne_world_stream(const NeWorld* w, void** stream) {
    if (!w || !stream) return set_err(NE_ERR_ARG, "NULL argument");
    *stream = (void*)w->stream;
    return NE_OK;
}

int ne_world_launch_count(const NeWorld* w, uint64_t* launches) {
    if (!w || !launches) return set_err(NE_ERR_ARG, "NULL argument");
    *launches = w->launches;
    return NE_OK;
}

int ne_world_set_graph(NeWorld* w, int enable) {
    if (!w) return set_err(NE_ERR_ARG, "world is NULL");
    w->graph_on = enable != 0;
    return NE_OK;
}

}  // extern "C"
