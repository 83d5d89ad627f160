// abi.cu -- the C ABI of include/lbflow.h: domain lifecycle, launches, host I/O.
//
// A domain owns its device memory: two population buffers (A/B, SoA planes),
// the per-node mask word, optional scalar buffers, the face-layer buffers used
// by anti-bounce-back and extrapolated wall velocities, the per-node moments of
// residual steps, and the FP64 partial-sum slots of the reductions.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_select.cuh>

#include "../../include/lbflow.h"
#include "dispatch.cuh"

using namespace lbf;

namespace {

thread_local std::string g_err;

lbf_status fail(lbf_status s, const std::string& msg) {
    g_err = msg;
    return s;
}

#define CK(call)                                                                                  \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return fail(e_ == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,               \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

int vs_q(int vs) { return vs == LBF_D2Q9 ? 9 : (vs == LBF_D3Q19 ? 19 : (vs == LBF_D3Q27 ? 27 : 0)); }
int vs_d(int vs) { return vs == LBF_D2Q9 ? 2 : 3; }
size_t st_bytes(int st) { return st == LBF_STORE_F64 ? 8 : (st == LBF_STORE_F32 ? 4 : 2); }
size_t rt_bytes(int st) { return st == LBF_STORE_F64 ? 8 : 4; }   // compute type

// ---- D3Q27 orthogonal moment basis (no reference counterpart: the reference's
// D3Q27 MRT is a placeholder, src/velocity_set/d3q27.rs:86 and
// src/velocity_set.rs:168).  Gram-Schmidt, plain dot product over the 27
// velocities, of 1; cx,cy,cz; |c|^2, 2cx^2-cy^2-cz^2, cy^2-cz^2, cxcy, cycz, cxcz;
// then the third- to sixth-order products of the squared and plain components.
double d3q27_monomial(int k, int x, int y, int z) {
    const double X = x, Y = y, Z = z, X2 = X * X, Y2 = Y * Y, Z2 = Z * Z;
    switch (k) {
        case 0: return 1.0;
        case 1: return X; case 2: return Y; case 3: return Z;
        case 4: return X2 + Y2 + Z2;
        case 5: return 2.0 * X2 - Y2 - Z2;
        case 6: return Y2 - Z2;
        case 7: return X * Y; case 8: return Y * Z; case 9: return X * Z;
        case 10: return X2 * Y; case 11: return X2 * Z; case 12: return Y2 * X;
        case 13: return Y2 * Z; case 14: return Z2 * X; case 15: return Z2 * Y;
        case 16: return X * Y * Z;
        case 17: return X2 * Y2; case 18: return X2 * Z2; case 19: return Y2 * Z2;
        case 20: return X2 * Y * Z; case 21: return Y2 * X * Z; case 22: return Z2 * X * Y;
        case 23: return X2 * Y2 * Z; case 24: return X2 * Z2 * Y; case 25: return Y2 * Z2 * X;
        default: return X2 * Y2 * Z2;
    }
}
void d3q27_basis(double* M, double* Minv) {
    using L = Lat<VS_D3Q27>;
    long double R[27][27];
    for (int k = 0; k < 27; ++k) {
        for (int i = 0; i < 27; ++i) R[k][i] = d3q27_monomial(k, L::c(i, 0), L::c(i, 1), L::c(i, 2));
        for (int j = 0; j < k; ++j) {
            long double num = 0, den = 0;
            for (int i = 0; i < 27; ++i) { num += R[k][i] * R[j][i]; den += R[j][i] * R[j][i]; }
            for (int i = 0; i < 27; ++i) R[k][i] -= num / den * R[j][i];
        }
    }
    for (int k = 0; k < 27; ++k) {
        double n2 = 0.0;
        for (int i = 0; i < 27; ++i) {
            M[k * 27 + i] = (double)R[k][i];
            n2 += M[k * 27 + i] * M[k * 27 + i];
        }
        for (int i = 0; i < 27; ++i) Minv[i * 27 + k] = M[k * 27 + i] / n2;
    }
}

template <int VS>
void tables_of(int* d, int* q, int* c, double* w, int* qbar, int* qfaces, int* normal, double* M, double* Minv) {
    using L = Lat<VS>;
    if (d) *d = L::D;
    if (q) *q = L::Q;
    for (int i = 0; i < L::Q; ++i) {
        if (c) for (int a = 0; a < 3; ++a) c[i * 3 + a] = a < L::D ? L::c(i, a) : 0;
        if (w) w[i] = L::w(i);
        if (qbar) qbar[i] = L::qbar(i);
    }
    for (int f = 0; f < 6; ++f) {
        int k = 0;
        for (int j = 0; j < 9; ++j) if (qfaces) qfaces[f * 9 + j] = -1;
        if (f < L::NF)
            for (int i = 0; i < L::Q; ++i)
                if (leaves<L>(i, f)) { if (qfaces) qfaces[f * 9 + k] = i; ++k; }
        if (normal) normal[f] = f < L::NF ? inward<L>(f) : -1;
    }
    if (VS == VS_D3Q27) {
        std::vector<double> m(729), mi(729);
        d3q27_basis(m.data(), mi.data());
        if (M) std::memcpy(M, m.data(), 729 * sizeof(double));
        if (Minv) std::memcpy(Minv, mi.data(), 729 * sizeof(double));
    } else {
        for (int k = 0; k < L::Q; ++k)
            for (int i = 0; i < L::Q; ++i) {
                if (M) M[k * L::Q + i] = L::M(k, i);
                if (Minv) Minv[k * L::Q + i] = mrt_inv<L>(k, i);
            }
    }
}

}  // namespace

// ============================================================== the domain
struct lbf_domain {
    lbf_domain_desc desc{};
    int vs = 0, q = 0, d = 0, st = 0, nfaces = 0;
    long long n[3] = {1, 1, 1};
    long long N = 0;
    unsigned long long n_fluid = 0, n_bb = 0;
    bool facebc = false, prepared = false, initialized = false;
    // host copies of the inputs (solid-node outputs, re-initialisation)
    std::vector<uint8_t> type;
    std::vector<double> rho0, u0, c0;
    double rho0u = 1.0, u0u[3] = {0, 0, 0}, c0u = 0.0;
    // scalar
    bool scalar = false;
    lbf_scalar_desc sdesc{};
    // device memory
    void* pop[2] = {nullptr, nullptr};
    void* gpop[2] = {nullptr, nullptr};
    uint32_t* mask = nullptr;
    uint8_t* dtype = nullptr;
    void* mom[2] = {nullptr, nullptr};
    void* pb[6][2] = {};
    void* snap[6] = {};
    unsigned outflow = 0;   // faces with a scalar extrapolation outflow (face pass)
    long long pb_plane[6] = {0, 0, 0, 0, 0, 0};
    void* qads = nullptr;
    void* cprev = nullptr;
    double* c_init_dev = nullptr;
    double* accum = nullptr;
    double* res_dev = nullptr;
    double* res_host = nullptr;   // pinned
    double* obs = nullptr;        // rho | u | c  (doubles)
    unsigned long long* counts = nullptr;
    std::vector<double> lam;      // D3Q27 MRT collision matrix
    long long t = 0;
    long long res_step = -1;
    int block_x = 0;
    bool stage = false;           // one-shot staged sweep (off: the pipelined sweep supersedes it)
    bool pipe = false;            // pipelined bulk-copy sweep on the lean path (option)
    int pipe_stages = 0;          // 0 = chosen from the shared-memory budget
    bool compact = false;         // compacted sweep over a work list on the lean path (in effect)
    int compact_opt = -1;         // -1 = default (FP64 storage only), 0 off, 1 on
    uint32_t* list = nullptr;     // work entries (fluid nodes + solid nodes sharing a sector)
    long long nlist = 0;
    long long Np = 0;             // population plane stride: N rounded up to 64 nodes
    int* err = nullptr;           // device flag: a bounded wait gave up
    cudaStream_t last_stream = nullptr;
    long long bytes = 0;

    ~lbf_domain() {
        for (int k = 0; k < 2; ++k) {
            cudaFree(pop[k]); cudaFree(gpop[k]); cudaFree(mom[k]);
            for (int f = 0; f < 6; ++f) cudaFree(pb[f][k]);
        }
        for (int f = 0; f < 6; ++f) cudaFree(snap[f]);
        cudaFree(mask); cudaFree(dtype); cudaFree(qads); cudaFree(cprev); cudaFree(c_init_dev);
        cudaFree(accum); cudaFree(res_dev); cudaFree(obs); cudaFree(counts); cudaFree(err); cudaFree(list);
        if (res_host) cudaFreeHost(res_host);
    }
    int nfields() const { return 1 + d + (scalar ? 1 : 0); }
};

namespace {

lbf_status dmalloc(lbf_domain* D, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,
                    std::string("cudaMalloc(") + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    D->bytes += (long long)bytes;
    return LBF_OK;
}

dim3 step_block(const lbf_domain* D) {
    int bx = D->block_x;
    if (bx <= 0) {
        bx = 256;
        const long long rows = D->n[1] * D->n[2];
        while (bx > 32 && (bx >= 2 * D->n[0] || ((D->n[0] + bx - 1) / bx) * rows < 4 * 148)) bx /= 2;
    }
    return dim3(bx, 1, 1);
}
dim3 step_grid(const lbf_domain* D, dim3 b) {
    return dim3((unsigned)((D->n[0] + b.x - 1) / b.x), (unsigned)D->n[1], (unsigned)D->n[2]);
}

bool mom_kind_ok(const lbf_domain_desc& ds, int vs, int f, std::string& why) {
    const lbf_bc_desc& b = ds.bc[f];
    switch (b.kind) {
        case LBF_BC_NO_SLIP: case LBF_BC_BOUNCE_BACK: case LBF_BC_ANTI_BOUNCE_BACK: case LBF_BC_PERIODIC:
            return true;
        case LBF_BC_ZOU_HE: {
            const int d = vs_d(vs), ax = f / 2;
            bool tang = true;
            for (int a = 0; a < d; ++a) if (a != ax) tang = tang && b.has_velocity[a];
            bool vel = !b.has_density && b.has_velocity[ax] && tang;
            bool prs = b.has_density && !b.has_velocity[ax] && tang;
            if (vs == LBF_D2Q9 || vs == LBF_D3Q19) {
                if (vel || prs) return true;
                why = "Error: Wrong input of Zou & He (1997) boundary conditions.";
                return false;
            }
            why = "Zou-He is built for D2Q9 (reference) and D3Q19 (extension) only";
            return false;
        }
        default:
            why = "unknown boundary-condition kind";
            return false;
    }
}

void fill_face_params(const lbf_domain* D, StepParams& P) {
    for (int f = 0; f < 6; ++f) {
        const lbf_bc_desc& b = D->desc.bc[f];
        P.face[f].kind = f < D->nfaces ? b.kind : BC_PERIODIC;
        P.face[f].has_rho = b.has_density;
        for (int a = 0; a < 3; ++a) { P.face[f].has_u[a] = b.has_velocity[a]; P.face[f].u[a] = b.velocity[a]; }
        P.face[f].rho = b.density;
        P.pb_plane[f] = D->pb_plane[f];
    }
    bool zero = true;
    for (int f = 0; f < 6; ++f) zero = zero && D->desc.face_order[f] == 0;
    for (int o = 0; o < 6; ++o) P.order[o] = zero ? o : D->desc.face_order[o];
    if (D->scalar) {
        for (int f = 0; f < 6; ++f) {
            const lbf_scalar_bc_desc& s = D->sdesc.bc[f];
            SFaceBC& o = P.sface[f];
            o.kind = f < D->nfaces ? s.kind : SBC_PERIODIC;
            o.unknown_only = s.unknown_populations_only;
            o.value = s.scalar_value;
            // wall velocity from the momentum BC of the same face (ps/bc.rs:43-59)
            const lbf_bc_desc& m = D->desc.bc[f];
            o.given_vel = 0;
            o.u[0] = o.u[1] = o.u[2] = 0.0;
            if (m.kind == LBF_BC_NO_SLIP) o.given_vel = 1;
            else if (m.kind == LBF_BC_BOUNCE_BACK) { o.given_vel = 1; for (int a = 0; a < 3; ++a) o.u[a] = m.velocity[a]; }
            else if (m.kind == LBF_BC_ZOU_HE) {
                bool all = true;
                for (int a = 0; a < D->d; ++a) all = all && m.has_velocity[a];
                if (all) { o.given_vel = 1; for (int a = 0; a < 3; ++a) o.u[a] = m.velocity[a]; }
            }
        }
    }
}

bool face_needs_layers(const lbf_domain* D, int f) {
    if (f >= D->nfaces) return false;
    if (D->desc.bc[f].kind == LBF_BC_ANTI_BOUNCE_BACK) return true;
    if (!D->scalar) return false;
    const int k = D->sdesc.bc[f].kind;
    if (k == LBF_SBC_ANTI_BB_NO_FLUX) return true;
    if (k == LBF_SBC_ANTI_BOUNCE_BACK) {
        const lbf_bc_desc& m = D->desc.bc[f];
        if (m.kind == LBF_BC_NO_SLIP || m.kind == LBF_BC_BOUNCE_BACK) return false;
        if (m.kind == LBF_BC_ZOU_HE) {
            bool all = true;
            for (int a = 0; a < D->d; ++a) all = all && m.has_velocity[a];
            return !all;
        }
        return true;
    }
    return false;
}

// Work list of the compacted sweep: fluid nodes and the solid nodes that share a
// 32-byte sector of a population plane with a fluid node, in node order.
lbf_status build_list(lbf_domain* D, cudaStream_t s) {
    const long long N = D->N;
    const int per = (int)(32 / st_bytes(D->st));
    uint8_t* keep = nullptr;
    uint32_t* val = nullptr;
    int* nsel = nullptr;
    void* tmp = nullptr;
    size_t tmp_bytes = 0;
    lbf_status st = LBF_OK;
    cudaError_t e = cudaMalloc(&keep, N);
    if (e == cudaSuccess) e = cudaMalloc(&val, N * 4);
    if (e == cudaSuccess) e = cudaMalloc(&nsel, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&D->list, N * 4);
    if (e == cudaSuccess) {
        const unsigned nb = (unsigned)((N + 255) / 256);
        if (D->d == 2) k_list_mark<2><<<nb, 256, 0, s>>>(D->mask, N, (int)D->n[0], (int)D->n[1], (int)D->n[2], per, keep, val);
        else k_list_mark<3><<<nb, 256, 0, s>>>(D->mask, N, (int)D->n[0], (int)D->n[1], (int)D->n[2], per, keep, val);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, tmp_bytes, val, keep, D->list, nsel, (int)N, s);
    if (e == cudaSuccess) e = cudaMalloc(&tmp, tmp_bytes);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, val, keep, D->list, nsel, (int)N, s);
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(keep); cudaFree(val); cudaFree(nsel); cudaFree(tmp);
    if (e != cudaSuccess) {
        cudaFree(D->list);
        D->list = nullptr;
        st = fail(e == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,
                  std::string("work list: ") + cudaGetErrorString(e));
    } else {
        D->nlist = h;
        D->bytes += N * 4;
    }
    return st;
}

// Node classification + device masks (Lattice::new), run once before init.
lbf_status prepare(lbf_domain* D, uint32_t* cls_out, uint32_t* links_out, cudaStream_t s) {
    const long long N = D->N;
    D->facebc = D->scalar;
    for (int f = 0; f < D->nfaces; ++f) {
        const int k = D->desc.bc[f].kind;
        if (k != LBF_BC_NO_SLIP && k != LBF_BC_PERIODIC) D->facebc = true;
    }
    unsigned fold = 0, expl = 0;
    for (int f = 0; f < D->nfaces; ++f) {
        const int k = D->desc.bc[f].kind;
        if (D->facebc) {
            if (k != LBF_BC_PERIODIC || (D->scalar && D->sdesc.bc[f].kind != LBF_SBC_PERIODIC)) expl |= 1u << f;
        } else if (k == LBF_BC_NO_SLIP) {
            fold |= 1u << f;
        }
    }
    uint32_t* cls = nullptr;
    uint32_t* links = nullptr;
    lbf_status st;
    if (!D->mask && (st = dmalloc(D, (void**)&D->mask, N * 4))) return st;
    if ((st = dmalloc(D, (void**)&cls, N * 4))) return st;
    if ((st = dmalloc(D, (void**)&links, N * 4))) { cudaFree(cls); return st; }
    D->bytes -= 8 * N;
    if (!D->counts && (st = dmalloc(D, (void**)&D->counts, 16))) { cudaFree(cls); cudaFree(links); return st; }
    if (!D->dtype && (st = dmalloc(D, (void**)&D->dtype, N))) { cudaFree(cls); cudaFree(links); return st; }
    cudaError_t e = cudaMemcpyAsync(D->dtype, D->type.data(), N, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(D->counts, 0, 16, s);
    SetupParams S{};
    S.nx = (int)D->n[0]; S.ny = (int)D->n[1]; S.nz = (int)D->n[2]; S.N = N;
    S.type = D->dtype; S.cls = cls; S.links = links; S.mask = D->mask;
    S.fold_faces = fold; S.explicit_faces = expl; S.skip_faces = D->outflow; S.counts = D->counts;
    Launch L{dim3((unsigned)((N + 255) / 256)), dim3(256), s};
    if (e == cudaSuccess) {
        e = D->vs == LBF_D2Q9 ? launch_setup<VS_D2Q9>(S, L)
          : D->vs == LBF_D3Q19 ? launch_setup<VS_D3Q19>(S, L) : launch_setup<VS_D3Q27>(S, L);
    }
    unsigned long long cnt[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, D->counts, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && cls_out) e = cudaMemcpyAsync(cls_out, cls, N * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && links_out) e = cudaMemcpyAsync(links_out, links, N * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(cls);
    cudaFree(links);
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("node classification: ") + cudaGetErrorString(e));
    D->n_fluid = cnt[0];
    D->n_bb = cnt[1];
    // face layers and outflow snapshots
    for (int f = 0; f < D->nfaces; ++f) D->pb_plane[f] = N / D->n[f / 2];
    for (int f = 0; f < 6; ++f) {
        const long long plane = D->pb_plane[f];
        if (face_needs_layers(D, f))
            for (int k = 0; k < 2; ++k)
                if (!D->pb[f][k] && (st = dmalloc(D, &D->pb[f][k], 2 * (D->d + 1) * plane * rt_bytes(D->st)))) return st;
        if ((D->outflow >> f & 1u) && !D->snap[f]) {
            const size_t b = 2 * (size_t)D->q * plane * rt_bytes(D->st);
            if ((st = dmalloc(D, &D->snap[f], b))) return st;
            CK(cudaMemsetAsync(D->snap[f], 0, b, s));   // solid neighbours read as zero populations
        }
    }
    D->nlist = 0;
    if (D->list) { cudaFree(D->list); D->list = nullptr; }
    const bool want = D->compact_opt < 0 ? D->st == LBF_STORE_F64 : D->compact_opt != 0;
    D->compact = want;
    if (!D->facebc && !D->scalar && want && N < (1ll << 30) && (st = build_list(D, s))) return st;
    D->prepared = true;
    return LBF_OK;
}

void base_params(const lbf_domain* D, StepParams& P, long long t) {
    std::memset(&P, 0, sizeof(P));
    P.nx = (int)D->n[0]; P.ny = (int)D->n[1]; P.nz = (int)D->n[2]; P.dims = D->d;
    P.N = D->N;
    P.mask = D->mask;
    P.err = D->err;
    P.list = D->list;
    P.nlist = D->nlist;
    P.inv_nx = 1.0 / (double)D->n[0];
    P.inv_ny = 1.0 / (double)D->n[1];
    const size_t eb = st_bytes(D->st);
    for (int i = 0; i < D->q; ++i) {
        P.srcp[i] = (const char*)D->pop[t & 1] + (size_t)i * D->Np * eb;
        P.dstp[i] = (char*)D->pop[(t + 1) & 1] + (size_t)i * D->Np * eb;
    }
    const lbf_collision_desc& c = D->desc.collision;
    P.coll = c.kind; P.compat = D->desc.compat; P.has_force = D->desc.has_force; P.first = t == 0;
    P.tau = c.tau; P.omega = c.kind == LBF_BGK ? 1.0 / c.tau : 0.0; P.op = c.omega_plus; P.om = c.omega_minus;
    for (int k = 0; k < 27; ++k) P.rates[k] = c.relaxation[k];
    for (int a = 0; a < 3; ++a) P.force[a] = D->desc.has_force ? D->desc.force[a] : 0.0;
    fill_face_params(D, P);
    P.any_face = 0;
    for (int f = 0; f < 6; ++f) {
        P.pb_src[f] = D->pb[f][(t + 1) & 1];
        P.pb_dst[f] = D->pb[f][t & 1];
        if (D->pb[f][0]) P.any_face = 1;
    }
    for (int f = 0; f < 6; ++f) P.snap[f] = D->snap[f];
    P.mom_prev = D->mom[(t + 1) & 1];
    P.mom_cur = D->mom[t & 1];
    P.accum = D->accum;
    if (D->scalar) {
        const lbf_scalar_desc& s = D->sdesc;
        P.has_scalar = 1;
        P.s_coll = s.collision.kind; P.s_inner = s.inner_boundary_condition; P.s_has_source = s.has_source;
        P.s_tau = s.collision.tau; P.s_omega = s.collision.kind == LBF_BGK ? 1.0 / s.collision.tau : 0.0;
        P.s_op = s.collision.omega_plus; P.s_om = s.collision.omega_minus; P.s_source = s.source_value;
        P.s_ads = s.has_adsorption;
        P.ka = s.adsorption_rate; P.kd = s.desorption_rate; P.qmax = s.q_max;
        P.c_solid = s.initial_scalar_value;
        P.c_init = D->c_init_dev;
        const size_t rb = rt_bytes(D->st);
        for (int i = 0; i < D->q; ++i) {
            P.gsrcp[i] = (const char*)D->gpop[t & 1] + (size_t)i * D->Np * rb;
            P.gdstp[i] = (char*)D->gpop[(t + 1) & 1] + (size_t)i * D->Np * rb;
        }
        P.qads = D->qads;
        P.cprev = D->cprev;
    }
}

cudaError_t launch_one(lbf_domain* D, const StepParams& P, bool stage, const Launch& L) {
    const int coll = D->desc.collision.kind;
    switch (D->vs) {
        case LBF_D2Q9: return launch_step<VS_D2Q9>(coll, D->st, D->facebc, D->scalar, stage, P, nullptr, L);
        case LBF_D3Q19: return launch_step<VS_D3Q19>(coll, D->st, D->facebc, D->scalar, stage, P, nullptr, L);
        default: return launch_step<VS_D3Q27>(coll, D->st, D->facebc, D->scalar, stage, P, D->lam.data(), L);
    }
}

// Whether the staged (bulk-copy) sweep applies: one block per x-row, rows
// 16-byte aligned, the staged rows fit in shared memory.
bool can_stage(const lbf_domain* D) {
    const size_t tb = st_bytes(D->st), rb = rt_bytes(D->st);
    if (D->n[0] > 512 || (D->n[0] * tb) % 16 != 0) return false;
    if (D->scalar && (D->n[0] * rb) % 16 != 0) return false;
    return stage_smem(D->q, D->n[0], tb, rb, D->scalar) <= 200 * 1024;
}

// Whether the pipelined sweep applies (lean path, aligned rows, two stages fit).
bool can_pipe(const lbf_domain* D) {
    const size_t rowb = D->n[0] * st_bytes(D->st);
    return !D->facebc && !D->scalar && rowb % 16 == 0 && 2 * D->q * rowb <= 200 * 1024;
}

cudaError_t launch_pipe(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    const size_t stage_b = (size_t)D->q * D->n[0] * st_bytes(D->st);
    // three blocks of <= 288 threads per SM share ~220 KB of shared memory
    int stages = D->pipe_stages > 0 ? D->pipe_stages : (int)std::max<size_t>(2, std::min<size_t>(8, (72 * 1024) / stage_b));
    while (stages > 2 && stages * stage_b > 200 * 1024) --stages;
    const int nc = (int)std::min<long long>(8, std::max<long long>(1, (D->n[0] + 31) / 32));
    const int coll = D->desc.collision.kind;
    switch (D->vs) {
        case LBF_D2Q9:
            return coll == LBF_BGK ? launch_step_pipe<VS_D2Q9, COLL_BGK>(D->st, P, nullptr, stages, nc, s)
                 : coll == LBF_TRT ? launch_step_pipe<VS_D2Q9, COLL_TRT>(D->st, P, nullptr, stages, nc, s)
                                   : launch_step_pipe<VS_D2Q9, COLL_MRT>(D->st, P, nullptr, stages, nc, s);
        case LBF_D3Q19:
            return coll == LBF_BGK ? launch_step_pipe<VS_D3Q19, COLL_BGK>(D->st, P, nullptr, stages, nc, s)
                 : coll == LBF_TRT ? launch_step_pipe<VS_D3Q19, COLL_TRT>(D->st, P, nullptr, stages, nc, s)
                                   : launch_step_pipe<VS_D3Q19, COLL_MRT>(D->st, P, nullptr, stages, nc, s);
        default:
            return coll == LBF_BGK ? launch_step_pipe<VS_D3Q27, COLL_BGK>(D->st, P, D->lam.data(), stages, nc, s)
                 : coll == LBF_TRT ? launch_step_pipe<VS_D3Q27, COLL_TRT>(D->st, P, D->lam.data(), stages, nc, s)
                                   : launch_step_pipe<VS_D3Q27, COLL_MRT>(D->st, P, D->lam.data(), stages, nc, s);
    }
}

cudaError_t launch_list(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    const int coll = D->desc.collision.kind;
    switch (D->vs) {
        case LBF_D2Q9:
            return coll == LBF_BGK ? launch_step_list<VS_D2Q9, COLL_BGK>(D->st, P, nullptr, s)
                 : coll == LBF_TRT ? launch_step_list<VS_D2Q9, COLL_TRT>(D->st, P, nullptr, s)
                                   : launch_step_list<VS_D2Q9, COLL_MRT>(D->st, P, nullptr, s);
        case LBF_D3Q19:
            return coll == LBF_BGK ? launch_step_list<VS_D3Q19, COLL_BGK>(D->st, P, nullptr, s)
                 : coll == LBF_TRT ? launch_step_list<VS_D3Q19, COLL_TRT>(D->st, P, nullptr, s)
                                   : launch_step_list<VS_D3Q19, COLL_MRT>(D->st, P, nullptr, s);
        default:
            return coll == LBF_BGK ? launch_step_list<VS_D3Q27, COLL_BGK>(D->st, P, D->lam.data(), s)
                 : coll == LBF_TRT ? launch_step_list<VS_D3Q27, COLL_TRT>(D->st, P, D->lam.data(), s)
                                   : launch_step_list<VS_D3Q27, COLL_MRT>(D->st, P, D->lam.data(), s);
    }
}

// The bulk sweep, then one face pass per scalar outflow face.
cudaError_t launch_step_any(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    const bool lean = !D->facebc && !D->scalar && !P.first && !P.observe && !P.face_pass;
    if (D->pipe && lean && can_pipe(D)) {
        cudaError_t e = launch_pipe(D, P, s);
        if (e != cudaErrorNotSupported) return e;
        cudaGetLastError();
    }
    if (lean && D->compact && D->list) return launch_list(D, P, s);
    const bool stage = D->stage && can_stage(D);
    const dim3 b = stage ? dim3((unsigned)D->n[0]) : step_block(D);
    cudaError_t e = launch_one(D, P, stage, Launch{step_grid(D, b), b, s});
    for (int f = 0; f < D->nfaces && e == cudaSuccess; ++f) {
        if (!(D->outflow >> f & 1u)) continue;
        StepParams F = P;
        F.face_pass = 1;
        F.fp_face = f;
        e = launch_one(D, F, false, Launch{dim3((unsigned)((D->pb_plane[f] + 127) / 128)), dim3(128), s});
    }
    return e;
}

// Reads the device error flag after a synchronisation point.
lbf_status check_err(lbf_domain* D) {
    int h = 0;
    CK(cudaMemcpy(&h, D->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) return fail(LBF_ETIMEOUT, "a bounded wait in the step kernel gave up (staged copy did not complete)");
    return LBF_OK;
}

lbf_status ensure_mom(lbf_domain* D) {
    if (D->mom[0]) return LBF_OK;
    lbf_status st;
    for (int k = 0; k < 2; ++k)
        if ((st = dmalloc(D, &D->mom[k], (size_t)D->nfields() * D->N * rt_bytes(D->st)))) return st;
    return LBF_OK;
}

lbf_status do_init(lbf_domain* D, cudaStream_t s) {
    lbf_status st;
    if (!D->prepared && (st = prepare(D, nullptr, nullptr, s))) return st;
    if ((st = ensure_mom(D))) return st;
    StepParams P;
    base_params(D, P, 0);
    P.mom_prev = D->mom[1];   // seeded with the initial moments (ShallowNode)
    InitParams I{};
    I.rho0 = D->rho0u;
    for (int a = 0; a < 3; ++a) I.u0[a] = D->u0u[a];
    I.c0 = D->scalar ? D->sdesc.initial_scalar_value : 0.0;
    I.q0 = D->scalar ? D->sdesc.initial_q_ads : 0.0;
    // upload per-node initial fields for the duration of the init kernel
    double* tmp = nullptr;
    const size_t nr = D->rho0.empty() ? 0 : D->N, nu = D->u0.empty() ? 0 : D->N * D->d;
    const size_t nc = D->c0.empty() ? 0 : D->N;
    if (nr + nu + nc) {
        CK(cudaMalloc(&tmp, (nr + nu + nc) * sizeof(double)));
        if (nr) CK(cudaMemcpyAsync(tmp, D->rho0.data(), nr * 8, cudaMemcpyHostToDevice, s));
        if (nu) CK(cudaMemcpyAsync(tmp + nr, D->u0.data(), nu * 8, cudaMemcpyHostToDevice, s));
        if (nc) CK(cudaMemcpyAsync(tmp + nr + nu, D->c0.data(), nc * 8, cudaMemcpyHostToDevice, s));
        I.rho_field = nr ? tmp : nullptr;
        I.u_field = nu ? tmp + nr : nullptr;
        I.c_field = nc ? tmp + nr + nu : nullptr;
    }
    void* pb[12];
    for (int f = 0; f < 6; ++f) { pb[2 * f] = D->pb[f][0]; pb[2 * f + 1] = D->pb[f][1]; }
    Launch L{dim3((unsigned)((D->N + 255) / 256)), dim3(256), s};
    cudaError_t e = D->vs == LBF_D2Q9 ? launch_init<VS_D2Q9>(D->st, D->scalar, P, I, pb, L)
                  : D->vs == LBF_D3Q19 ? launch_init<VS_D3Q19>(D->st, D->scalar, P, I, pb, L)
                                       : launch_init<VS_D3Q27>(D->st, D->scalar, P, I, pb, L);
    if (tmp) {
        cudaStreamSynchronize(s);
        cudaFree(tmp);
    }
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("init kernel: ") + cudaGetErrorString(e));
    CK(cudaMemsetAsync(D->accum, 0, NSLOT * NACC * sizeof(double), s));
    D->t = 0;
    D->res_step = -1;
    D->initialized = true;
    D->last_stream = s;
    return LBF_OK;
}

lbf_status do_steps(lbf_domain* D, long long nsteps, long long k, cudaStream_t s) {
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called before stepping");
    lbf_status st;
    if (k > 0 && (st = ensure_mom(D))) return st;
    for (long long it = 0; it < nsteps; ++it) {
        const long long t = D->t;
        StepParams P;
        base_params(D, P, t);
        P.residual = (k > 0 && t % k == 0) ? 1 : 0;
        P.write_mom = (k > 0 && (t % k == 0 || (t + 1) % k == 0)) ? 1 : 0;
        cudaError_t e = launch_step_any(D, P, s);
        if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("step kernel: ") + cudaGetErrorString(e));
        if (P.residual) {
            k_finalize<<<1, 32, 0, s>>>(D->accum, 5, 1, D->res_dev);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(D->res_host, D->res_dev, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
            D->res_step = t;
        }
        D->t = t + 1;
    }
    D->last_stream = s;
    return LBF_OK;
}

lbf_status do_observe(lbf_domain* D, cudaStream_t s) {
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called first");
    lbf_status st;
    if (!D->obs && (st = dmalloc(D, (void**)&D->obs, (size_t)D->N * (D->d + 2) * sizeof(double)))) return st;
    StepParams P;
    base_params(D, P, D->t);
    P.observe = 1;
    P.obs_rho = D->obs;
    P.obs_u = D->obs + D->N;
    P.obs_c = D->obs + D->N * (1 + D->d);
    cudaError_t e = launch_step_any(D, P, s);
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("observe kernel: ") + cudaGetErrorString(e));
    return LBF_OK;
}

}  // namespace

// Lets the other translation units of the library report through lbf_last_error().
__attribute__((visibility("hidden"))) lbf_status lbf_internal_fail(lbf_status s, const char* msg) {
    return fail(s, msg);
}

// ============================================================== C API
extern "C" {

int32_t lbf_abi_version(void) { return LBF_ABI_VERSION; }
const char* lbf_last_error(void) { return g_err.c_str(); }
size_t lbf_sizeof(int32_t which) {
    switch (which) {
        case 0: return sizeof(lbf_domain_desc);
        case 1: return sizeof(lbf_scalar_desc);
        case 2: return sizeof(lbf_bc_desc);
        case 3: return sizeof(lbf_collision_desc);
        default: return 0;
    }
}

lbf_status lbf_velocity_set_tables(int32_t vs, int32_t* d, int32_t* q, int32_t* c, double* w, int32_t* q_bar,
                                   int32_t* q_faces, int32_t* face_normal, double* mrt, double* mrt_inverse) {
    switch (vs) {
        case LBF_D2Q9: tables_of<VS_D2Q9>(d, q, c, w, q_bar, q_faces, face_normal, mrt, mrt_inverse); return LBF_OK;
        case LBF_D3Q19: tables_of<VS_D3Q19>(d, q, c, w, q_bar, q_faces, face_normal, mrt, mrt_inverse); return LBF_OK;
        case LBF_D3Q27: tables_of<VS_D3Q27>(d, q, c, w, q_bar, q_faces, face_normal, mrt, mrt_inverse); return LBF_OK;
        default: return fail(LBF_EUNSUPPORTED, "velocity set not built on the device (D2Q9, D3Q19, D3Q27 are)");
    }
}

lbf_status lbf_domain_create(const lbf_domain_desc* ds, lbf_domain** out) {
    if (!ds || !out) return fail(LBF_EINVAL, "null argument");
    *out = nullptr;
    const int vs = ds->velocity_set;
    if (vs != LBF_D2Q9 && vs != LBF_D3Q19 && vs != LBF_D3Q27)
        return fail(LBF_EUNSUPPORTED, "velocity set not built on the device (D2Q9, D3Q19, D3Q27 are)");
    if (ds->storage < LBF_STORE_F64 || ds->storage > LBF_STORE_BF16DEV) return fail(LBF_EINVAL, "bad storage");
    const int d = vs_d(vs);
    long long n[3] = {ds->n[0], ds->n[1], d == 3 ? ds->n[2] : 1};
    for (int a = 0; a < 3; ++a)
        if (n[a] < 1) return fail(LBF_EINVAL, "lattice dimensions must be >= 1");
    if (n[1] > 65535 || n[2] > 65535) return fail(LBF_EINVAL, "ny and nz must be <= 65535");
    const long long N = n[0] * n[1] * n[2];
    if (N >= (1ll << 31)) return fail(LBF_EINVAL, "more than 2^31 nodes");
    const lbf_collision_desc& c = ds->collision;
    if (c.kind == LBF_BGK && !(c.tau > 0.0)) return fail(LBF_EINVAL, "BGK tau must be > 0");
    if (c.kind < LBF_BGK || c.kind > LBF_MRT) return fail(LBF_EINVAL, "bad collision kind");
    const int nf = d == 2 ? 4 : 6;
    for (int f = 0; f < nf; ++f) {
        std::string why;
        if (!mom_kind_ok(*ds, vs, f, why)) return fail(LBF_EINVAL, why);
    }
    bool zero = true;
    for (int f = 0; f < 6; ++f) zero = zero && ds->face_order[f] == 0;
    if (!zero) {
        int seen = 0;
        for (int o = 0; o < nf; ++o) {
            const int f = ds->face_order[o];
            if (f < 0 || f >= nf || (seen >> f & 1)) return fail(LBF_EINVAL, "face_order is not a permutation of the faces");
            seen |= 1 << f;
        }
    }
    lbf_domain* D = new lbf_domain();
    D->desc = *ds;
    D->desc.node_type = nullptr;
    D->desc.initial_density_field = nullptr;
    D->desc.initial_velocity_field = nullptr;
    D->vs = vs; D->q = vs_q(vs); D->d = d; D->st = ds->storage; D->nfaces = nf;
    for (int a = 0; a < 3; ++a) D->n[a] = n[a];
    D->N = N;
    D->type.assign(N, 0);
    if (ds->node_type) for (long long i = 0; i < N; ++i) D->type[i] = ds->node_type[i] ? 1 : 0;
    D->rho0u = ds->initial_density;
    for (int a = 0; a < 3; ++a) D->u0u[a] = ds->initial_velocity[a];
    if (ds->initial_density_field) D->rho0.assign(ds->initial_density_field, ds->initial_density_field + N);
    if (ds->initial_velocity_field) D->u0.assign(ds->initial_velocity_field, ds->initial_velocity_field + N * d);
    if (vs == LBF_D3Q27 && c.kind == LBF_MRT) {
        std::vector<double> M(729), Mi(729);
        d3q27_basis(M.data(), Mi.data());
        D->lam.assign(729, 0.0);
        for (int i = 0; i < 27; ++i)
            for (int j = 0; j < 27; ++j) {
                double s = 0.0;
                for (int k = 0; k < 27; ++k) s += Mi[i * 27 + k] * c.relaxation[k] * M[k * 27 + j];
                D->lam[i * 27 + j] = s;
            }
    }
    lbf_status st;
    D->Np = (N + 63) / 64 * 64;   // every plane starts on a 256-byte boundary
    const size_t pbytes = (size_t)D->q * D->Np * st_bytes(D->st);
    for (int k = 0; k < 2; ++k)
        if ((st = dmalloc(D, &D->pop[k], pbytes))) { delete D; return st; }
    if ((st = dmalloc(D, (void**)&D->accum, NSLOT * NACC * sizeof(double)))) { delete D; return st; }
    if ((st = dmalloc(D, (void**)&D->res_dev, 8 * sizeof(double)))) { delete D; return st; }
    if ((st = dmalloc(D, (void**)&D->err, sizeof(int)))) { delete D; return st; }
    if (cudaMemset(D->err, 0, sizeof(int)) != cudaSuccess) { delete D; return fail(LBF_EDEVICE, "memset"); }
    if (cudaMallocHost(&D->res_host, 8 * sizeof(double)) != cudaSuccess) { delete D; return fail(LBF_ENOMEM, "pinned alloc"); }
    std::memset(D->res_host, 0, 8 * sizeof(double));
    if (cudaMemset(D->accum, 0, NSLOT * NACC * sizeof(double)) != cudaSuccess) { delete D; return fail(LBF_EDEVICE, "memset"); }
    *out = D;
    return LBF_OK;
}

lbf_status lbf_scalar_attach(lbf_domain* D, const lbf_scalar_desc* s) {
    if (!D || !s) return fail(LBF_EINVAL, "null argument");
    if (D->scalar) return fail(LBF_EINVAL, "one scalar per domain");
    if (D->initialized || D->prepared) return fail(LBF_ESTATE, "attach the scalar before lbf_domain_init");
    if (s->velocity_set != D->vs)
        return fail(LBF_EUNSUPPORTED, "on the device the scalar uses the momentum velocity set");
    if (D->st != LBF_STORE_F64 && D->st != LBF_STORE_F32)
        return fail(LBF_EUNSUPPORTED, "the scalar is built for F64 and F32 storage");
    if (s->collision.kind == LBF_MRT) return fail(LBF_EUNSUPPORTED, "scalar MRT is not built on the device");
    if (s->collision.kind == LBF_BGK && !(s->collision.tau > 0.0)) return fail(LBF_EINVAL, "scalar tau must be > 0");
    for (int f = 0; f < D->nfaces; ++f) {
        const int k = s->bc[f].kind;
        if (k < LBF_SBC_ANTI_BOUNCE_BACK || k > LBF_SBC_PERIODIC) return fail(LBF_EINVAL, "bad scalar BC kind");
    }
    unsigned outflow = 0;
    for (int f = 0; f < D->nfaces; ++f) {
        const int k = s->bc[f].kind;
        if (k != LBF_SBC_ZEROTH_ORDER_NO_FLUX && k != LBF_SBC_SECOND_ORDER_NO_FLUX) continue;
        if (D->n[f / 2] < 4) return fail(LBF_EINVAL, "an extrapolation outflow face needs >= 4 nodes along its normal");
        outflow |= 1u << f;
    }
    for (int f = 0; f < D->nfaces; ++f)
        for (int g = 0; g < D->nfaces; ++g)
            if ((outflow >> f & 1u) && (outflow >> g & 1u) && f / 2 != g / 2)
                return fail(LBF_EUNSUPPORTED, "extrapolation outflow on two faces that share an edge is not built");
    D->outflow = outflow;
    D->sdesc = *s;
    D->sdesc.initial_scalar_field = nullptr;
    if (s->initial_scalar_field) D->c0.assign(s->initial_scalar_field, s->initial_scalar_field + D->N);
    lbf_status st;
    const size_t rb = rt_bytes(D->st);
    for (int k = 0; k < 2; ++k)
        if ((st = dmalloc(D, &D->gpop[k], (size_t)D->q * D->Np * rb))) return st;
    if (s->has_adsorption) {
        if ((st = dmalloc(D, &D->qads, D->N * rb))) return st;
        if ((st = dmalloc(D, &D->cprev, D->N * rb))) return st;
    }
    if (!D->c0.empty()) {
        if ((st = dmalloc(D, (void**)&D->c_init_dev, D->N * sizeof(double)))) return st;
        CK(cudaMemcpy(D->c_init_dev, D->c0.data(), D->N * sizeof(double), cudaMemcpyHostToDevice));
    }
    D->scalar = true;
    return LBF_OK;
}

lbf_status lbf_domain_init(lbf_domain* D, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    return do_init(D, (cudaStream_t)stream);
}

lbf_status lbf_domain_step(lbf_domain* D, int64_t nsteps, int64_t residual_interval, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (nsteps < 0) return fail(LBF_EINVAL, "nsteps < 0");
    return do_steps(D, nsteps, residual_interval, (cudaStream_t)stream);
}

lbf_status lbf_domain_run(lbf_domain* D, int64_t max_iterations, int64_t k, double tr, double tu, double tc,
                          int64_t* steps_done, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (k < 1) k = 1;
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    for (;;) {
        const long long t = D->t;
        if ((st = do_steps(D, 1, k, s))) return st;
        bool stop = t > max_iterations;
        if (!stop && t > 10 && D->res_step == t) {
            CK(cudaStreamSynchronize(s));
            bool conv = D->res_host[0] <= tr;
            for (int a = 0; a < D->d; ++a) conv = conv && D->res_host[1 + a] <= tu;
            if (D->scalar) conv = conv && D->res_host[4] <= tc;
            if (!std::isfinite(D->res_host[0])) return fail(LBF_ENAN, "non-finite residual");
            stop = conv;
        }
        if (stop) break;
    }
    CK(cudaStreamSynchronize(s));
    if (steps_done) *steps_done = D->t;
    return LBF_OK;
}

lbf_status lbf_domain_residuals(lbf_domain* D, double* out, int64_t* time_step) {
    if (!D || !out) return fail(LBF_EINVAL, "null argument");
    CK(cudaStreamSynchronize(D->last_stream));
    lbf_status est = check_err(D);
    if (est) return est;
    for (int k = 0; k < D->nfields(); ++k) out[k] = D->res_host[k];
    if (D->scalar && D->d == 2) out[3] = D->res_host[4];
    if (time_step) *time_step = D->res_step;
    return LBF_OK;
}

lbf_status lbf_domain_get_moments(lbf_domain* D, double* rho, double* u, double* c, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    if ((st = do_observe(D, s))) return st;
    const long long N = D->N;
    if (rho) CK(cudaMemcpyAsync(rho, D->obs, N * 8, cudaMemcpyDeviceToHost, s));
    if (u) CK(cudaMemcpyAsync(u, D->obs + N, N * D->d * 8, cudaMemcpyDeviceToHost, s));
    if (c && D->scalar) CK(cudaMemcpyAsync(c, D->obs + N * (1 + D->d), N * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if ((st = check_err(D))) return st;
    // solid nodes keep their initial values (they are never updated)
    for (long long i = 0; i < N; ++i) {
        if (!D->type[i]) continue;
        if (rho) rho[i] = D->rho0.empty() ? D->rho0u : D->rho0[i];
        if (u) for (int a = 0; a < D->d; ++a) u[i * D->d + a] = D->u0.empty() ? D->u0u[a] : D->u0[i * D->d + a];
        if (c && D->scalar) c[i] = D->c0.empty() ? D->sdesc.initial_scalar_value : D->c0[i];
    }
    return LBF_OK;
}

lbf_status lbf_domain_get_q_ads(lbf_domain* D, double* q) {
    if (!D || !q) return fail(LBF_EINVAL, "null argument");
    CK(cudaStreamSynchronize(D->last_stream));
    if (!D->qads) {
        std::fill(q, q + D->N, 0.0);
        return LBF_OK;
    }
    if (D->st == LBF_STORE_F64) {
        CK(cudaMemcpy(q, D->qads, D->N * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(D->N);
        CK(cudaMemcpy(tmp.data(), D->qads, D->N * 4, cudaMemcpyDeviceToHost));
        for (long long i = 0; i < D->N; ++i) q[i] = tmp[i];
    }
    return LBF_OK;
}

lbf_status lbf_domain_inventory(lbf_domain* D, double* out, void* stream) {
    if (!D || !out) return fail(LBF_EINVAL, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    if ((st = do_observe(D, s))) return st;
    const long long N = D->N;
    const double* c = D->scalar ? D->obs + N * (1 + D->d) : nullptr;
    const unsigned nb = (unsigned)((N + 255) / 256);
    if (D->d == 2) {
        if (D->st == LBF_STORE_F64) k_inventory<2, double><<<nb, 256, 0, s>>>(D->mask, N, D->obs, D->obs + N, c, (const double*)D->qads, D->accum);
        else k_inventory<2, float><<<nb, 256, 0, s>>>(D->mask, N, D->obs, D->obs + N, c, (const float*)D->qads, D->accum);
    } else {
        if (D->st == LBF_STORE_F64) k_inventory<3, double><<<nb, 256, 0, s>>>(D->mask, N, D->obs, D->obs + N, c, (const double*)D->qads, D->accum);
        else k_inventory<3, float><<<nb, 256, 0, s>>>(D->mask, N, D->obs, D->obs + N, c, (const float*)D->qads, D->accum);
    }
    CK(cudaGetLastError());
    double* tmp = nullptr;
    CK(cudaMalloc(&tmp, 8 * sizeof(double)));
    k_finalize<<<1, 32, 0, s>>>(D->accum, 6, 0, tmp);
    double h[8];
    cudaError_t e = cudaMemcpyAsync(h, tmp, 8 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(tmp);
    if (e != cudaSuccess) return fail(LBF_EDEVICE, cudaGetErrorString(e));
    for (int k = 0; k < 3 + D->d; ++k) out[k] = h[k];
    return LBF_OK;
}

lbf_status lbf_domain_get_node_class(lbf_domain* D, uint32_t* cls, uint32_t* links) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    return prepare(D, cls, links, D->last_stream);
}

lbf_status lbf_domain_time_step(lbf_domain* D, int64_t* t) {
    if (!D || !t) return fail(LBF_EINVAL, "null argument");
    *t = D->t;
    return LBF_OK;
}

lbf_status lbf_domain_device_bytes(lbf_domain* D, int64_t* b) {
    if (!D || !b) return fail(LBF_EINVAL, "null argument");
    *b = D->bytes;
    return LBF_OK;
}

lbf_status lbf_domain_set_option(lbf_domain* D, int32_t option, int64_t value) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    switch (option) {
        case LBF_OPT_BLOCK_X:
            if (value < 0 || value > 1024 || (value % 32)) return fail(LBF_EINVAL, "block_x must be 0 or a multiple of 32 <= 1024");
            D->block_x = (int)value;
            return LBF_OK;
        case LBF_OPT_STAGE:
            D->stage = value != 0;
            return LBF_OK;
        case LBF_OPT_PIPE:
            D->pipe = value != 0;
            return LBF_OK;
        case LBF_OPT_PIPE_STAGES:
            if (value < 0 || value == 1 || value > 16) return fail(LBF_EINVAL, "pipeline stages must be 0 (auto) or 2..16");
            D->pipe_stages = (int)value;
            return LBF_OK;
        case LBF_OPT_COMPACT:
            if (D->prepared) return fail(LBF_ESTATE, "set LBF_OPT_COMPACT before lbf_domain_init");
            D->compact_opt = value != 0 ? 1 : 0;
            return LBF_OK;
        default:
            return fail(LBF_EINVAL, "unknown option");
    }
}

lbf_status lbf_domain_get_option(lbf_domain* D, int32_t option, int64_t* value) {
    if (!D || !value) return fail(LBF_EINVAL, "null argument");
    switch (option) {
        case LBF_OPT_BLOCK_X: *value = D->block_x; return LBF_OK;
        case LBF_OPT_STAGE: *value = (D->stage && can_stage(D)) ? 1 : 0; return LBF_OK;
        case LBF_OPT_PIPE: *value = (D->pipe && can_pipe(D)) ? 1 : 0; return LBF_OK;
        case LBF_OPT_PIPE_STAGES: *value = D->pipe_stages; return LBF_OK;
        case LBF_OPT_COMPACT: *value = (D->compact && D->list) ? 1 : 0; return LBF_OK;
        default: return fail(LBF_EINVAL, "unknown option");
    }
}

lbf_status lbf_domain_destroy(lbf_domain* D) {
    if (D) {
        if (D->last_stream) cudaStreamSynchronize(D->last_stream);
        delete D;
    }
    return LBF_OK;
}

lbf_status lbf_solve(const lbf_domain_desc* desc, const lbf_scalar_desc* sdesc, int64_t nsteps, double* rho,
                     double* u, double* c, void* stream) {
    lbf_domain* D = nullptr;
    lbf_status st = lbf_domain_create(desc, &D);
    if (st) return st;
    if (sdesc && (st = lbf_scalar_attach(D, sdesc))) { lbf_domain_destroy(D); return st; }
    if ((st = lbf_domain_init(D, stream)) || (st = lbf_domain_step(D, nsteps, 0, stream)) ||
        (st = lbf_domain_get_moments(D, rho, u, c, stream))) {
        lbf_domain_destroy(D);
        return st;
    }
    return lbf_domain_destroy(D);
}

}  // extern "C"
