// abi.cu -- the C ABI of include/lbflow.h: domain lifecycle, launches, host I/O.
//
// A domain owns its device memory: two population buffers (A/B, SoA planes),
// the per-node mask word, optional scalar buffers, the face-layer buffers used
// by anti-bounce-back and extrapolated wall velocities, the per-node moments of
// residual steps, and the FP64 partial-sum slots of the reductions.
#include <cuda_runtime.h>
#include <sys/mman.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "../../include/lbflow.h"
#include "batch.cuh"
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

// Residual and inventory partial sums: six accumulators, one slot per block of
// the widest launch a domain can make (the dense sweep at 32 threads per block,
// plus one face pass per face at 32 threads per block: an upper bound of every
// other launch shape, 256-thread sparse and inventory sweeps included).
constexpr int ACCUM_PLANES = 4 + NSMAX;   // residual accumulators of a scalar sweep (the most)
static_assert(NSMAX == LBF_MAX_SCALARS, "the header's scalar limit is the kernels'");
long long accum_slots(const long long* n, int nfaces) {
    long long s = (n[0] + 31) / 32 * n[1] * n[2];
    const long long N = n[0] * n[1] * n[2];
    for (int f = 0; f < nfaces; ++f) s += (N / n[f / 2] + 31) / 32;
    return s + 16;
}

// ---- device and pinned memory --------------------------------------------------
// Serving creates and destroys domains continuously.  cudaMalloc / cudaFree (and
// cudaFreeHost) synchronise the whole device and return memory to the driver
// each time, tens of milliseconds per domain on a busy GPU.  The library
// therefore allocates device memory from its own stream-ordered pool per device
// with an unlimited release threshold (freed blocks stay cached for the next
// domain), on a private non-blocking stream: an allocation waits for that stream
// only and is then ready for any stream.  A free must come after the last work
// that uses the memory: lbf_domain_destroy first waits for the domain's last stream.
constexpr int MAX_DEV = 64;
struct DevPool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t s = nullptr;
};
std::mutex g_pool_mu;
DevPool g_pools[MAX_DEV];

cudaError_t pool_of(int dev, DevPool** out) {
    if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    DevPool& P = g_pools[dev];
    if (!P.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaError_t e = cudaMemPoolCreate(&P.pool, &props);
        if (e != cudaSuccess) { P.pool = nullptr; return e; }
        unsigned long long thr = ~0ull;
        e = cudaMemPoolSetAttribute(P.pool, cudaMemPoolAttrReleaseThreshold, &thr);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&P.s, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(P.pool);
            P.pool = nullptr;
            return e;
        }
    }
    *out = &P;
    return cudaSuccess;
}

int current_device() {
    int dev = 0;
    cudaGetDevice(&dev);
    return dev;
}

cudaError_t dev_alloc(void** p, size_t bytes, int dev) {
    *p = nullptr;
    DevPool* P = nullptr;
    cudaError_t e = pool_of(dev, &P);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, P->pool, P->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(P->s);
    if (e != cudaSuccess) *p = nullptr;
    return e;
}

void dev_free(void* p, int dev) {
    if (!p) return;
    DevPool* P = nullptr;
    if (pool_of(dev, &P) == cudaSuccess) cudaFreeAsync(p, P->s);
}

// Pinned 64-byte slots (residual read-backs) carved from 4 KiB pinned pages that
// are never released, so that no cudaFreeHost runs while serving.
std::mutex g_pin_mu;
std::vector<void*> g_pin_free;

void* pinned64() {
    std::lock_guard<std::mutex> lk(g_pin_mu);
    if (g_pin_free.empty()) {
        void* page = nullptr;
        if (cudaMallocHost(&page, 4096) != cudaSuccess) return nullptr;
        for (int i = 0; i < 64; ++i) g_pin_free.push_back((char*)page + 64 * i);
    }
    void* p = g_pin_free.back();
    g_pin_free.pop_back();
    return p;
}

void pinned64_free(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

// Device -> host copies of large results into caller memory (pageable, as a
// numpy array is): the bytes go through two pinned staging buffers, so the DMA
// of one chunk overlaps the host threads' copy of the previous one out of
// pinned memory.  The staging buffers are allocated once per process.
constexpr size_t STAGE_CHUNK = 32u << 20;
std::mutex g_stage_mu;
char* g_stage[2] = {nullptr, nullptr};
cudaEvent_t g_stage_ev[2] = {nullptr, nullptr};

void host_copy_parallel(char* dst, const char* src, size_t bytes) {
    const size_t per = 4u << 20;
    const int nt = (int)std::min<size_t>(std::max(1u, std::min(32u, std::thread::hardware_concurrency())),
                                         (bytes + per - 1) / per);
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t part = (bytes + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const size_t a = (size_t)t * part, b = std::min(bytes, a + part);
        if (a < b) th.emplace_back([=] { std::memcpy(dst + a, src + a, b - a); });
    }
    for (auto& x : th) x.join();
}

cudaError_t download(void* dst, const void* src, size_t bytes, cudaStream_t s) {
    // page-locked caller memory (cudaMallocHost, cudaHostRegister, a pinned tensor):
    // one direct copy at the full link rate
    cudaPointerAttributes pa;
    const cudaError_t ea = cudaPointerGetAttributes(&pa, dst);
    if (ea != cudaSuccess) cudaGetLastError();   // an unknown pointer is pageable memory, not an error
    const bool pinned = ea == cudaSuccess && pa.type == cudaMemoryTypeHost;
    if (pinned || bytes < (4u << 20)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
    }
    // fresh caller memory is faulted in by the copy: ask for huge pages (a hint,
    // ignored where transparent huge pages are off) to cut the page faults
    {
        const uintptr_t a = ((uintptr_t)dst + (2u << 20) - 1) & ~(uintptr_t)((2u << 20) - 1);
        const uintptr_t b = ((uintptr_t)dst + bytes) & ~(uintptr_t)((2u << 20) - 1);
        if (b > a) madvise((void*)a, b - a, MADV_HUGEPAGE);
    }
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (!g_stage[0]) {
        for (int k = 0; k < 2; ++k) {
            cudaError_t e = cudaMallocHost((void**)&g_stage[k], STAGE_CHUNK);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g_stage_ev[k], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
    }
    const size_t n = (bytes + STAGE_CHUNK - 1) / STAGE_CHUNK;
    for (size_t c = 0; c <= n; ++c) {
        if (c < n) {   // chunk c into buffer c & 1 (free: its previous chunk was copied out below)
            const size_t off = c * STAGE_CHUNK, len = std::min(STAGE_CHUNK, bytes - off);
            cudaError_t e = cudaMemcpyAsync(g_stage[c & 1], (const char*)src + off, len, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(g_stage_ev[c & 1], s);
            if (e != cudaSuccess) return e;
        }
        if (c > 0) {   // chunk c - 1 is in flight or landed: copy it out while chunk c transfers
            const size_t off = (c - 1) * STAGE_CHUNK, len = std::min(STAGE_CHUNK, bytes - off);
            cudaError_t e = cudaEventSynchronize(g_stage_ev[(c - 1) & 1]);
            if (e != cudaSuccess) return e;
            host_copy_parallel((char*)dst + off, g_stage[(c - 1) & 1], len);
        }
    }
    return cudaSuccess;
}

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
struct lbf_batch;
// An allocator whose resize leaves the new elements uninitialised (the caller
// writes every one): a lattice-sized host array is then touched once, not twice.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept { ::new ((void*)p) U; }
    template <class U, class... A>
    void construct(U* p, A&&... a) { ::new ((void*)p) U(std::forward<A>(a)...); }
};

struct lbf_domain {
    lbf_domain_desc desc{};
    int vs = 0, q = 0, d = 0, st = 0, nfaces = 0;
    long long n[3] = {1, 1, 1};
    long long N = 0;
    unsigned long long n_fluid = 0, n_bb = 0;
    bool facebc = false, prepared = false, initialized = false;
    unsigned folded = 0;   // no-slip faces applied through the link bits of the pull
    // host copies of the inputs (solid-node outputs, re-initialisation)
    std::vector<uint8_t, NoInitAlloc<uint8_t>> type;   // filled once, in lbf_domain_create
    std::vector<double> rho0, u0;
    double rho0u = 1.0, u0u[3] = {0, 0, 0};
    // passive scalars (passive_scalar::LatticeVec): one momentum sweep advances all
    int ns = 0;
    bool scalar = false;          // ns > 0
    lbf_scalar_desc sdesc[NSMAX] = {};
    std::vector<double> c0[NSMAX];   // per-node initial scalar (host copy), or empty
    // device memory
    void* pop[2] = {nullptr, nullptr};
    void* gpop[NSMAX][2] = {};
    uint32_t* mask = nullptr;
    uint8_t* dtype = nullptr;
    void* mom[2] = {nullptr, nullptr};
    void* pb[6][2] = {};
    void* snap[NSMAX][6] = {};
    unsigned outflow = 0;   // faces with a scalar extrapolation outflow of any scalar (face pass)
    unsigned outflow_s[NSMAX] = {};
    long long pb_plane[6] = {0, 0, 0, 0, 0, 0};
    void* qads[NSMAX] = {};
    void* cprev[NSMAX] = {};
    double* c_init_dev[NSMAX] = {};
    double* accum = nullptr;      // per-block partial sums: [accumulator][accum_cap]
    long long accum_cap = 0;      // slots per accumulator (the most blocks any launch of the domain uses)
    long long slot_next = 0;      // next free slot of the step being launched
    double* res_dev = nullptr;
    double* res_host = nullptr;   // pinned
    double* obs = nullptr;        // rho | u | c  (doubles)
    unsigned long long* counts = nullptr;
    std::vector<double> lam;      // D3Q27 MRT collision matrix
    long long t = 0;
    bool part_pending = false;    // a split step ran its part 0 (boundary planes) and waits for part 1
    long long res_step = -1;
    int block_x = 0;
    bool stage = false;           // one-shot staged sweep (off: the pipelined sweep supersedes it)
    bool pipe = false;            // pipelined bulk-copy sweep on the lean path (option)
    int pipe_stages = 0;          // 0 = chosen from the shared-memory budget
    bool compact = false;         // compacted sweep over a work list on the lean path (in effect)
    int compact_opt = -1;         // -1 = default (FP64 storage, D3Q27), 0 off, 1 on
    long long z_begin = 0, z_end = 0;   // planes swept (0, 0 = all); a z-slab sweeps its owned planes
    int sparse_opt = -1;          // fluid-only layout on the lean path: 1 on, 0 off, -1 auto (>= 5 % solid)
    bool sparse = false;          // the sparse layout is in effect: list = fluid cells, pop planes of Np fluid slots
    uint32_t* fmask = nullptr;    // sparse: mask word per fluid node
    uint2* rw = nullptr;          // sparse: row words (fluid bits, first fluid index), plus a sentinel row
    std::vector<long long> zoff;  // sparse: first fluid index of each z plane, then the fluid count
    int rw_w = 0;                 // sparse: words per row
    bool sparse_packed = false;   // sparse: list entries hold packed coordinates
    int stream_opt = -1;          // LBF_OPT_STREAMING: streaming scheme of the lean sparse layout (-1 auto)
    bool inplace = false;         // in effect: AA pattern, one population buffer (pop[0]); steps alternate even / odd
    bool push = false;            // in effect: push sweep (two buffers, the state is the post-stream field)
    int sround = 1;               // 16-bit storage: stochastic rounding
    long long wait_limit = -1;    // LBF_OPT_WAIT_LIMIT: polls of the staged sweeps' bounded waits (-1 default)
    long long seed_offset = 0;    // LBF_OPT_SEED_OFFSET: node index of node 0 in the whole lattice
    uint32_t* list = nullptr;     // work entries (fluid nodes + solid nodes sharing a sector)
    long long nlist = 0;
    long long Np = 0;             // population plane stride: N rounded up to 64 nodes
    int* err = nullptr;           // device flag: a bounded wait gave up
    cudaStream_t last_stream = nullptr;
    // the side stream and events of the face-pass overlap (do_steps), made on first use
    cudaStream_t side = nullptr;
    cudaEvent_t ev_bulk = nullptr, ev_head = nullptr;
    long long bytes = 0;
    lbf_batch* batch = nullptr;   // set while the domain is admitted to a batch
    int dev = 0;                  // device that holds the domain's memory

    ~lbf_domain() {
        if (ev_bulk) cudaEventDestroy(ev_bulk);
        if (ev_head) cudaEventDestroy(ev_head);
        if (side) cudaStreamDestroy(side);
        for (int k = 0; k < 2; ++k) {
            dev_free(pop[k], dev); dev_free(mom[k], dev);
            for (int f = 0; f < 6; ++f) dev_free(pb[f][k], dev);
        }
        for (int si = 0; si < NSMAX; ++si) {
            dev_free(gpop[si][0], dev); dev_free(gpop[si][1], dev);
            for (int f = 0; f < 6; ++f) dev_free(snap[si][f], dev);
            dev_free(qads[si], dev); dev_free(cprev[si], dev); dev_free(c_init_dev[si], dev);
        }
        for (void* p : {(void*)mask, (void*)dtype, (void*)accum, (void*)res_dev,
                        (void*)obs, (void*)counts, (void*)err, (void*)list, (void*)fmask, (void*)rw})
            dev_free(p, dev);
        pinned64_free(res_host);
    }
    // per-node moment fields: rho, u_0..u_{d-1}, one per scalar
    int nfields() const { return 1 + d + ns; }
    // residual accumulators of the step kernel: rho, u_0..u_2, then one per scalar slot
    int nacc() const { return ns > 0 ? 4 + NSMAX : 5; }
    // fields of a face layer: u_0..u_{d-1}, then one per scalar (at least one)
    int pb_nf() const { return d + std::max(ns, 1); }
};

namespace {

lbf_status dmalloc(lbf_domain* D, void** p, size_t bytes) {
    cudaError_t e = dev_alloc(p, bytes, D->dev);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,
                    std::string("device allocation (") + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e));
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
long long zb(const lbf_domain* D) { return D->z_end > 0 ? D->z_begin : 0; }
long long ze(const lbf_domain* D) { return D->z_end > 0 ? D->z_end : D->n[2]; }
bool z_restricted(const lbf_domain* D) { return zb(D) != 0 || ze(D) != D->n[2]; }

dim3 step_grid(const lbf_domain* D, dim3 b) {
    return dim3((unsigned)((D->n[0] + b.x - 1) / b.x), (unsigned)D->n[1], (unsigned)(ze(D) - zb(D)));
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
            if (vel || prs) return true;
            why = "Error: Wrong input of Zou & He (1997) boundary conditions.";
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
        // a folded face has no explicit rule left: the pull's link bits apply it
        P.face[f].kind = f < D->nfaces && !(D->folded >> f & 1u) ? b.kind : BC_PERIODIC;
        P.face[f].has_rho = b.has_density;
        for (int a = 0; a < 3; ++a) { P.face[f].has_u[a] = b.has_velocity[a]; P.face[f].u[a] = b.velocity[a]; }
        P.face[f].rho = b.density;
        P.pb_plane[f] = D->pb_plane[f];
    }
    bool zero = true;
    for (int f = 0; f < 6; ++f) zero = zero && D->desc.face_order[f] == 0;
    for (int o = 0; o < 6; ++o) P.order[o] = zero ? o : D->desc.face_order[o];
    for (int si = 0; si < D->ns; ++si) {
        for (int f = 0; f < 6; ++f) {
            const lbf_scalar_bc_desc& s = D->sdesc[si].bc[f];
            SFaceBC& o = P.sc[si].face[f];
            o.kind = f < D->nfaces && !(D->folded >> f & 1u) ? s.kind : SBC_PERIODIC;
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

// Scalars with adsorption, one bit each (checkpoint header).
int32_t ads_bits(const lbf_domain* D) {
    int32_t b = 0;
    for (int si = 0; si < D->ns; ++si) if (D->qads[si]) b |= 1 << si;
    return b;
}

// Observed moments (doubles, N each): rho, u_0..u_{d-1}, one per scalar (at least one).
int obs_fields(const lbf_domain* D) { return 1 + D->d + std::max(D->ns, 1); }

bool face_needs_layers(const lbf_domain* D, int f) {
    if (f >= D->nfaces) return false;
    if (D->desc.bc[f].kind == LBF_BC_ANTI_BOUNCE_BACK) return true;
    for (int si = 0; si < D->ns; ++si) {
        const int k = D->sdesc[si].bc[f].kind;
        if (k == LBF_SBC_ANTI_BB_NO_FLUX) return true;
        if (k == LBF_SBC_ANTI_BOUNCE_BACK) {
            const lbf_bc_desc& m = D->desc.bc[f];
            if (m.kind == LBF_BC_NO_SLIP || m.kind == LBF_BC_BOUNCE_BACK) continue;
            if (m.kind == LBF_BC_ZOU_HE) {
                bool all = true;
                for (int a = 0; a < D->d; ++a) all = all && m.has_velocity[a];
                if (all) continue;
            }
            return true;
        }
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
    cudaError_t e = dev_alloc((void**)&keep, N, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&val, N * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&nsel, sizeof(int), D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&D->list, N * 4, D->dev);
    if (e == cudaSuccess) {
        const unsigned nb = (unsigned)((N + 255) / 256);
        if (D->d == 2) k_list_mark<2><<<nb, 256, 0, s>>>(D->mask, N, (int)D->n[0], (int)D->n[1], (int)D->n[2], per, keep, val);
        else k_list_mark<3><<<nb, 256, 0, s>>>(D->mask, N, (int)D->n[0], (int)D->n[1], (int)D->n[2], per, keep, val);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, tmp_bytes, val, keep, D->list, nsel, (int)N, s);
    if (e == cudaSuccess) e = dev_alloc(&tmp, tmp_bytes, D->dev);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tmp_bytes, val, keep, D->list, nsel, (int)N, s);
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(keep, D->dev); dev_free(val, D->dev); dev_free(nsel, D->dev); dev_free(tmp, D->dev);
    if (e != cudaSuccess) {
        dev_free(D->list, D->dev);
        D->list = nullptr;
        st = fail(e == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,
                  std::string("work list: ") + cudaGetErrorString(e));
    } else {
        D->nlist = h;
        D->bytes += N * 4;
    }
    return st;
}

// The sparse layout (lean path): the fluid cells in node order, their mask
// words, the row words, and population planes of fluid slots only.
lbf_status build_sparse(lbf_domain* D, cudaStream_t s) {
    const long long N = D->N, F = (long long)D->n_fluid;
    // nothing to sweep, or element offsets of the planes beyond 32 bits: stay dense
    if (F == 0 || F >= (1ll << 31) || (long long)D->q * ((F + 63) / 64 * 64) >= (1ll << 32)) return LBF_OK;
    const int nx = (int)D->n[0];
    const int W = (nx + 31) / 32;
    const long long nrows = D->n[1] * D->n[2], nw = nrows * W;
    uint8_t* flag = nullptr;
    uint32_t *val = nullptr, *flist = nullptr, *bits = nullptr, *cnt = nullptr, *off = nullptr;
    int* nsel = nullptr;
    void* tmp = nullptr;
    size_t tb1 = 0, tb2 = 0;
    lbf_status st = LBF_OK;
    cudaError_t e = dev_alloc((void**)&flag, N, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&val, N * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&nsel, sizeof(int), D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&bits, nw * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&cnt, nw * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&off, nw * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&flist, F * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&D->fmask, F * 4, D->dev);
    if (e == cudaSuccess) e = dev_alloc((void**)&D->rw, (nw + W) * sizeof(uint2), D->dev);
    if (e == cudaSuccess) {
        k_fluid_flags<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(D->mask, N, flag, val);
        k_row_bits<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(D->mask, nx, nrows, W, bits, cnt);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(nullptr, tb1, val, flag, flist, nsel, (int)N, s);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(nullptr, tb2, cnt, off, (int)nw, s);
    if (e == cudaSuccess) e = dev_alloc(&tmp, std::max(tb1, tb2), D->dev);
    if (e == cudaSuccess) e = cub::DeviceSelect::Flagged(tmp, tb1, val, flag, flist, nsel, (int)N, s);
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(tmp, tb2, cnt, off, (int)nw, s);
    if (e == cudaSuccess) {
        k_row_words<<<(unsigned)((nw + W + 255) / 256), 256, 0, s>>>(bits, off, nw, W, (uint32_t)F, D->rw);
        k_gather_mask<<<(unsigned)((F + 255) / 256), 256, 0, s>>>(D->mask, flist, F, D->fmask);
        D->sparse_packed = D->n[0] <= 2048 && D->n[1] <= 2048 && D->n[2] <= 1024;
        if (D->sparse_packed) k_pack_xyz<<<(unsigned)((F + 255) / 256), 256, 0, s>>>(flist, F, nx, (int)D->n[1]);
        e = cudaGetLastError();
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, s);
    // the first row word of every z plane (and of the sentinel row) holds the
    // plane's first fluid index
    std::vector<uint2> zw((size_t)D->n[2] + 1);
    if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(zw.data(), sizeof(uint2), D->rw, (size_t)D->n[1] * W * sizeof(uint2), sizeof(uint2),
                              (size_t)D->n[2] + 1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && h != F) e = cudaErrorUnknown;
    if (e == cudaSuccess) {
        D->zoff.resize(zw.size());
        for (size_t z = 0; z < zw.size(); ++z) D->zoff[z] = zw[z].y;
    }
    dev_free(flag, D->dev); dev_free(val, D->dev); dev_free(nsel, D->dev); dev_free(tmp, D->dev);
    dev_free(bits, D->dev); dev_free(cnt, D->dev); dev_free(off, D->dev);
    // population planes of fluid slots only (one buffer when streaming in place)
    const long long Fp = (F + 63) / 64 * 64;
    const size_t eb = st_bytes(D->st);
    const bool lean = !D->facebc && !D->scalar;
    const bool whole = !z_restricted(D) && lean;
    const int scheme = D->stream_opt < 0 ? LBF_STREAM_PULL : D->stream_opt;
    const bool inplace = whole && scheme == LBF_STREAM_INPLACE;
    D->push = whole && scheme == LBF_STREAM_PUSH;
    void* np[2] = {nullptr, nullptr};
    void* ng[NSMAX][2] = {};
    const size_t rb = rt_bytes(D->st);
    if (e == cudaSuccess) e = dev_alloc(&np[0], (size_t)D->q * Fp * eb, D->dev);
    if (e == cudaSuccess && !inplace) e = dev_alloc(&np[1], (size_t)D->q * Fp * eb, D->dev);
    for (int si = 0; si < D->ns; ++si)
        for (int k = 0; k < 2 && e == cudaSuccess; ++k) e = dev_alloc(&ng[si][k], (size_t)D->q * Fp * rb, D->dev);
    if (e != cudaSuccess) {
        dev_free(flist, D->dev); dev_free(np[0], D->dev); dev_free(np[1], D->dev);
        for (int si = 0; si < D->ns; ++si) { dev_free(ng[si][0], D->dev); dev_free(ng[si][1], D->dev); }
        dev_free(D->fmask, D->dev); dev_free(D->rw, D->dev);
        D->fmask = nullptr; D->rw = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? LBF_ENOMEM : LBF_EDEVICE,
                    std::string("sparse layout: ") + cudaGetErrorString(e));
    }
    const long long old_bytes = D->pop[0] ? 2ll * D->q * D->Np * (long long)eb : 0;
    dev_free(D->pop[0], D->dev);
    dev_free(D->pop[1], D->dev);
    D->pop[0] = np[0];
    D->pop[1] = np[1];
    for (int si = 0; si < D->ns; ++si) {
        const long long old_g = D->gpop[si][0] ? 2ll * D->q * D->Np * (long long)rb : 0;
        dev_free(D->gpop[si][0], D->dev);
        dev_free(D->gpop[si][1], D->dev);
        D->gpop[si][0] = ng[si][0];
        D->gpop[si][1] = ng[si][1];
        D->bytes += 2ll * D->q * Fp * (long long)rb - old_g;
    }
    D->Np = Fp;
    D->inplace = inplace;
    D->bytes += (inplace ? 1ll : 2ll) * D->q * Fp * (long long)eb - old_bytes + F * 8 + (nw + W) * 8;
    D->list = flist;
    D->nlist = F;
    D->rw_w = W;
    D->sparse = true;
    return st;
}

// A no-slip face (bc.rs NoSlip: f[ibar] = f*[i] of the node itself for each i
// leaving through the face) is the inner bounce-back of a solid layer beyond the
// face, so the pull applies it through the node's link bits.  Among explicit
// faces that is exact when the folded rule would run first at every node it
// shares with an explicit face, i.e. the face precedes, in the face order, each
// explicit face that meets it along an edge (folded rules read only the node's
// own post-collision slots, so they commute with one another).  With a scalar
// the scalar rule of the face must be the same bounce-back (BBNoFlux) and the
// inner rule InnerBounceBack, which the link bits apply to the scalar.
// Folding keeps the long face code off the bulk of the lattice: only nodes on
// the remaining explicit faces run it.
unsigned foldable_faces(const lbf_domain* D, unsigned expl) {
    int pos[6] = {0, 1, 2, 3, 4, 5};
    bool zero = true;
    for (int f = 0; f < 6; ++f) zero = zero && D->desc.face_order[f] == 0;
    if (!zero)
        for (int o = 0; o < D->nfaces; ++o)
            if (D->desc.face_order[o] >= 0 && D->desc.face_order[o] < 6) pos[D->desc.face_order[o]] = o;
    unsigned cand = 0;
    for (int f = 0; f < D->nfaces; ++f) {
        if (D->desc.bc[f].kind != LBF_BC_NO_SLIP) continue;
        bool same = true;
        for (int si = 0; si < D->ns; ++si)
            same = same && D->sdesc[si].bc[f].kind == LBF_SBC_BB_NO_FLUX &&
                   D->sdesc[si].inner_boundary_condition == LBF_INNER_BOUNCE_BACK;
        if (same) cand |= 1u << f;
    }
    unsigned fold = 0;
    for (int f = 0; f < D->nfaces; ++f) {
        if (!(cand >> f & 1u)) continue;
        bool ok = true;
        for (int g = 0; g < D->nfaces; ++g) {
            const bool meets = g / 2 != f / 2 || (g != f && D->n[f / 2] == 1);
            if ((expl >> g & 1u) && !(cand >> g & 1u) && meets && pos[g] < pos[f]) ok = false;
        }
        if (ok) fold |= 1u << f;
    }
    return fold;
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
            bool sper = true;
            for (int si = 0; si < D->ns; ++si) sper = sper && D->sdesc[si].bc[f].kind == LBF_SBC_PERIODIC;
            if (k != LBF_BC_PERIODIC || !sper) expl |= 1u << f;
        } else if (k == LBF_BC_NO_SLIP) {
            fold |= 1u << f;
        }
    }
    if (D->facebc) {
        fold = foldable_faces(D, expl);
        expl &= ~fold;
    }
    D->folded = fold;
    uint32_t* cls = nullptr;
    uint32_t* links = nullptr;
    lbf_status st;
    if (!D->mask && (st = dmalloc(D, (void**)&D->mask, N * 4))) return st;
    if ((st = dmalloc(D, (void**)&cls, N * 4))) return st;
    if ((st = dmalloc(D, (void**)&links, N * 4))) { dev_free(cls, D->dev); return st; }
    D->bytes -= 8 * N;
    if (!D->counts && (st = dmalloc(D, (void**)&D->counts, 16))) { dev_free(cls, D->dev); dev_free(links, D->dev); return st; }
    if (!D->dtype && (st = dmalloc(D, (void**)&D->dtype, N))) { dev_free(cls, D->dev); dev_free(links, D->dev); return st; }
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
    dev_free(cls, D->dev);
    dev_free(links, D->dev);
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("node classification: ") + cudaGetErrorString(e));
    D->n_fluid = cnt[0];
    D->n_bb = cnt[1];
    // face layers and outflow snapshots
    for (int f = 0; f < D->nfaces; ++f) D->pb_plane[f] = N / D->n[f / 2];
    for (int f = 0; f < 6; ++f) {
        const long long plane = D->pb_plane[f];
        if (face_needs_layers(D, f))
            for (int k = 0; k < 2; ++k)
                if (!D->pb[f][k] && (st = dmalloc(D, &D->pb[f][k], 2 * D->pb_nf() * plane * rt_bytes(D->st)))) return st;
        for (int si = 0; si < D->ns; ++si) {
            if ((D->outflow_s[si] >> f & 1u) && !D->snap[si][f]) {
                const size_t b = 2 * (size_t)D->q * plane * rt_bytes(D->st);
                if ((st = dmalloc(D, &D->snap[si][f], b))) return st;
                CK(cudaMemsetAsync(D->snap[si][f], 0, b, s));   // solid neighbours read as zero populations
            }
        }
    }
    if (D->sparse) {             // already laid out (a repeated classification keeps the state)
        D->prepared = true;
        return LBF_OK;
    }
    D->nlist = 0;
    if (D->list) { dev_free(D->list, D->dev); D->list = nullptr; }
    // the sparse sweep also serves z-slabs (it updates the fluid slots of the owned
    // planes) and, whole lattices only, explicit faces and the scalar
    const bool lean = !D->facebc && !D->scalar;
    const bool porous = (double)D->n_fluid <= 0.95 * (double)N;
    if ((lean || !z_restricted(D)) && (D->sparse_opt > 0 || (D->sparse_opt < 0 && porous)) && !D->initialized) {
        if ((st = build_sparse(D, s))) return st;
        if (D->sparse) {
            D->compact = false;
            D->prepared = true;
            return LBF_OK;
        }
    }
    // the dense layout: A/B population buffers of every node (and the scalar's)
    for (int k = 0; k < 2; ++k) {
        if (!D->pop[k] && (st = dmalloc(D, &D->pop[k], (size_t)D->q * D->Np * st_bytes(D->st)))) return st;
        for (int si = 0; si < D->ns; ++si)
            if (!D->gpop[si][k] && (st = dmalloc(D, &D->gpop[si][k], (size_t)D->q * D->Np * rt_bytes(D->st))))
                return st;
    }
    // the work list wins for FP64 and for D3Q27 (its 256-thread blocks fit 64
    // registers, four per SM, for BGK, TRT and central moments; the dense D3Q27
    // sweep keeps 128): Taylor-Green 384^3, central, FP32 24.5k MLUPS against
    // 16.3k dense, FP16 deviations 25.4k against 18.8k.  D3Q27 MRT (the 27 x 27
    // population-space matrix) spills at 64 registers and stays dense.
    const bool dflt = D->st == LBF_STORE_F64 || (D->vs == LBF_D3Q27 && D->desc.collision.kind != LBF_MRT);
    const bool want = (D->compact_opt < 0 ? dflt : D->compact_opt != 0) && !z_restricted(D);
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
    P.wait_limit = D->wait_limit;
    P.list = D->list;
    P.nlist = D->nlist;
    P.kbeg = 0;
    P.kend = D->nlist;
    if (D->sparse && z_restricted(D)) {
        P.kbeg = D->zoff[(size_t)zb(D)];
        P.kend = D->zoff[(size_t)ze(D)];
    }
    P.inv_nx = 1.0 / (double)D->n[0];
    P.inv_ny = 1.0 / (double)D->n[1];
    P.z0 = (int)zb(D);
    P.fmask = D->fmask;
    P.rw = D->rw;
    P.rw_w = D->rw_w;
    P.np = D->Np;
    P.packed = D->sparse_packed ? 1 : 0;
    const size_t eb = st_bytes(D->st);
    // in place: one buffer, read and written by every step (even and odd placements)
    const int rd = D->inplace ? 0 : (int)(t & 1), wr = D->inplace ? 0 : (int)((t + 1) & 1);
    for (int i = 0; i < D->q; ++i) {
        P.srcp[i] = (const char*)D->pop[rd] + (size_t)i * D->Np * eb;
        P.dstp[i] = (char*)D->pop[wr] + (size_t)i * D->Np * eb;
    }
    P.sweep_mode = D->inplace ? ((t & 1) ? SWEEP_AA_ODD : SWEEP_AA_EVEN) : (D->push ? SWEEP_PUSH : SWEEP_PULL);
    P.sround = D->sround;
    P.tstep = (unsigned)t;
    P.seed_offset = D->seed_offset;
    const lbf_collision_desc& c = D->desc.collision;
    P.coll = c.kind; P.compat = D->desc.compat; P.has_force = D->desc.has_force; P.first = t == 0;
    P.tau = c.tau;
    P.omega = (c.kind == LBF_BGK || c.kind == LBF_CENTRAL) ? 1.0 / c.tau : 0.0;
    P.op = c.omega_plus; P.om = c.omega_minus;
    P.bgk_cb = c.kind == LBF_BGK ? 1.0 - 0.5 / c.tau : 0.0;
    for (int k = 0; k < 27; ++k) P.rates[k] = c.relaxation[k];
    if (c.kind == LBF_CENTRAL)   // bulk, 3rd .. 6th order rates; <= 0 means full relaxation
        for (int k = 0; k < 5; ++k) P.rates[k] = c.relaxation[k] > 0.0 ? c.relaxation[k] : 1.0;
    for (int a = 0; a < 3; ++a) P.force[a] = D->desc.has_force ? D->desc.force[a] : 0.0;
    fill_face_params(D, P);
    P.any_face = 0;
    for (int f = 0; f < 6; ++f) {
        P.pb_src[f] = D->pb[f][(t + 1) & 1];
        P.pb_dst[f] = D->pb[f][t & 1];
        if (D->pb[f][0]) P.any_face = 1;
    }
    P.mom_prev = D->mom[(t + 1) & 1];
    P.mom_cur = D->mom[t & 1];
    P.accum = D->accum;
    P.accum_stride = D->accum_cap;
    P.slot0 = 0;
    P.pb_nf = D->pb_nf();
    P.has_scalar = D->ns > 0 ? 1 : 0;
    P.nscalar = D->ns;
    for (int si = 0; si < D->ns; ++si) {
        const lbf_scalar_desc& s = D->sdesc[si];
        ScalarParams& o = P.sc[si];
        o.coll = s.collision.kind; o.inner = s.inner_boundary_condition; o.has_source = s.has_source;
        o.tau = s.collision.tau; o.omega = s.collision.kind == LBF_BGK ? 1.0 / s.collision.tau : 0.0;
        o.bgk_cb = s.collision.kind == LBF_BGK ? 1.0 - 0.5 / s.collision.tau : 0.0;
        o.op = s.collision.omega_plus; o.om = s.collision.omega_minus; o.source = s.source_value;
        o.ads = s.has_adsorption;
        o.ka = s.adsorption_rate; o.kd = s.desorption_rate; o.qmax = s.q_max;
        o.c_solid = s.initial_scalar_value;
        o.c_init = D->c_init_dev[si];
        o.gsrc = D->gpop[si][t & 1];
        o.gdst = D->gpop[si][(t + 1) & 1];
        o.qads = D->qads[si];
        o.cprev = D->cprev[si];
        for (int f = 0; f < 6; ++f) o.snap[f] = D->snap[si][f];
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
    if (z_restricted(D)) return false;
    const size_t rowb = D->n[0] * st_bytes(D->st);
    return !D->facebc && !D->scalar && rowb % 16 == 0 && 2 * D->q * rowb <= 200 * 1024;
}

// Every launch of a residual step writes its blocks' partial sums to its own
// range of slots, from D->slot_next on (reset at the start of each step); the
// finalize sums the D->slot_next slots the step filled.
long long take_slots(lbf_domain* D, StepParams& P, long long blocks) {
    P.slot0 = D->slot_next;
    D->slot_next += blocks;
    return blocks;
}

// Calls fn(IC<VS>, IC<COLL>) for the domain's velocity set and collision (the
// central-moment collision exists for the tensor-product sets only).
template <class Fn>
cudaError_t by_kind(const lbf_domain* D, Fn&& fn) {
    const int c = D->desc.collision.kind;
    switch (D->vs) {
        case LBF_D2Q9:
            switch (c) {
                case LBF_BGK: return fn(IC<VS_D2Q9>{}, IC<COLL_BGK>{});
                case LBF_TRT: return fn(IC<VS_D2Q9>{}, IC<COLL_TRT>{});
                case LBF_MRT: return fn(IC<VS_D2Q9>{}, IC<COLL_MRT>{});
                default: return fn(IC<VS_D2Q9>{}, IC<COLL_CENTRAL>{});
            }
        case LBF_D3Q19:
            switch (c) {
                case LBF_BGK: return fn(IC<VS_D3Q19>{}, IC<COLL_BGK>{});
                case LBF_TRT: return fn(IC<VS_D3Q19>{}, IC<COLL_TRT>{});
                case LBF_MRT: return fn(IC<VS_D3Q19>{}, IC<COLL_MRT>{});
                default: return cudaErrorInvalidValue;
            }
        default:
            switch (c) {
                case LBF_BGK: return fn(IC<VS_D3Q27>{}, IC<COLL_BGK>{});
                case LBF_TRT: return fn(IC<VS_D3Q27>{}, IC<COLL_TRT>{});
                case LBF_MRT: return fn(IC<VS_D3Q27>{}, IC<COLL_MRT>{});
                default: return fn(IC<VS_D3Q27>{}, IC<COLL_CENTRAL>{});
            }
    }
}
const double* lam_of(const lbf_domain* D) { return D->lam.empty() ? nullptr : D->lam.data(); }

cudaError_t launch_pipe(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    const size_t stage_b = (size_t)D->q * D->n[0] * st_bytes(D->st);
    // three blocks of <= 288 threads per SM share ~220 KB of shared memory
    int stages = D->pipe_stages > 0 ? D->pipe_stages : (int)std::max<size_t>(2, std::min<size_t>(8, (72 * 1024) / stage_b));
    while (stages > 2 && stages * stage_b > 200 * 1024) --stages;
    const int nc = (int)std::min<long long>(8, std::max<long long>(1, (D->n[0] + 31) / 32));
    return by_kind(D, [&](auto V, auto C) {
        return launch_step_pipe<decltype(V)::value, decltype(C)::value>(D->st, P, lam_of(D), stages, nc, s);
    });
}

cudaError_t launch_list(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    return by_kind(D, [&](auto V, auto C) {
        return launch_step_list<decltype(V)::value, decltype(C)::value>(D->st, P, lam_of(D), s);
    });
}

// Sparse sweep with explicit faces and/or the scalar: the bulk launch, then one
// face pass per scalar outflow face (as launch_step_any does for the dense sweep).
cudaError_t sparse_fs_launch(lbf_domain* D, const StepParams& Q, unsigned blocks, cudaStream_t s) {
    return by_kind(D, [&](auto V, auto C) {
        return launch_step_sparse_fs<decltype(V)::value, decltype(C)::value>(D->st, D->scalar, Q, lam_of(D), blocks,
                                                                             s);
    });
}

// The bulk launch of the sparse face/scalar sweep over the fluid slots [kb, ke).
cudaError_t sparse_fs_bulk(lbf_domain* D, const StepParams& P, long long kb, long long ke, cudaStream_t s) {
    if (ke <= kb) return cudaSuccess;
    StepParams B = P;
    B.kbeg = kb;
    B.kend = ke;
    const unsigned nb = (unsigned)((ke - kb + 255) / 256);
    take_slots(D, B, nb);
    return sparse_fs_launch(D, B, nb, s);
}

// The face passes of the scalar outflow faces (after the bulk launch of the step).
cudaError_t sparse_fs_faces(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    for (int f = 0; f < D->nfaces && e == cudaSuccess; ++f) {
        if (!(D->outflow >> f & 1u)) continue;
        StepParams F = P;
        F.face_pass = 1;
        F.fp_face = f;
        const unsigned nf = (unsigned)((D->pb_plane[f] + 255) / 256);
        take_slots(D, F, nf);
        e = sparse_fs_launch(D, F, nf, s);
    }
    return e;
}

cudaError_t launch_sparse_fs(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    auto one = [&](const StepParams& Q, unsigned blocks) -> cudaError_t { return sparse_fs_launch(D, Q, blocks, s); };
    StepParams B = P;
    const unsigned nb = (unsigned)((P.kend - P.kbeg + 255) / 256);
    take_slots(D, B, nb);
    cudaError_t e = one(B, nb);
    for (int f = 0; f < D->nfaces && e == cudaSuccess; ++f) {
        if (!(D->outflow >> f & 1u)) continue;
        StepParams F = P;
        F.face_pass = 1;
        F.fp_face = f;
        const unsigned nf = (unsigned)((D->pb_plane[f] + 255) / 256);
        take_slots(D, F, nf);
        e = one(F, nf);
    }
    return e;
}

cudaError_t launch_sparse(lbf_domain* D, const StepParams& P, cudaStream_t s) {
    if (D->facebc || D->scalar) return launch_sparse_fs(D, P, s);
    StepParams B = P;
    take_slots(D, B, (P.kend - P.kbeg + 255) / 256);
    return by_kind(D, [&](auto V, auto C) {
        return launch_step_sparse<decltype(V)::value, decltype(C)::value>(D->st, B, lam_of(D), s);
    });
}

// The bulk sweep, then one face pass per scalar outflow face.
cudaError_t launch_step_any(lbf_domain* D, const StepParams& P0, cudaStream_t s) {
    StepParams P = P0;
    if (D->sparse) return launch_sparse(D, P, s);
    const bool lean = !D->facebc && !D->scalar && !P.first && !P.observe && !P.face_pass;
    // the persistent pipelined sweep is used on steps without residuals only
    if (D->pipe && lean && !P.residual && can_pipe(D)) {
        cudaError_t e = launch_pipe(D, P, s);
        if (e != cudaErrorNotSupported) return e;
        cudaGetLastError();
    }
    if (lean && D->compact && D->list) {
        take_slots(D, P, (D->nlist + 255) / 256);
        return launch_list(D, P, s);
    }
    const bool stage = D->stage && can_stage(D);
    const dim3 b = stage ? dim3((unsigned)D->n[0]) : step_block(D);
    const dim3 g = step_grid(D, b);
    take_slots(D, P, (long long)g.x * g.y * g.z);
    cudaError_t e = launch_one(D, P, stage, Launch{g, b, s});
    for (int f = 0; f < D->nfaces && e == cudaSuccess; ++f) {
        if (!(D->outflow >> f & 1u)) continue;
        StepParams F = P;
        F.face_pass = 1;
        F.fp_face = f;
        const unsigned nb = (unsigned)((D->pb_plane[f] + 127) / 128);
        take_slots(D, F, nb);
        e = launch_one(D, F, false, Launch{dim3(nb), dim3(128), s});
    }
    return e;
}

// The slots a residual step (not the first step) of the whole lattice fills: the
// same launch shapes as launch_step_any.
long long residual_step_slots(const lbf_domain* D) {
    long long faces = 0;
    if (D->sparse) {
        for (int f = 0; f < D->nfaces; ++f)
            if (D->outflow >> f & 1u) faces += (D->pb_plane[f] + 255) / 256;
        return (D->nlist + 255) / 256 + faces;
    }
    for (int f = 0; f < D->nfaces; ++f)
        if (D->outflow >> f & 1u) faces += (D->pb_plane[f] + 127) / 128;
    if (!D->facebc && !D->scalar && D->compact && D->list) return (D->nlist + 255) / 256;
    const dim3 b = (D->stage && can_stage(D)) ? dim3((unsigned)D->n[0]) : step_block(D);
    const dim3 g = step_grid(D, b);
    return (long long)g.x * g.y * g.z + faces;
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
    if (D->z_end > 0 && D->z_begin >= D->z_end) return fail(LBF_EINVAL, "swept z planes: need z_begin < z_end");
    if (!D->prepared && (st = prepare(D, nullptr, nullptr, s))) return st;
    if ((st = ensure_mom(D))) return st;
    StepParams P;
    base_params(D, P, 0);
    P.mom_prev = D->mom[1];   // seeded with the initial moments (ShallowNode)
    InitParams I{};
    I.rho0 = D->rho0u;
    for (int a = 0; a < 3; ++a) I.u0[a] = D->u0u[a];
    for (int si = 0; si < D->ns; ++si) {
        I.c0[si] = D->sdesc[si].initial_scalar_value;
        I.q0[si] = D->sdesc[si].initial_q_ads;
        I.c_field[si] = D->c_init_dev[si];   // the per-node initial scalar, resident since attach
    }
    // upload per-node initial fields for the duration of the init kernel
    double* tmp = nullptr;
    const size_t nr = D->rho0.empty() ? 0 : D->N, nu = D->u0.empty() ? 0 : D->N * D->d;
    if (nr + nu) {
        CK(dev_alloc((void**)&tmp, (nr + nu) * sizeof(double), D->dev));
        if (nr) CK(cudaMemcpyAsync(tmp, D->rho0.data(), nr * 8, cudaMemcpyHostToDevice, s));
        if (nu) CK(cudaMemcpyAsync(tmp + nr, D->u0.data(), nu * 8, cudaMemcpyHostToDevice, s));
        I.rho_field = nr ? tmp : nullptr;
        I.u_field = nu ? tmp + nr : nullptr;
    }
    void* pb[12];
    for (int f = 0; f < 6; ++f) { pb[2 * f] = D->pb[f][0]; pb[2 * f + 1] = D->pb[f][1]; }
    Launch L{dim3((unsigned)((D->N + 255) / 256)), dim3(256), s};
    cudaError_t e = cudaSuccess;
    if (D->sparse && (D->facebc || D->scalar)) {
        // the per-node side arrays (residual moments, adsorbed amount, previous
        // scalar value, face layers) by node; the populations by fluid slot below
        I.skip_pops = 1;
        e = D->vs == LBF_D2Q9 ? launch_init<VS_D2Q9>(D->st, D->scalar, P, I, pb, L)
          : D->vs == LBF_D3Q19 ? launch_init<VS_D3Q19>(D->st, D->scalar, P, I, pb, L)
                               : launch_init<VS_D3Q27>(D->st, D->scalar, P, I, pb, L);
        I.skip_pops = 0;
    }
    if (e == cudaSuccess && D->sparse)
        e = D->vs == LBF_D2Q9 ? launch_init_sparse<VS_D2Q9>(D->st, P, I, s)
          : D->vs == LBF_D3Q19 ? launch_init_sparse<VS_D3Q19>(D->st, P, I, s)
                               : launch_init_sparse<VS_D3Q27>(D->st, P, I, s);
    else if (e == cudaSuccess)
        e = D->vs == LBF_D2Q9 ? launch_init<VS_D2Q9>(D->st, D->scalar, P, I, pb, L)
          : D->vs == LBF_D3Q19 ? launch_init<VS_D3Q19>(D->st, D->scalar, P, I, pb, L)
                               : launch_init<VS_D3Q27>(D->st, D->scalar, P, I, pb, L);
    if (tmp) {
        cudaStreamSynchronize(s);
        dev_free(tmp, D->dev);
    }
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("init kernel: ") + cudaGetErrorString(e));
    CK(cudaMemsetAsync(D->err, 0, sizeof(int), s));   // a re-initialised domain starts without an error
    D->t = 0;
    D->res_step = -1;
    D->initialized = true;
    D->last_stream = s;
    return LBF_OK;
}

// The outflow face pass of step t runs beside the sweep of step t + 1 over the
// planes below ZCUT = nz - 4 (on a side stream), when the only outflow face is
// the top face of a whole lattice in the sparse layout and the bottom and top
// faces are explicit for the momentum and every scalar.  With buffers X (read
// by step t) and Y (written):
//  - the face pass reads X at the top plane and the plane below it, the
//    snapshots of planes nz - 2 and nz - 3 and the top face's layers, and writes
//    Y at the top plane and those layers;
//  - the lower sweep of step t + 1 reads Y at planes <= nz - 4 (all written by
//    step t's bulk launch, which precedes it) and writes X at planes < nz - 4;
//  - the pulls that wrap in z (the top plane from plane 0, plane 0 from the top
//    plane) fetch populations that the explicit bottom and top face rules replace
//    before any use, so when those reads land relative to the other stream's
//    writes changes no result.
// The rest of step t + 1 (planes >= nz - 4) follows the face pass on the main
// stream, and step t + 2's lower sweep waits for both parts of step t + 1.
// Steps that compute residuals or write moments, and the first step, run in order.
constexpr long long OVL_CUT = 4;

bool face_overlap_ok(const lbf_domain* D) {
    if (!D->sparse || !(D->facebc || D->scalar) || z_restricted(D) || D->d != 3) return false;
    if (D->outflow != (1u << 5) || D->n[2] < 3 * OVL_CUT) return false;
    for (int f = 4; f < 6; ++f) {
        if (D->desc.bc[f].kind == LBF_BC_PERIODIC) return false;
        for (int si = 0; si < D->ns; ++si)
            if (D->sdesc[si].bc[f].kind == LBF_SBC_PERIODIC) return false;
    }
    return true;
}

lbf_status do_steps(lbf_domain* D, long long nsteps, long long k, cudaStream_t s) {
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called before stepping");
    if (D->part_pending) return fail(LBF_ESTATE, "a split step waits for its part 1");
    lbf_status st;
    if (k > 0 && (st = ensure_mom(D))) return st;
    const bool ovl = face_overlap_ok(D) && nsteps > 1;
    if (ovl && !D->side) {
        CK(cudaStreamCreateWithFlags(&D->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&D->ev_bulk, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&D->ev_head, cudaEventDisableTiming));
    }
    const long long kcut = ovl ? D->zoff[(size_t)(D->n[2] - OVL_CUT)] : 0;
    auto plain = [&](long long t) {   // a step that takes part in no overlap
        return t == 0 || (k > 0 && (t % k == 0 || (t + 1) % k == 0));
    };
    bool head_ran = false;   // the lower sweep of this step already ran on the side stream
    for (long long it = 0; it < nsteps; ++it) {
        const long long t = D->t;
        StepParams P;
        base_params(D, P, t);
        P.residual = (k > 0 && t % k == 0) ? 1 : 0;
        P.write_mom = (k > 0 && (t % k == 0 || (t + 1) % k == 0)) ? 1 : 0;
        D->slot_next = 0;
        cudaError_t e;
        if (ovl) {
            const bool next = it + 1 < nsteps && !plain(t) && !plain(t + 1);
            e = sparse_fs_bulk(D, P, head_ran ? kcut : P.kbeg, P.kend, s);
            if (head_ran && e == cudaSuccess) e = cudaStreamWaitEvent(s, D->ev_head, 0);
            if (next && e == cudaSuccess) e = cudaEventRecord(D->ev_bulk, s);
            // the face pass is submitted first, so that its single wave of blocks is
            // dispatched before the lower sweep's blocks take every SM
            if (e == cudaSuccess) e = sparse_fs_faces(D, P, s);
            if (next && e == cudaSuccess) {
                StepParams N1;
                base_params(D, N1, t + 1);
                e = cudaStreamWaitEvent(D->side, D->ev_bulk, 0);
                if (e == cudaSuccess) e = sparse_fs_bulk(D, N1, N1.kbeg, kcut, D->side);
                if (e == cudaSuccess) e = cudaEventRecord(D->ev_head, D->side);
            }
            head_ran = next;
        } else {
            e = launch_step_any(D, P, s);
        }
        if (e != cudaSuccess) {
            if (ovl) cudaStreamSynchronize(D->side);   // nothing of this domain stays in flight on it
            return fail(LBF_EDEVICE, std::string("step kernel: ") + cudaGetErrorString(e));
        }
        if (P.residual) {
            k_finalize<<<1, FINALIZE_THREADS, 0, s>>>(D->accum, D->accum_cap, D->slot_next, D->nacc(), 1, D->res_dev);
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
    if (D->part_pending) return fail(LBF_ESTATE, "a split step waits for its part 1");
    lbf_status st;
    if (!D->obs && (st = dmalloc(D, (void**)&D->obs, (size_t)D->N * obs_fields(D) * sizeof(double)))) return st;
    StepParams P;
    base_params(D, P, D->t);
    P.observe = 1;
    D->slot_next = 0;
    P.obs_rho = D->obs;
    P.obs_u = D->obs + D->N;
    P.obs_c = D->obs + D->N * (1 + D->d);
    cudaError_t e = launch_step_any(D, P, s);
    if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("observe kernel: ") + cudaGetErrorString(e));
    return LBF_OK;
}

// The sweep of planes [zlo, zhi) of step P (a z-slab's split step).
cudaError_t sweep_planes(lbf_domain* D, StepParams P, long long zlo, long long zhi, cudaStream_t s) {
    if (zlo >= zhi) return cudaSuccess;
    if (D->sparse) {
        P.kbeg = D->zoff[(size_t)zlo];
        P.kend = D->zoff[(size_t)zhi];
        return launch_sparse(D, P, s);
    }
    P.z0 = (int)zlo;
    const bool stage = D->stage && can_stage(D);
    const dim3 b = stage ? dim3((unsigned)D->n[0]) : step_block(D);
    const dim3 g((unsigned)((D->n[0] + b.x - 1) / b.x), (unsigned)D->n[1], (unsigned)(zhi - zlo));
    take_slots(D, P, (long long)g.x * g.y * g.z);
    return launch_one(D, P, stage, Launch{g, b, s});
}

void tables_c(int vs, int i, int* c) {
    for (int a = 0; a < 3; ++a)
        c[a] = vs == LBF_D2Q9 ? (a < 2 ? Lat<VS_D2Q9>::c(i, a) : 0)
             : vs == LBF_D3Q19 ? Lat<VS_D3Q19>::c(i, a) : Lat<VS_D3Q27>::c(i, a);
}

// Pack (unpack = false) the leaving directions of the owned boundary plane of
// `face` into buf, or unpack (true) buf into the entering directions of the
// ghost plane beyond it, in the state the next step reads (buffer t & 1).
lbf_status halo_copy(lbf_domain* D, int face, bool unpack, void* buf, cudaStream_t s) {
    if (!D || !buf) return fail(LBF_EINVAL, "null argument");
    if (D->d != 3) return fail(LBF_EINVAL, "halos apply to 3-D lattices");
    if (face != LBF_BOTTOM && face != LBF_TOP) return fail(LBF_EINVAL, "halo face must be LBF_BOTTOM or LBF_TOP");
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called first");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch");
    if (D->inplace || D->push) return fail(LBF_EUNSUPPORTED, "halos need the pull sweep (LBF_STREAM_PULL)");
    const long long z0 = zb(D), z1 = ze(D);
    if (z0 < 1 || z1 > D->n[2] - 1) return fail(LBF_EINVAL, "halos need a ghost plane below z_begin and above z_end - 1");
    // bottom: pack plane z0, c_z = -1; unpack ghost z0 - 1, c_z = +1
    // top:    pack plane z1 - 1, c_z = +1; unpack ghost z1, c_z = -1
    const bool bottom = face == LBF_BOTTOM;
    const int want = bottom ? (unpack ? +1 : -1) : (unpack ? -1 : +1);
    const long long z = bottom ? (unpack ? z0 - 1 : z0) : (unpack ? z1 : z1 - 1);
    const long long plane = D->n[0] * D->n[1];
    const size_t eb = st_bytes(D->st);
    // between the parts of a split step, the boundary planes of step t are in buffer (t + 1) & 1
    const long long tb = D->t + (D->part_pending ? 1 : 0);
    HaloPlanes H{};
    H.plane = plane;
    // slots of plane z: dense z * plane .. + plane; sparse its fluid nodes
    const long long first = D->sparse ? D->zoff[(size_t)z] : z * plane;
    H.count = D->sparse ? D->zoff[(size_t)z + 1] - D->zoff[(size_t)z] : plane;
    for (int i = 0; i < D->q; ++i) {
        int c[3];
        tables_c(D->vs, i, c);
        if (c[2] != want) continue;
        H.planes[H.nd++] = (char*)D->pop[tb & 1] + ((size_t)i * D->Np + (size_t)first) * eb;
    }
    const long long n = (long long)H.nd * H.count;
    if (n == 0) { D->last_stream = s; return LBF_OK; }
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 4 * 148);
    if (eb == 8) {
        if (unpack) k_halo_unpack<double><<<blocks, 256, 0, s>>>(H, (const double*)buf);
        else k_halo_pack<double><<<blocks, 256, 0, s>>>(H, (double*)buf);
    } else if (eb == 4) {
        if (unpack) k_halo_unpack<float><<<blocks, 256, 0, s>>>(H, (const float*)buf);
        else k_halo_pack<float><<<blocks, 256, 0, s>>>(H, (float*)buf);
    } else {
        if (unpack) k_halo_unpack<unsigned short><<<blocks, 256, 0, s>>>(H, (const unsigned short*)buf);
        else k_halo_pack<unsigned short><<<blocks, 256, 0, s>>>(H, (unsigned short*)buf);
    }
    CK(cudaGetLastError());
    D->last_stream = s;
    return LBF_OK;
}

// ---- checkpoints --------------------------------------------------------------
// The state a run carries from one step to the next: the post-collision
// populations (and scalar populations) the next step reads, the in-place scalar
// fields, the residual moments of the last residual steps, the face layers of the
// previous step, and the time step with the last residuals.
struct CkptHeader {
    char magic[8];        // "LBFCKPT1"
    int32_t vs, q, st, d;
    int64_t N, Np, nlist;
    int32_t sparse, scalar, ads, nsec;
    int64_t t, res_step;
    double res[8];
    int64_t sec_bytes[32];
};

struct Section {
    void* dev;
    size_t bytes;
};

// `t` selects the population buffers: the ones the step at time t reads.
// Sections: populations; per scalar (at least one triple, empty without
// scalars) its populations, adsorbed amount and previous value; the residual
// moments; the face layers.
std::vector<Section> ckpt_sections(const lbf_domain* D, long long t) {
    std::vector<Section> s;
    const size_t eb = st_bytes(D->st), rb = rt_bytes(D->st);
    s.push_back({D->pop[D->inplace ? 0 : (t & 1)], (size_t)D->q * D->Np * eb});
    for (int si = 0; si < std::max(D->ns, 1); ++si) {
        const bool has = si < D->ns;
        s.push_back({has ? D->gpop[si][t & 1] : nullptr, has ? (size_t)D->q * D->Np * rb : 0});
        s.push_back({D->qads[si], D->qads[si] ? (size_t)D->N * rb : 0});
        s.push_back({D->cprev[si], D->cprev[si] ? (size_t)D->N * rb : 0});
    }
    for (int k = 0; k < 2; ++k)
        s.push_back({D->mom[k], D->mom[k] ? (size_t)D->nfields() * D->N * rb : 0});
    for (int f = 0; f < 6; ++f)
        for (int k = 0; k < 2; ++k)
            s.push_back({D->pb[f][k], D->pb[f][k] ? (size_t)2 * D->pb_nf() * D->pb_plane[f] * rb : 0});
    return s;
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
    if (c.kind < LBF_BGK || c.kind > LBF_CENTRAL) return fail(LBF_EINVAL, "bad collision kind");
    if (c.kind == LBF_CENTRAL && !(c.tau > 0.0)) return fail(LBF_EINVAL, "central-moment tau must be > 0");
    if (c.kind == LBF_CENTRAL && vs == LBF_D3Q19)
        return fail(LBF_EUNSUPPORTED, "the central-moment collision needs a tensor-product set (D2Q9, D3Q27)");
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
    D->dev = current_device();
    D->desc = *ds;
    D->desc.node_type = nullptr;
    D->desc.initial_density_field = nullptr;
    D->desc.initial_velocity_field = nullptr;
    D->vs = vs; D->q = vs_q(vs); D->d = d; D->st = ds->storage; D->nfaces = nf;
    for (int a = 0; a < 3; ++a) D->n[a] = n[a];
    D->N = N;
    D->type.resize((size_t)N);
    if (ds->node_type) {
        // any non-zero value means solid: normalised to 1, in one pass
        const uint8_t* src = ds->node_type;
        uint8_t* dst = D->type.data();
        for (long long i = 0; i < N; ++i) dst[i] = src[i] != 0;
    } else {
        std::memset(D->type.data(), 0, (size_t)N);
    }
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
    // the population buffers are allocated once the layout is known (prepare)
    D->accum_cap = accum_slots(n, nf);
    if ((st = dmalloc(D, (void**)&D->accum, (size_t)ACCUM_PLANES * D->accum_cap * sizeof(double)))) { delete D; return st; }
    if ((st = dmalloc(D, (void**)&D->res_dev, 8 * sizeof(double)))) { delete D; return st; }
    if ((st = dmalloc(D, (void**)&D->err, sizeof(int)))) { delete D; return st; }
    if (cudaMemset(D->err, 0, sizeof(int)) != cudaSuccess) { delete D; return fail(LBF_EDEVICE, "memset"); }
    if (!(D->res_host = (double*)pinned64())) { delete D; return fail(LBF_ENOMEM, "pinned alloc"); }
    std::memset(D->res_host, 0, 8 * sizeof(double));
    if (cudaMemset(D->accum, 0, (size_t)ACCUM_PLANES * D->accum_cap * sizeof(double)) != cudaSuccess) {
        delete D;
        return fail(LBF_EDEVICE, "memset");
    }
    *out = D;
    return LBF_OK;
}

lbf_status lbf_scalar_attach(lbf_domain* D, const lbf_scalar_desc* s) {
    if (!D || !s) return fail(LBF_EINVAL, "null argument");
    if (D->ns >= NSMAX) return fail(LBF_EUNSUPPORTED, "at most LBF_MAX_SCALARS scalars per domain");
    if (D->initialized || D->prepared) return fail(LBF_ESTATE, "attach the scalars before lbf_domain_init");
    if (z_restricted(D)) return fail(LBF_EUNSUPPORTED, "z-slab domains with a scalar are not built");
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
    // the face pass serves the outflow faces of every scalar at once
    const unsigned all = outflow | D->outflow;
    for (int f = 0; f < D->nfaces; ++f)
        for (int g = 0; g < D->nfaces; ++g)
            if ((all >> f & 1u) && (all >> g & 1u) && f / 2 != g / 2)
                return fail(LBF_EUNSUPPORTED, "extrapolation outflow on two faces that share an edge is not built");
    const int si = D->ns;
    lbf_status st;
    const size_t rb = rt_bytes(D->st);
    // the scalar populations are allocated with the momentum ones, once the layout is known
    if (s->has_adsorption) {
        if ((st = dmalloc(D, &D->qads[si], D->N * rb))) return st;
        if ((st = dmalloc(D, &D->cprev[si], D->N * rb))) return st;
    }
    if (s->initial_scalar_field) {
        if ((st = dmalloc(D, (void**)&D->c_init_dev[si], D->N * sizeof(double)))) return st;
        CK(cudaMemcpy(D->c_init_dev[si], s->initial_scalar_field, D->N * sizeof(double), cudaMemcpyHostToDevice));
        D->c0[si].assign(s->initial_scalar_field, s->initial_scalar_field + D->N);
    }
    D->outflow = all;
    D->outflow_s[si] = outflow;
    D->sdesc[si] = *s;
    D->sdesc[si].initial_scalar_field = nullptr;
    D->ns = si + 1;
    D->scalar = true;
    return LBF_OK;
}

lbf_status lbf_domain_init(lbf_domain* D, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    return do_init(D, (cudaStream_t)stream);
}

lbf_status lbf_domain_step(lbf_domain* D, int64_t nsteps, int64_t residual_interval, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    if (nsteps < 0) return fail(LBF_EINVAL, "nsteps < 0");
    return do_steps(D, nsteps, residual_interval, (cudaStream_t)stream);
}

lbf_status lbf_domain_step_part(lbf_domain* D, int32_t part, int64_t k, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called before stepping");
    if (D->d != 3 || !z_restricted(D)) return fail(LBF_EINVAL, "split steps apply to z-slab domains");
    if (D->outflow) return fail(LBF_EUNSUPPORTED, "split steps with an outflow face pass are not built");
    if (part != 0 && part != 1) return fail(LBF_EINVAL, "part must be 0 or 1");
    if ((part == 1) != D->part_pending) return fail(LBF_ESTATE, part ? "part 1 before part 0" : "part 0 twice");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    if (k > 0 && (st = ensure_mom(D))) return st;
    const long long t = D->t, z0 = zb(D), z1 = ze(D);
    StepParams P;
    base_params(D, P, t);
    P.residual = (k > 0 && t % k == 0) ? 1 : 0;
    P.write_mom = (k > 0 && (t % k == 0 || (t + 1) % k == 0)) ? 1 : 0;
    cudaError_t e = cudaSuccess;
    if (part == 0) {
        D->slot_next = 0;   // the slots of both parts of the step
        e = sweep_planes(D, P, z0, z0 + 1, s);
        if (e == cudaSuccess && z1 - 1 > z0) e = sweep_planes(D, P, z1 - 1, z1, s);
        if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("step kernel: ") + cudaGetErrorString(e));
        D->part_pending = true;
    } else {
        e = sweep_planes(D, P, z0 + 1, z1 - 1, s);
        if (e != cudaSuccess) return fail(LBF_EDEVICE, std::string("step kernel: ") + cudaGetErrorString(e));
        if (P.residual) {
            k_finalize<<<1, FINALIZE_THREADS, 0, s>>>(D->accum, D->accum_cap, D->slot_next, D->nacc(), 1, D->res_dev);
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(D->res_host, D->res_dev, 8 * sizeof(double), cudaMemcpyDeviceToHost, s));
            D->res_step = t;
        }
        D->t = t + 1;
        D->part_pending = false;
    }
    D->last_stream = s;
    return LBF_OK;
}

lbf_status lbf_domain_run(lbf_domain* D, int64_t max_iterations, int64_t k, double tr, double tu, double tc,
                          int64_t* steps_done, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
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
            for (int si = 0; si < D->ns; ++si) conv = conv && D->res_host[4 + si] <= tc;
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
    for (int k = 0; k < 1 + D->d; ++k) out[k] = D->res_host[k];
    for (int si = 0; si < D->ns; ++si) out[1 + D->d + si] = D->res_host[4 + si];
    if (time_step) *time_step = D->res_step;
    return LBF_OK;
}

}  // extern "C"

namespace {
// Observed moments of f_t into D->obs; solid nodes keep their initial values
// (they are never updated), filled on the device when those are uniform.
// `uniform` tells whether the host still has to fill them.
lbf_status observe_filled(lbf_domain* D, cudaStream_t s, bool& uniform) {
    lbf_status st;
    if ((st = do_observe(D, s))) return st;
    const long long N = D->N;
    uniform = D->rho0.empty() && D->u0.empty();
    for (int si = 0; si < D->ns; ++si) uniform = uniform && D->c0[si].empty();
    if (uniform && D->n_fluid < (unsigned long long)N) {
        const unsigned nb = (unsigned)((N + 255) / 256);
        for (int si = 0; si < std::max(D->ns, 1); ++si) {
            // the first launch fills rho and u as well; the others are the same values again
            k_fill_solid<<<nb, 256, 0, s>>>(D->dtype, N, D->d, D->obs, D->obs + N,
                                            si < D->ns ? D->obs + N * (1 + D->d + si) : nullptr, D->rho0u, D->u0u[0],
                                            D->u0u[1], D->u0u[2], si < D->ns ? D->sdesc[si].initial_scalar_value : 0.0);
        }
        CK(cudaGetLastError());
    }
    return LBF_OK;
}

double scalar_init_at(const lbf_domain* D, int si, long long i) {
    return D->c0[si].empty() ? D->sdesc[si].initial_scalar_value : D->c0[si][(size_t)i];
}
}  // namespace

extern "C" {

lbf_status lbf_domain_get_moments(lbf_domain* D, double* rho, double* u, double* c, void* stream) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    bool uniform = true;
    if ((st = observe_filled(D, s, uniform))) return st;
    const long long N = D->N;
    if (rho) CK(download(rho, D->obs, N * 8, s));
    if (u) CK(download(u, D->obs + N, N * D->d * 8, s));
    if (c && D->scalar) CK(download(c, D->obs + N * (1 + D->d), N * 8, s));
    CK(cudaStreamSynchronize(s));
    if ((st = check_err(D))) return st;
    if (uniform) return LBF_OK;
    for (long long i = 0; i < N; ++i) {
        if (!D->type[i]) continue;
        if (rho) rho[i] = D->rho0.empty() ? D->rho0u : D->rho0[i];
        if (u) for (int a = 0; a < D->d; ++a) u[i * D->d + a] = D->u0.empty() ? D->u0u[a] : D->u0[i * D->d + a];
        if (c && D->scalar) c[i] = scalar_init_at(D, 0, i);
    }
    return LBF_OK;
}

lbf_status lbf_domain_get_scalar(lbf_domain* D, int32_t index, double* c, void* stream) {
    if (!D || !c) return fail(LBF_EINVAL, "null argument");
    if (index < 0 || index >= D->ns) return fail(LBF_EINVAL, "no scalar with that index");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    bool uniform = true;
    if ((st = observe_filled(D, s, uniform))) return st;
    const long long N = D->N;
    CK(download(c, D->obs + N * (1 + D->d + index), N * 8, s));
    CK(cudaStreamSynchronize(s));
    if ((st = check_err(D))) return st;
    if (!uniform)
        for (long long i = 0; i < N; ++i)
            if (D->type[i]) c[i] = scalar_init_at(D, index, i);
    return LBF_OK;
}

lbf_status lbf_domain_get_q_ads_at(lbf_domain* D, int32_t index, double* q) {
    if (!D || !q) return fail(LBF_EINVAL, "null argument");
    if (index < 0 || (index >= D->ns && !(index == 0 && D->ns == 0))) return fail(LBF_EINVAL, "no scalar with that index");
    CK(cudaStreamSynchronize(D->last_stream));
    void* qa = D->qads[index];
    if (!qa) {
        std::fill(q, q + D->N, 0.0);
        return LBF_OK;
    }
    if (D->st == LBF_STORE_F64) {
        CK(cudaMemcpy(q, qa, D->N * 8, cudaMemcpyDeviceToHost));
    } else {
        std::vector<float> tmp(D->N);
        CK(cudaMemcpy(tmp.data(), qa, D->N * 4, cudaMemcpyDeviceToHost));
        for (long long i = 0; i < D->N; ++i) q[i] = tmp[i];
    }
    return LBF_OK;
}

lbf_status lbf_domain_get_q_ads(lbf_domain* D, double* q) { return lbf_domain_get_q_ads_at(D, 0, q); }

lbf_status lbf_domain_inventory(lbf_domain* D, double* out, void* stream) {
    if (!D || !out) return fail(LBF_EINVAL, "null argument");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch (poll or evict it first)");
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    if ((st = do_observe(D, s))) return st;
    const long long N = D->N;
    const double* c = D->scalar ? D->obs + N * (1 + D->d) : nullptr;   // scalar 0
    const void* qa0 = D->qads[0];
    // the swept planes only (all of them unless the domain is a z-slab)
    const long long o = zb(D) * D->n[0] * D->n[1], M = (ze(D) - zb(D)) * D->n[0] * D->n[1];
    const unsigned nb = (unsigned)((M + 255) / 256);
    const double* rho = D->obs + o;
    const double* uu = D->obs + N + o * D->d;
    const double* cc = c ? c + o : nullptr;
    if (D->d == 2) {
        if (D->st == LBF_STORE_F64) k_inventory<2, double><<<nb, 256, 0, s>>>(D->mask + o, M, rho, uu, cc, qa0 ? (const double*)qa0 + o : nullptr, D->accum, D->accum_cap);
        else k_inventory<2, float><<<nb, 256, 0, s>>>(D->mask + o, M, rho, uu, cc, qa0 ? (const float*)qa0 + o : nullptr, D->accum, D->accum_cap);
    } else {
        if (D->st == LBF_STORE_F64) k_inventory<3, double><<<nb, 256, 0, s>>>(D->mask + o, M, rho, uu, cc, qa0 ? (const double*)qa0 + o : nullptr, D->accum, D->accum_cap);
        else k_inventory<3, float><<<nb, 256, 0, s>>>(D->mask + o, M, rho, uu, cc, qa0 ? (const float*)qa0 + o : nullptr, D->accum, D->accum_cap);
    }
    CK(cudaGetLastError());
    double* tmp = nullptr;
    CK(dev_alloc((void**)&tmp, 8 * sizeof(double), D->dev));
    k_finalize<<<1, FINALIZE_THREADS, 0, s>>>(D->accum, D->accum_cap, (long long)nb, 6, 0, tmp);
    double h[8];
    cudaError_t e = cudaMemcpyAsync(h, tmp, 8 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dev_free(tmp, D->dev);
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
        case LBF_OPT_SPARSE:
            if (D->prepared) return fail(LBF_ESTATE, "set LBF_OPT_SPARSE before lbf_domain_init");
            D->sparse_opt = value != 0 ? 1 : 0;
            return LBF_OK;
        case LBF_OPT_STREAMING:
            if (D->prepared) return fail(LBF_ESTATE, "set LBF_OPT_STREAMING before lbf_domain_init");
            if (value < -1 || value > LBF_STREAM_INPLACE) return fail(LBF_EINVAL, "streaming: -1, PULL, PUSH or INPLACE");
            D->stream_opt = (int)value;
            return LBF_OK;
        case LBF_OPT_SROUND:
            D->sround = value != 0 ? 1 : 0;
            return LBF_OK;
        case LBF_OPT_WAIT_LIMIT:
            if (value < -1) return fail(LBF_EINVAL, "wait limit: -1 (default) or a number of polls >= 0");
            D->wait_limit = value;
            return LBF_OK;
        case LBF_OPT_SEED_OFFSET:
            D->seed_offset = value;
            return LBF_OK;
        case LBF_OPT_Z_BEGIN:
        case LBF_OPT_Z_END:
            if (D->prepared) return fail(LBF_ESTATE, "set the swept z planes before lbf_domain_init");
            if (D->d != 3) return fail(LBF_EINVAL, "z planes apply to 3-D lattices");
            if (D->scalar) return fail(LBF_EUNSUPPORTED, "z-slab domains with a scalar are not built");
            if (value < 0 || value > D->n[2]) return fail(LBF_EINVAL, "z plane out of range");
            (option == LBF_OPT_Z_BEGIN ? D->z_begin : D->z_end) = value;
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
        case LBF_OPT_SPARSE: *value = D->sparse ? 1 : 0; return LBF_OK;
        case LBF_OPT_STREAMING:
            *value = D->inplace ? LBF_STREAM_INPLACE : (D->push ? LBF_STREAM_PUSH : LBF_STREAM_PULL);
            return LBF_OK;
        case LBF_OPT_SROUND: *value = D->sround; return LBF_OK;
        case LBF_OPT_WAIT_LIMIT: *value = D->wait_limit; return LBF_OK;
        case LBF_OPT_SEED_OFFSET: *value = D->seed_offset; return LBF_OK;
        case LBF_OPT_Z_BEGIN: *value = zb(D); return LBF_OK;
        case LBF_OPT_Z_END: *value = ze(D); return LBF_OK;
        default: return fail(LBF_EINVAL, "unknown option");
    }
}

lbf_status lbf_domain_destroy(lbf_domain* D) {
    if (D) {
        if (D->batch) lbf_batch_evict(D->batch, D);
        if (D->last_stream) cudaStreamSynchronize(D->last_stream);
        delete D;
    }
    return LBF_OK;
}

lbf_status lbf_domain_checkpoint_bytes(lbf_domain* D, int64_t* bytes) {
    if (!D || !bytes) return fail(LBF_EINVAL, "null argument");
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called first");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch");
    int64_t b = sizeof(CkptHeader);
    for (const Section& s : ckpt_sections(D, D->t)) b += (int64_t)s.bytes;
    *bytes = b;
    return LBF_OK;
}

lbf_status lbf_domain_save(lbf_domain* D, void* host, int64_t cap, void* stream) {
    int64_t need = 0;
    lbf_status st = lbf_domain_checkpoint_bytes(D, &need);
    if (st) return st;
    if (D->part_pending) return fail(LBF_ESTATE, "a split step waits for its part 1");
    if (!host || cap < need) return fail(LBF_EINVAL, "checkpoint buffer smaller than lbf_domain_checkpoint_bytes");
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaStreamSynchronize(D->last_stream));
    const std::vector<Section> secs = ckpt_sections(D, D->t);
    CkptHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, "LBFCKPT1", 8);
    h.vs = D->vs; h.q = D->q; h.st = D->st; h.d = D->d;
    h.N = D->N; h.Np = D->Np; h.nlist = D->sparse ? D->nlist : 0;
    h.sparse = D->sparse ? 1 : 0; h.scalar = D->ns; h.ads = ads_bits(D);
    h.nsec = (int32_t)secs.size();
    h.t = D->t; h.res_step = D->res_step;
    for (int i = 0; i < 8; ++i) h.res[i] = D->res_host[i];
    char* p = (char*)host;
    for (size_t i = 0; i < secs.size(); ++i) h.sec_bytes[i] = (int64_t)secs[i].bytes;
    std::memcpy(p, &h, sizeof(h));
    p += sizeof(h);
    for (const Section& sec : secs) {
        if (sec.bytes) CK(cudaMemcpyAsync(p, sec.dev, sec.bytes, cudaMemcpyDeviceToHost, s));
        p += sec.bytes;
    }
    CK(cudaStreamSynchronize(s));
    return LBF_OK;
}

lbf_status lbf_domain_load(lbf_domain* D, const void* host, int64_t bytes, void* stream) {
    if (!D || !host) return fail(LBF_EINVAL, "null argument");
    if (!D->initialized) return fail(LBF_ESTATE, "create and initialise the domain from the same descriptors first");
    if (D->batch) return fail(LBF_ESTATE, "the domain is in a batch");
    if (D->part_pending) return fail(LBF_ESTATE, "a split step waits for its part 1");
    if (bytes < (int64_t)sizeof(CkptHeader)) return fail(LBF_EINVAL, "not a checkpoint (too short)");
    CkptHeader h;
    std::memcpy(&h, host, sizeof(h));
    if (std::memcmp(h.magic, "LBFCKPT1", 8) != 0) return fail(LBF_EINVAL, "not a checkpoint (bad magic)");
    if (h.vs != D->vs || h.q != D->q || h.st != D->st || h.N != D->N || h.Np != D->Np ||
        h.sparse != (D->sparse ? 1 : 0) || (h.sparse && h.nlist != D->nlist) || h.scalar != D->ns ||
        h.ads != ads_bits(D))
        return fail(LBF_EINVAL, "checkpoint of a different lattice, storage, layout or scalar set-up");
    if (h.t < 0 || h.res_step < -1 || h.res_step > h.t) return fail(LBF_EINVAL, "checkpoint time step out of range");
    // everything is validated before the domain changes: a rejected checkpoint
    // leaves the time step, the residuals and every field as they were
    const bool need_mom = h.sec_bytes[4] != 0 || h.sec_bytes[5] != 0;
    std::vector<Section> secs = ckpt_sections(D, h.t);   // the buffers of the checkpoint's parity
    if (h.nsec != (int32_t)secs.size()) return fail(LBF_EINVAL, "checkpoint section count differs");
    int64_t total = sizeof(CkptHeader);
    for (size_t i = 0; i < secs.size(); ++i) {
        // the residual-moment buffers (sections 4, 5) are allocated on demand below
        const int64_t want = (i == 4 || i == 5) && !secs[i].dev
                                 ? (int64_t)D->nfields() * D->N * (int64_t)rt_bytes(D->st)
                                 : (int64_t)secs[i].bytes;
        if (h.sec_bytes[i] != want && h.sec_bytes[i] != 0) return fail(LBF_EINVAL, "checkpoint section sizes differ");
        if (h.sec_bytes[i] < 0) return fail(LBF_EINVAL, "checkpoint section sizes differ");
        total += h.sec_bytes[i];
    }
    if (bytes < total) return fail(LBF_EINVAL, "checkpoint truncated");
    lbf_status st;
    if (need_mom && (st = ensure_mom(D))) return st;
    secs = ckpt_sections(D, h.t);
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaStreamSynchronize(D->last_stream));
    const char* p = (const char*)host + sizeof(CkptHeader);
    for (size_t i = 0; i < secs.size(); ++i) {
        if (h.sec_bytes[i]) CK(cudaMemcpyAsync(secs[i].dev, p, (size_t)h.sec_bytes[i], cudaMemcpyHostToDevice, s));
        p += h.sec_bytes[i];
    }
    CK(cudaStreamSynchronize(s));
    D->t = h.t;
    D->res_step = h.res_step;
    for (int i = 0; i < 8; ++i) D->res_host[i] = h.res[i];
    D->last_stream = s;
    return LBF_OK;
}

lbf_status lbf_domain_halo_info(lbf_domain* D, int32_t* ndir, int64_t* plane_nodes, int64_t* bytes) {
    if (!D) return fail(LBF_EINVAL, "null domain");
    if (D->d != 3) return fail(LBF_EINVAL, "halos apply to 3-D lattices");
    int nd = 0;
    for (int i = 0; i < D->q; ++i) {
        int c[3];
        tables_c(D->vs, i, c);
        nd += c[2] < 0;
    }
    const long long plane = D->n[0] * D->n[1];
    if (ndir) *ndir = nd;
    if (plane_nodes) *plane_nodes = plane;
    if (bytes) *bytes = (int64_t)nd * plane * (int64_t)st_bytes(D->st);
    return LBF_OK;
}

lbf_status lbf_domain_halo_pack(lbf_domain* D, int32_t face, void* dst, void* stream) {
    return halo_copy(D, face, false, dst, (cudaStream_t)stream);
}

lbf_status lbf_domain_halo_unpack(lbf_domain* D, int32_t face, const void* src, void* stream) {
    return halo_copy(D, face, true, const_cast<void*>(src), (cudaStream_t)stream);
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

// ============================================================== batches
// A batch advances many initialised domains together: the domains of each kernel
// configuration (velocity set, collision, storage, explicit faces) form a group,
// and one launch per group and time step covers all of them (k_step_batch).  A
// chunk is k time steps (k = residual interval) followed by one finalize launch
// per group that evaluates each domain's residuals and stop rule on the device;
// the chunk is captured once as a CUDA graph and replayed until the membership
// changes.  Every domain joins in phase: its next time step t has
// t % k == 1 % k, so that the last step of every chunk is its residual step and
// it stops exactly where lbf_domain_run(max_iterations, k) would.
struct lbf_batch {
    struct Member {
        lbf_domain* D;
        long long max_it;
        double tol[3];
    };
    struct Group {
        int vs = 0, coll = 0, st = 0;
        bool facebc = false, sparse = false;
        bool solo = false;             // one large member launched with its own single-domain sweep
        std::vector<int> mem;          // indices into members
        void* tab = nullptr;           // KParams<vs>[n] (device)
        BatchState* bs = nullptr;      // device state
        BatchState* host = nullptr;    // pinned mirror, copied at the end of every chunk
        int* blk = nullptr;            // block -> position in the group
        unsigned nblocks = 0;
    };
    std::mutex mu;
    int k = 1;
    bool chunk_launch = false;         // a group's k steps in one cooperative launch (LBF_BATCH_OPT_CHUNK_LAUNCH)
    long long budget = 0, bytes = 0;
    std::vector<Member> members;
    std::vector<std::pair<lbf_domain*, int>> finished;   // (domain, status) not yet polled
    std::vector<std::pair<lbf_domain*, long long>> admitted;   // device bytes counted at admission
    std::vector<Group> groups;
    bool dirty = true;
    cudaStream_t cap = nullptr;        // private stream the chunk graph is captured on
    // the groups' step chains are captured on side streams forked from cap, so that
    // the chunk graph runs independent groups (and large members) concurrently
    static constexpr int NSIDE = 8;
    cudaStream_t side[NSIDE] = {};
    cudaEvent_t fork = nullptr, join[NSIDE] = {};
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev = nullptr;
    cudaStream_t last = nullptr;
    bool launched = false;
    int dev = 0;
    BatchState* host_buf = nullptr;   // pinned, grows only (no cudaFreeHost while serving)
    size_t host_cap = 0;

    void free_groups() {
        for (auto& g : groups) {
            dev_free(g.tab, dev); dev_free(g.bs, dev); dev_free(g.blk, dev);
        }
        groups.clear();
        if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    }
    ~lbf_batch() {
        if (launched) cudaEventSynchronize(ev);   // the null stream is a valid stream: sync on the event
        free_groups();
        if (host_buf) cudaFreeHost(host_buf);
        if (ev) cudaEventDestroy(ev);
        if (fork) cudaEventDestroy(fork);
        for (int q = 0; q < NSIDE; ++q) {
            if (join[q]) cudaEventDestroy(join[q]);
            if (side[q]) cudaStreamDestroy(side[q]);
        }
        if (cap) cudaStreamDestroy(cap);
    }
};

namespace {

// Releases the budget share of a domain that leaves the batch.
void batch_release(lbf_batch* b, lbf_domain* D) {
    for (size_t i = 0; i < b->admitted.size(); ++i)
        if (b->admitted[i].first == D) {
            b->bytes -= b->admitted[i].second;
            b->admitted.erase(b->admitted.begin() + i);
            break;
        }
    D->batch = nullptr;
}

size_t kparams_size(int vs) {
    return vs == LBF_D2Q9 ? sizeof(KParams<VS_D2Q9>)
         : vs == LBF_D3Q19 ? sizeof(KParams<VS_D3Q19>) : sizeof(KParams<VS_D3Q27>);
}

// The domain's step parameters laid out for an even time step (t = 0 layout).
void fill_kparams(const lbf_domain* D, unsigned char* dst, long long res_slots) {
    StepParams P;
    base_params(D, P, 0);
    P.first = 0;
    P.res_slots = res_slots;
    if (D->vs == LBF_D3Q27) {
        KParams<VS_D3Q27>* kp = new KParams<VS_D3Q27>();
        static_cast<StepParams&>(*kp) = P;
        fill_lam(*kp, D->lam.empty() ? nullptr : D->lam.data());
        std::memcpy(dst, kp, sizeof(*kp));
        delete kp;
    } else {
        std::memcpy(dst, &P, sizeof(StepParams));   // KParams<VS> adds nothing for D2Q9 / D3Q19
    }
}

// Reads the device state of every member (as of the last completed chunk) into
// the domains: time step, residuals; members that stopped move to `finished`.
void batch_harvest(lbf_batch* b) {
    std::vector<bool> gone(b->members.size(), false);
    for (auto& g : b->groups) {
        for (size_t p = 0; p < g.mem.size(); ++p) {
            const int mi = g.mem[p];
            if (mi < 0 || gone[mi]) continue;
            lbf_domain* D = b->members[mi].D;
            const BatchState& s = g.host[p];
            D->t = s.done_t >= 0 ? s.done_t + 1 : s.t0;
            if (s.res_t >= 0) {
                for (int i = 0; i < 8; ++i) D->res_host[i] = s.res[i];
                D->res_step = s.res_t;
            }
            D->last_stream = b->last;
            if (s.done_t >= 0) {
                b->finished.emplace_back(D, s.status);
                gone[mi] = true;
                g.mem[p] = -1;
            }
        }
    }
    std::vector<int> remap(b->members.size(), -1);
    std::vector<lbf_batch::Member> keep;
    for (size_t i = 0; i < b->members.size(); ++i) {
        if (gone[i]) continue;
        remap[i] = (int)keep.size();
        keep.push_back(b->members[i]);
    }
    if (keep.size() != b->members.size()) b->dirty = true;
    for (auto& g : b->groups)
        for (auto& m : g.mem) m = m >= 0 ? remap[m] : -1;
    b->members.swap(keep);
}

// Single steps (standalone path) until the domain's next step t has t % k == 1 % k.
// *stopped = the stop status if the rule of lbf_domain_run ended it meanwhile.
lbf_status phase_align(lbf_domain* D, const lbf_batch::Member& m, int k, cudaStream_t s, int* stopped) {
    *stopped = 0;
    while (D->t % k != 1 % k) {
        const long long t = D->t;
        lbf_status st = do_steps(D, 1, k, s);
        if (st) return st;
        if (t > m.max_it) { *stopped = 2; break; }
        if (t > 10 && D->res_step == t) {
            CK(cudaStreamSynchronize(s));
            if (!std::isfinite(D->res_host[0])) { *stopped = 3; break; }
            bool conv = D->res_host[0] <= m.tol[0];
            for (int a = 0; a < D->d; ++a) conv = conv && D->res_host[1 + a] <= m.tol[1];
            if (conv) { *stopped = 1; break; }
        }
    }
    return LBF_OK;
}

cudaError_t batch_launch_step(const lbf_batch::Group& g, int j, cudaStream_t s) {
    switch (g.vs) {
        case LBF_D2Q9:
            return launch_step_batch<VS_D2Q9>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, j, g.nblocks, s);
        case LBF_D3Q19:
            return launch_step_batch<VS_D3Q19>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, j, g.nblocks, s);
        default:
            return launch_step_batch<VS_D3Q27>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, j, g.nblocks, s);
    }
}
cudaError_t batch_launch_chunk(const lbf_batch::Group& g, int k, cudaStream_t s) {
    switch (g.vs) {
        case LBF_D2Q9:
            return launch_batch_chunk<VS_D2Q9>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, k, g.nblocks, s);
        case LBF_D3Q19:
            return launch_batch_chunk<VS_D3Q19>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, k, g.nblocks, s);
        default:
            return launch_batch_chunk<VS_D3Q27>(g.coll, g.st, g.facebc, g.sparse, g.tab, g.bs, g.blk, k, g.nblocks, s);
    }
}
cudaError_t batch_launch_finalize(const lbf_batch::Group& g, cudaStream_t s) {
    const int n = (int)g.mem.size();
    switch (g.vs) {
        case LBF_D2Q9: return launch_batch_finalize<VS_D2Q9>(g.tab, g.bs, n, s);
        case LBF_D3Q19: return launch_batch_finalize<VS_D3Q19>(g.tab, g.bs, n, s);
        default: return launch_batch_finalize<VS_D3Q27>(g.tab, g.bs, n, s);
    }
}

// New groups, device tables and chunk graph for the current members.
// Domains that the batched kernels do not cover (scalars, the central-moment
// collision, the sparse layout with explicit faces) run their own single-domain
// sweep inside the chunk graph, gated by their batch state like the large members.
bool solo_only(const lbf_domain* D) {
    return D->scalar || D->desc.collision.kind == LBF_CENTRAL || (D->sparse && D->facebc);
}

lbf_status batch_rebuild(lbf_batch* b, cudaStream_t s) {
    if (b->launched) CK(cudaEventSynchronize(b->ev));
    if (b->launched) batch_harvest(b);
    b->launched = false;
    b->free_groups();
    // phase alignment (may finish some members)
    std::vector<lbf_batch::Member> keep;
    for (auto& m : b->members) {
        int stopped = 0;
        lbf_status st = phase_align(m.D, m, b->k, s, &stopped);
        if (st) return st;
        if (stopped) b->finished.emplace_back(m.D, stopped);
        else keep.push_back(m);
    }
    b->members.swap(keep);
    CK(cudaStreamSynchronize(s));
    b->last = s;
    // groups by kernel configuration
    for (size_t i = 0; i < b->members.size(); ++i) {
        const lbf_domain* D = b->members[i].D;
        const int coll = D->desc.collision.kind;
        // a large member runs its own sweep in the graph; its launch parameters are
        // fixed per chunk step only when k is even (t0 keeps its parity)
        const long long units = D->sparse ? D->nlist : D->N;
        const bool solo = b->k % 2 == 0 && (units >= SOLO_UNITS || solo_only(D)) && !D->pipe && !D->stage;
        lbf_batch::Group* g = nullptr;
        for (auto& x : b->groups)
            if (!solo && !x.solo && x.vs == D->vs && x.coll == coll && x.st == D->st && x.facebc == D->facebc &&
                x.sparse == D->sparse)
                g = &x;
        if (!g) {
            b->groups.emplace_back();
            g = &b->groups.back();
            g->vs = D->vs; g->coll = coll; g->st = D->st; g->facebc = D->facebc; g->sparse = D->sparse;
            g->solo = solo;
        }
        g->mem.push_back((int)i);
    }
    size_t total = 0;
    for (auto& g : b->groups) total += g.mem.size();
    if (total > b->host_cap) {
        const size_t cap = std::max<size_t>(total, 2 * b->host_cap + 64);
        if (b->host_buf) cudaFreeHost(b->host_buf);
        b->host_buf = nullptr;
        b->host_cap = 0;
        CK(cudaMallocHost((void**)&b->host_buf, cap * sizeof(BatchState)));
        b->host_cap = cap;
    }
    size_t host_off = 0;
    for (auto& g : b->groups) {
        const size_t n = g.mem.size(), ks = kparams_size(g.vs);
        std::vector<unsigned char> tab(n * ks);
        std::vector<BatchState> bs(n);
        std::vector<int> blk;
        for (size_t p = 0; p < n; ++p) {
            const lbf_batch::Member& m = b->members[g.mem[p]];
            const lbf_domain* D = m.D;
            const long long units = D->sparse ? D->nlist : D->N;   // fluid nodes, or all nodes
            const long long nb = g.solo ? 0 : (units + BATCH_BLOCK - 1) / BATCH_BLOCK;
            fill_kparams(D, tab.data() + p * ks, g.solo ? residual_step_slots(D) : nb);
            BatchState& x = bs[p];
            std::memset(&x, 0, sizeof(x));
            x.t0 = D->t;
            x.last_t = m.max_it + 1;
            x.block0 = (long long)blk.size();
            x.done_t = -1;
            x.res_t = D->res_step;
            for (int i = 0; i < 8; ++i) x.res[i] = D->res_host[i];
            x.k = b->k;
            x.d = D->d;
            x.ns = D->ns;
            for (int i = 0; i < 3; ++i) x.tol[i] = m.tol[i];
            blk.insert(blk.end(), (size_t)nb, (int)p);
        }
        if (blk.size() >= (1ull << 31)) return fail(LBF_EUNSUPPORTED, "batch group larger than 2^31 blocks");
        g.nblocks = (unsigned)blk.size();
        CK(dev_alloc(&g.tab, tab.size(), b->dev));
        CK(dev_alloc((void**)&g.bs, n * sizeof(BatchState), b->dev));
        CK(dev_alloc((void**)&g.blk, blk.size() * sizeof(int), b->dev));
        g.host = b->host_buf + host_off;
        host_off += n;
        std::memcpy(g.host, bs.data(), n * sizeof(BatchState));
        CK(cudaMemcpy(g.tab, tab.data(), tab.size(), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(g.bs, bs.data(), n * sizeof(BatchState), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(g.blk, blk.data(), blk.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    // capture one chunk: k steps of every group, finalize, copy the states back.
    // Groups are independent: each group's chain runs on a side stream forked
    // from the capture stream.  The large members (solo groups), which fill the
    // GPU one at a time, share side stream 0 and keep running one after another;
    // the batched groups of small members take the other side streams in turn and
    // overlap with them.
    if (!b->members.empty()) {
        CK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        const int ns = (int)std::min<size_t>(lbf_batch::NSIDE, b->groups.size() + 1);
        cudaError_t e = cudaEventRecord(b->fork, b->cap);
        for (int q = 0; q < ns && e == cudaSuccess; ++q) e = cudaStreamWaitEvent(b->side[q], b->fork, 0);
        const int forked = e == cudaSuccess ? ns : 0;
        for (size_t gi = 0; gi < b->groups.size() && e == cudaSuccess; ++gi) {
            lbf_batch::Group& g = b->groups[gi];
            cudaStream_t sg = g.solo || ns == 1 ? b->side[0] : b->side[1 + gi % (size_t)(ns - 1)];
            if (!g.solo && b->chunk_launch && b->k > 1) {
                e = batch_launch_chunk(g, b->k, sg);   // the chunk's k steps in one launch
            }
            for (int j = 0; j < b->k && e == cudaSuccess && !(!g.solo && b->chunk_launch && b->k > 1); ++j) {
                if (!g.solo) {
                    e = batch_launch_step(g, j, sg);
                    continue;
                }
                lbf_domain* D = b->members[g.mem[0]].D;
                const long long t = D->t + j;
                StepParams P;
                base_params(D, P, t);
                P.residual = t % b->k == 0 ? 1 : 0;
                P.write_mom = (t % b->k == 0 || (t + 1) % b->k == 0) ? 1 : 0;
                P.gate = (const GateView*)g.bs;
                P.gate_j = j;
                D->slot_next = 0;   // the step's partial-sum slots start at 0
                e = launch_step_any(D, P, sg);
            }
            if (e == cudaSuccess) e = batch_launch_finalize(g, sg);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(g.host, g.bs, g.mem.size() * sizeof(BatchState), cudaMemcpyDeviceToHost, sg);
        }
        // every forked side stream rejoins the capture stream, also after an error
        for (int q = 0; q < forked; ++q) {
            cudaError_t r = cudaEventRecord(b->join[q], b->side[q]);
            if (r == cudaSuccess) r = cudaStreamWaitEvent(b->cap, b->join[q], 0);
            if (e == cudaSuccess) e = r;
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->cap, &graph);
        if (e == cudaSuccess) e = e2;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(LBF_EDEVICE, std::string("batch graph: ") + cudaGetErrorString(e));
        }
    }
    b->dirty = false;
    return LBF_OK;
}

long long estimate_bytes(const lbf_domain_desc* ds, const lbf_scalar_desc* sd) {
    const int vs = ds->velocity_set, q = vs_q(vs), d = vs_d(vs);
    const long long N = ds->n[0] * ds->n[1] * (d == 3 ? ds->n[2] : 1);
    const long long Np = (N + 63) / 64 * 64;
    const long long sb = (long long)st_bytes(ds->storage), rb = (long long)rt_bytes(ds->storage);
    const int nf = 1 + d + (sd ? 1 : 0);
    long long b = 2 * q * Np * sb;                       // populations A/B
    b += 4 * N + N + 8 * N;                              // mask, node types, set-up scratch
    b += 2 * nf * N * rb;                                // residual moments
    b += N * (d + 2) * 8;                                // observed moments (FP64)
    if (ds->storage == LBF_STORE_F64) b += 4 * N;        // work list of the compacted sweep
    if (sd) b += 2 * q * Np * rb + 3 * N * 8;            // scalar populations, q_ads, C_prev, C_init
    const long long plane = N / std::min({ds->n[0], ds->n[1], d == 3 ? ds->n[2] : ds->n[1]});
    b += 6 * 2 * 2 * (d + 1) * plane * rb;               // face layers (upper bound)
    if (sd) b += 6 * 2 * q * plane * rb;                 // outflow snapshots (upper bound)
    {
        const long long nn[3] = {ds->n[0], ds->n[1], d == 3 ? ds->n[2] : 1};
        b += ACCUM_PLANES * accum_slots(nn, d == 2 ? 4 : 6) * 8 + 4096;
    }
    return b;
}

}  // namespace

extern "C" {

lbf_status lbf_domain_estimate_bytes(const lbf_domain_desc* desc, const lbf_scalar_desc* scalar, int64_t* bytes) {
    if (!desc || !bytes) return fail(LBF_EINVAL, "null argument");
    if (vs_q(desc->velocity_set) == 0) return fail(LBF_EUNSUPPORTED, "velocity set not built on the device");
    for (int a = 0; a < 3; ++a)
        if (desc->n[a] < 1 && (a < vs_d(desc->velocity_set))) return fail(LBF_EINVAL, "lattice dimensions must be >= 1");
    *bytes = estimate_bytes(desc, scalar);
    return LBF_OK;
}

lbf_status lbf_batch_create(int64_t budget_bytes, int64_t residual_interval, lbf_batch** out) {
    if (!out) return fail(LBF_EINVAL, "null argument");
    *out = nullptr;
    if (residual_interval < 1 || residual_interval > 100000) return fail(LBF_EINVAL, "residual_interval must be in [1, 1e5]");
    if (budget_bytes < 0) return fail(LBF_EINVAL, "budget_bytes must be >= 0");
    lbf_batch* b = new lbf_batch();
    b->k = (int)residual_interval;
    b->dev = current_device();
    if (budget_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaError_t e = cudaMemGetInfo(&fr, &tot);
        if (e != cudaSuccess) { delete b; return fail(LBF_EDEVICE, std::string("cudaMemGetInfo: ") + cudaGetErrorString(e)); }
        budget_bytes = (int64_t)(0.9 * (double)fr);
    }
    b->budget = budget_bytes;
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    for (int q = 0; q < lbf_batch::NSIDE && e == cudaSuccess; ++q) {
        e = cudaStreamCreateWithFlags(&b->side[q], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[q], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) { delete b; return fail(LBF_EDEVICE, std::string("batch: ") + cudaGetErrorString(e)); }
    *out = b;
    return LBF_OK;
}

lbf_status lbf_batch_admit(lbf_batch* b, lbf_domain* D, int64_t max_iterations, double tol_density,
                           double tol_velocity, double tol_scalar) {
    if (!b || !D) return fail(LBF_EINVAL, "null argument");
    std::lock_guard<std::mutex> lock(b->mu);
    if (D->batch) return fail(LBF_ESTATE, "the domain is already in a batch");
    if (!D->initialized) return fail(LBF_ESTATE, "lbf_domain_init must be called before lbf_batch_admit");
    if (solo_only(D) && b->k % 2)
        return fail(LBF_EUNSUPPORTED, "a domain with scalars, the central-moment collision or the sparse layout with "
                                      "explicit faces is batched with an even residual interval only (it runs its own "
                                      "sweep in the chunk graph)");
    if (solo_only(D) && (D->pipe || D->stage))
        return fail(LBF_EUNSUPPORTED, "a domain that runs its own sweep in a batch takes neither the pipelined nor "
                                      "the staged sweep");
    if (z_restricted(D)) return fail(LBF_EUNSUPPORTED, "z-slab domains are not batched");
    if (max_iterations < 0) return fail(LBF_EINVAL, "max_iterations must be >= 0");
    lbf_status st;
    if ((st = ensure_mom(D))) return st;
    if (b->bytes + D->bytes > b->budget)
        return fail(LBF_ENOMEM, "batch memory budget exceeded (" + std::to_string(b->bytes + D->bytes) + " > " +
                                    std::to_string(b->budget) + " bytes)");
    if (D->last_stream) CK(cudaStreamSynchronize(D->last_stream));
    b->members.push_back({D, max_iterations, {tol_density, tol_velocity, tol_scalar}});
    D->batch = b;
    b->bytes += D->bytes;
    b->admitted.emplace_back(D, D->bytes);
    b->dirty = true;
    return LBF_OK;
}

lbf_status lbf_batch_step(lbf_batch* b, int64_t nchunks, void* stream) {
    if (!b) return fail(LBF_EINVAL, "null batch");
    if (nchunks < 0) return fail(LBF_EINVAL, "nchunks < 0");
    std::lock_guard<std::mutex> lock(b->mu);
    cudaStream_t s = (cudaStream_t)stream;
    lbf_status st;
    if (b->dirty && (st = batch_rebuild(b, s))) return st;
    if (b->members.empty() || nchunks == 0) return LBF_OK;
    for (int64_t c = 0; c < nchunks; ++c) CK(cudaGraphLaunch(b->exec, s));
    CK(cudaEventRecord(b->ev, s));
    b->last = s;
    b->launched = true;
    return LBF_OK;
}

lbf_status lbf_batch_poll(lbf_batch* b, lbf_domain** done, int32_t* status, int32_t cap, int32_t* ndone,
                          int32_t wait) {
    if (!b || !ndone || (cap > 0 && !done)) return fail(LBF_EINVAL, "null argument");
    std::lock_guard<std::mutex> lock(b->mu);
    *ndone = 0;
    if (b->launched) {
        if (wait) {
            CK(cudaEventSynchronize(b->ev));
        } else {
            const cudaError_t q = cudaEventQuery(b->ev);
            if (q == cudaErrorNotReady) return LBF_OK;
            if (q != cudaSuccess) return fail(LBF_EDEVICE, std::string("batch: ") + cudaGetErrorString(q));
        }
        batch_harvest(b);
    }
    int32_t n = 0;
    while (n < cap && !b->finished.empty()) {
        auto [D, code] = b->finished.front();
        b->finished.erase(b->finished.begin());
        batch_release(b, D);
        done[n] = D;
        if (status) status[n] = code;
        ++n;
    }
    *ndone = n;
    return LBF_OK;
}

lbf_status lbf_batch_evict(lbf_batch* b, lbf_domain* D) {
    if (!b || !D) return fail(LBF_EINVAL, "null argument");
    std::lock_guard<std::mutex> lock(b->mu);
    if (D->batch != b) return fail(LBF_EINVAL, "the domain is not in this batch");
    if (b->launched) CK(cudaEventSynchronize(b->ev));
    if (b->launched) batch_harvest(b);
    for (size_t i = 0; i < b->finished.size(); ++i)
        if (b->finished[i].first == D) { b->finished.erase(b->finished.begin() + i); break; }
    for (size_t i = 0; i < b->members.size(); ++i)
        if (b->members[i].D == D) {
            b->members.erase(b->members.begin() + i);
            for (auto& g : b->groups)
                for (auto& m : g.mem) m = m == (int)i ? -1 : (m > (int)i ? m - 1 : m);
            b->dirty = true;
            break;
        }
    batch_release(b, D);
    return LBF_OK;
}

lbf_status lbf_batch_info(lbf_batch* b, int64_t* running, int64_t* finished, int64_t* bytes, int64_t* budget) {
    if (!b) return fail(LBF_EINVAL, "null batch");
    std::lock_guard<std::mutex> lock(b->mu);
    if (running) *running = (int64_t)b->members.size();
    if (finished) *finished = (int64_t)b->finished.size();
    if (bytes) *bytes = b->bytes;
    if (budget) *budget = b->budget;
    return LBF_OK;
}

lbf_status lbf_batch_set_option(lbf_batch* b, int32_t option, int64_t value) {
    if (!b) return fail(LBF_EINVAL, "null batch");
    std::lock_guard<std::mutex> lock(b->mu);
    switch (option) {
        case LBF_BATCH_OPT_CHUNK_LAUNCH:
            if (b->chunk_launch != (value != 0)) b->dirty = true;   // the chunk graph is captured again
            b->chunk_launch = value != 0;
            return LBF_OK;
        default:
            return fail(LBF_EINVAL, "unknown batch option");
    }
}

lbf_status lbf_batch_destroy(lbf_batch* b) {
    if (!b) return LBF_OK;
    {
        std::lock_guard<std::mutex> lock(b->mu);
        if (b->launched) cudaEventSynchronize(b->ev);
        for (auto& m : b->members) m.D->batch = nullptr;
        for (auto& f : b->finished) f.first->batch = nullptr;
    }
    delete b;
    return LBF_OK;
}

}  // extern "C"
