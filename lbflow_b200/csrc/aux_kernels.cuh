// aux_kernels.cuh -- node classification, initialisation and FP64 reductions.
#pragma once

#include "kernels.cuh"

namespace lbf {

struct SetupParams {
    int nx, ny, nz, pad;
    long long N;
    const uint8_t* type;      // 0 fluid, 1 solid
    uint32_t* cls;            // LBF_CLASS_* bits
    uint32_t* links;          // bit i: neighbour along c_i is solid
    uint32_t* mask;           // kernel mask word (M_* bits)
    unsigned fold_faces;      // faces whose no-slip walls fold into the link bits
    unsigned explicit_faces;  // faces whose BCs run explicitly (M_FACE)
    unsigned skip_faces;      // faces updated by the face pass (M_SKIP)
    unsigned pad2;
    unsigned long long* counts;   // [0] fluid nodes, [1] bounce-back nodes
};

// Lattice::new node classification (src/momentum/lattice.rs:156-191): fluid
// nodes, face membership of fluid nodes, and bounce-back nodes with the
// directions whose (periodic) neighbour is solid.
template <int VS>
__global__ void k_setup(const SetupParams S) {
    using L = Lat<VS>;
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= S.N) return;
    const int x = (int)(cell % S.nx);
    const int y = (int)((cell / S.nx) % S.ny);
    const int z = (int)(cell / ((long long)S.nx * S.ny));
    if (S.type[cell]) {
        S.cls[cell] = 1u;
        S.links[cell] = 0u;
        S.mask[cell] = M_SOLID;
        return;
    }
    uint32_t links = 0u;
    sfor<L::Q>([&](auto I) {
        constexpr int i = I;
        int xx = x + L::c(i, 0), yy = y + L::c(i, 1), zz = z + (L::D == 3 ? L::c(i, 2) : 0);
        xx = xx < 0 ? xx + S.nx : (xx >= S.nx ? xx - S.nx : xx);
        yy = yy < 0 ? yy + S.ny : (yy >= S.ny ? yy - S.ny : yy);
        zz = zz < 0 ? zz + S.nz : (zz >= S.nz ? zz - S.nz : zz);
        const long long n = (long long)xx + (long long)S.nx * ((long long)yy + (long long)S.ny * zz);
        if (S.type[n]) links |= 1u << i;
    });
    uint32_t cls = links ? 2u : 0u;
    uint32_t mask = links | (links ? M_BB : 0u);
    const int on[6] = {x == 0, x == S.nx - 1, y == 0, y == S.ny - 1, z == 0, z == S.nz - 1};
    sfor<L::NF>([&](auto FF) {
        constexpr int F = FF;
        if (on[F]) {
            cls |= 1u << (2 + F);
            if (S.fold_faces >> F & 1u) {
                sfor<L::Q>([&](auto I) {
                    if constexpr (leaves<L>(I, F)) mask |= 1u << int(I);
                });
            }
            if (S.explicit_faces >> F & 1u) mask |= M_FACE;
            if (S.skip_faces >> F & 1u) mask |= M_SKIP;
        }
    });
    const int dist[6] = {x, S.nx - 1 - x, y, S.ny - 1 - y, z, S.nz - 1 - z};
    for (int F = 0; F < L::NF; ++F)
        if ((S.skip_faces >> F & 1u) && (dist[F] == 1 || dist[F] == 2)) mask |= M_NEAR;
    S.cls[cell] = cls;
    S.links[cell] = links;
    S.mask[cell] = mask;
    atomicAdd(&S.counts[0], 1ull);
    if (links) atomicAdd(&S.counts[1], 1ull);
}

struct InitParams {
    double rho0, u0[3];
    double c0[NSMAX], q0[NSMAX];       // per scalar: uniform initial value and adsorbed amount
    const double* rho_field;           // or null
    const double* u_field;             // [N][D] or null
    const double* c_field[NSMAX];      // per scalar, or null
    int skip_pops;             // k_init: leave the populations (the sparse layout sets them by fluid slot)
    int pad;
};

// Lattice::initialize_nodes (src/momentum/lattice.rs:322-328,
// src/passive_scalar/lattice.rs:241-246): f = f_eq(rho0, u0), g = g_eq(C0, u0)
// on fluid nodes, evaluated in FP64 and stored in the storage format.  Also
// seeds the residual "previous" moments with the initial values (the
// ShallowNode of src/momentum/node.rs:93-111) and both parities of the
// face-layer buffers.
template <int VS, int ST, bool SCALAR>
__global__ void k_init(const StepParams P, const InitParams I0, void* pb0_0, void* pb0_1, void* pb1_0, void* pb1_1,
                       void* pb2_0, void* pb2_1, void* pb3_0, void* pb3_1, void* pb4_0, void* pb4_1, void* pb5_0,
                       void* pb5_1) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q, D = L::D;
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= P.N) return;
    Geo g;
    g.x = (int)(cell % P.nx);
    g.y = (int)((cell / P.nx) % P.ny);
    g.z = (int)(cell / ((long long)P.nx * P.ny));
    g.cell = cell;
    g.slot = cell;
    const double rho = I0.rho_field ? I0.rho_field[cell] : I0.rho0;
    double u[3] = {I0.u0[0], I0.u0[1], I0.u0[2]};
    if (I0.u_field)
        for (int a = 0; a < D; ++a) u[a] = I0.u_field[cell * D + a];
    const uint32_t mk = P.mask[cell];
    const bool fluid = !(mk & M_SOLID);
    double uu = 0.0;
    for (int a = 0; a < D; ++a) uu += u[a] * u[a];
    if (fluid && !I0.skip_pops) {
        sfor<Q>([&](auto Ii) {
            constexpr int i = Ii;
            // FP32-compute formats store h = f_eq - w (evaluated in FP64)
            const double fe = S::DEV ? heq_i<L, double>(i, rho, rho - 1.0, u, uu) : feq_i<L, double>(i, rho, u, uu);
            S::st(const_cast<void*>(P.srcp[i]), cell, S::sc(R(fe)));
        });
    }
    if (fluid && P.mom_prev) {
        R* mp = (R*)P.mom_prev;
        mp[cell] = R(rho);
        for (int a = 0; a < D; ++a) mp[(1 + a) * P.N + cell] = R(u[a]);
    }
    if constexpr (SCALAR) {
        for (int si = 0; si < P.nscalar; ++si) {
            const ScalarParams& sc = P.sc[si];
            const double c0 = I0.c_field[si] ? I0.c_field[si][cell] : I0.c0[si];
            if (fluid && !I0.skip_pops) {
                sfor<Q>([&](auto Ii) {
                    constexpr int i = Ii;
                    ((R*)sc.gsrc)[i * P.np + cell] = R(feq_i<L, double>(i, c0, u, uu));
                });
            }
            // every node, solid ones included: device memory comes uninitialised from the pool
            if (sc.qads) ((R*)sc.qads)[cell] = (fluid && (mk & M_BB)) ? R(I0.q0[si]) : R(0);
            if (sc.cprev) ((R*)sc.cprev)[cell] = R(c0);
            if (fluid && P.mom_prev) ((R*)P.mom_prev)[(1 + D + si) * P.N + cell] = R(c0);
        }
    }
    void* pbs[6][2] = {{pb0_0, pb0_1}, {pb1_0, pb1_1}, {pb2_0, pb2_1}, {pb3_0, pb3_1}, {pb4_0, pb4_1}, {pb5_0, pb5_1}};
    for (int F = 0; F < L::NF; ++F) {
        if (!pbs[F][0]) continue;
        const int dist = face_dist(g, F, P);
        if (dist > 1) continue;
        const long long pl = P.pb_plane[F], pos = face_pos(g, F, P);
        for (int par = 0; par < 2; ++par) {
            R* pb = (R*)pbs[F][par];
            for (int a = 0; a < D; ++a) pb[(dist * P.pb_nf + a) * pl + pos] = R(u[a]);
            for (int si = 0; si < P.pb_nf - D; ++si) {
                const double c0 = si < P.nscalar && I0.c_field[si] ? I0.c_field[si][cell]
                                                                    : (si < P.nscalar ? I0.c0[si] : 0.0);
                pb[(dist * P.pb_nf + D + si) * pl + pos] = R(c0);
            }
        }
    }
}

// initialize_nodes for the sparse (fluid-only) layout: fluid node k (cell
// list[k]) gets f = f_eq(rho0, u0) at population index k; the residual moments
// stay indexed by cell.
template <int VS, int ST>
__global__ void k_init_sparse(const StepParams P, const InitParams I0) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q, D = L::D;
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= P.nlist) return;
    const uint32_t e = P.list[k];
    const long long cell = P.packed ? (long long)(e & 2047u) +
                                          (long long)P.nx * ((long long)((e >> 11) & 2047u) + (long long)P.ny * (e >> 22))
                                    : (long long)e;
    const double rho = I0.rho_field ? I0.rho_field[cell] : I0.rho0;
    double u[3] = {I0.u0[0], I0.u0[1], I0.u0[2]};
    if (I0.u_field)
        for (int a = 0; a < D; ++a) u[a] = I0.u_field[cell * D + a];
    double uu = 0.0;
    for (int a = 0; a < D; ++a) uu += u[a] * u[a];
    sfor<Q>([&](auto Ii) {
        constexpr int i = Ii;
        const double fe = S::DEV ? heq_i<L, double>(i, rho, rho - 1.0, u, uu) : feq_i<L, double>(i, rho, u, uu);
        S::st(const_cast<void*>(P.srcp[i]), (int)k, S::sc(R(fe)));
    });
    for (int si = 0; si < P.nscalar; ++si) {   // g = g_eq(C0, u0) at the same slot (FP64 / FP32 storage only)
        const double c0 = I0.c_field[si] ? I0.c_field[si][cell] : I0.c0[si];
        sfor<Q>([&](auto Ii) {
            constexpr int i = Ii;
            ((R*)P.sc[si].gsrc)[i * P.np + k] = R(feq_i<L, double>(i, c0, u, uu));
        });
    }
    if (P.mom_prev) {
        R* mp = (R*)P.mom_prev;
        mp[cell] = R(rho);
        for (int a = 0; a < D; ++a) mp[(1 + a) * P.N + cell] = R(u[a]);
    }
}

// ---- set-up of the sparse layout --------------------------------------------------
// flag[cell] = fluid, val[cell] = cell (input of the fluid-list selection)
static __global__ void k_fluid_flags(const uint32_t* mask, long long N, uint8_t* flag, uint32_t* val) {
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= N) return;
    flag[c] = (mask[c] & M_SOLID) ? 0 : 1;
    val[c] = (uint32_t)c;
}
// fluid bits of word w of each row (rows = ny * nz, W words of 32 x each) and their counts
static __global__ void k_row_bits(const uint32_t* mask, int nx, long long nrows, int W, uint32_t* bits,
                                  uint32_t* cnt) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j >= nrows * W) return;
    const long long row = j / W;
    const int w = (int)(j - row * W);
    uint32_t b = 0;
    for (int t = 0; t < 32; ++t) {
        const int x = 32 * w + t;
        if (x < nx && !(mask[row * nx + x] & M_SOLID)) b |= 1u << t;
    }
    bits[j] = b;
    cnt[j] = __popc(b);
}
// row words {bits, first fluid index at or after the word}, then a sentinel row
static __global__ void k_row_words(const uint32_t* bits, const uint32_t* off, long long n, int W, uint32_t total,
                                   uint2* rw) {
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (j < n) rw[j] = make_uint2(bits[j], off[j]);
    else if (j < n + W) rw[j] = make_uint2(0u, total);
}
static __global__ void k_gather_mask(const uint32_t* mask, const uint32_t* list, long long n, uint32_t* out) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k < n) out[k] = mask[list[k]];
}
// node index -> x | y << 11 | z << 22 (lattices up to 2048 x 2048 x 1024)
static __global__ void k_pack_xyz(uint32_t* list, long long n, int nx, int ny) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t c = list[k];
    const uint32_t x = c % (uint32_t)nx, r = c / (uint32_t)nx;
    const uint32_t y = r % (uint32_t)ny, z = r / (uint32_t)ny;
    list[k] = x | (y << 11) | (z << 22);
}

// Solid nodes are never updated: their observed moments are the uniform initial
// values (the observe pass writes the fluid nodes only).
static __global__ void k_fill_solid(const uint8_t* type, long long N, int d, double* rho, double* u, double* c,
                                    double rho0, double u0x, double u0y, double u0z, double c0) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= N || !type[i]) return;
    rho[i] = rho0;
    u[i * d] = u0x;
    u[i * d + 1] = u0y;
    if (d == 3) u[i * d + 2] = u0z;
    if (c) c[i] = c0;
}

// Sum the per-block partials (slots [0, nslots) of each of nacc accumulators,
// accum[k * stride + slot]) in a fixed order: thread t adds slots t, t + T, ...
// in turn, then a fixed tree adds the threads' sums.  out[k] = sqrt(sum) for
// residuals, the plain sum for inventories.  One block of FINALIZE_THREADS.
constexpr int FINALIZE_THREADS = 512;
static __global__ void k_finalize(const double* accum, long long stride, long long nslots, int nacc, int take_sqrt,
                                  double* out) {
    __shared__ double part[FINALIZE_THREADS];
    for (int k = 0; k < nacc; ++k) {
        double s = 0.0;
        for (long long j = threadIdx.x; j < nslots; j += FINALIZE_THREADS) s += accum[k * stride + j];
        part[threadIdx.x] = s;
        __syncthreads();
        for (int o = FINALIZE_THREADS / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[k] = take_sqrt ? sqrt(part[0]) : part[0];
        __syncthreads();
    }
}

// FP64 inventories over fluid nodes from observed moments:
// [sum rho, sum rho*u_a (D), sum C, sum q_ads].
template <int D, class R>
__global__ void k_inventory(const uint32_t* mask, long long N, const double* rho, const double* u, const double* c,
                            const R* qads, double* accum, long long stride) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double vq = 0.0;
    if (cell < N && !(mask[cell] & M_SOLID)) {
        v[0] = rho[cell];
        for (int a = 0; a < D; ++a) v[1 + a] = rho[cell] * u[cell * D + a];
        if (c) v[1 + D] = c[cell];
        if (qads) vq = double(qads[cell]);
    }
    if (D == 2) v[4] = vq;   // slots: rho, j0, j1, C, q   (2-D)
    double w[6] = {v[0], v[1], v[2], v[3], v[4], D == 3 ? vq : 0.0};
    block_partials<6>(w, accum, stride, blockIdx.x);
}

}  // namespace lbf
