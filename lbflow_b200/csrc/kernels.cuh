// kernels.cuh -- the fused lattice Boltzmann step for sm_100a.
//
// One kernel advances every fluid node by one reference `main_steps`
// (src/momentum/lattice.rs:431-441; src/passive_scalar/lattice.rs:342-350):
//
//   pull-stream + inner bounce-back + face BCs  ->  f_t        (read Q values)
//   moments (rho, u with the F/2 shift)         ->  rho_t, u_t
//   equilibrium + BGK/TRT/MRT (+ Guo source)    ->  f*_t       (write Q values)
//   [passive scalar: the same on g, Langmuir adsorption, with u_t]
//
// State between launches is the post-collision field f*_{t-1} in SoA planes
// (plane i holds direction i for all nodes, node index x + nx*(y + ny*z)).  The
// step for time t pulls f_t(x)[i] = f*_{t-1}(x - c_i)[i] with periodic wrap
// (src/lib.rs:141-152, src/momentum/lattice.rs:127-154), replaces the directions
// whose neighbour is solid by the node's own reflected value (src/lib.rs:154-165),
// applies the face BCs in order (src/momentum/bc.rs:29-149), and only then
// collides.  Two population buffers alternate (A/B): each node's Q values are
// read once and written once per step, and the boundary rules keep the exact
// reference semantics: wall rules, periodic wrap and asymmetric periodic/wall
// pairs act on the same post-stream populations as in the reference.
//
// The step at t = 0 reads f_0 = f_eq(rho0, u0) from the node itself
// (Lattice::initialize_nodes, src/momentum/lattice.rs:322-328).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lattice.cuh"

namespace lbf {

constexpr int COLL_BGK = 0, COLL_TRT = 1, COLL_MRT = 2, COLL_CENTRAL = 3;
constexpr int ST_F64 = 0, ST_F32 = 1, ST_F16 = 2, ST_BF16 = 3;
constexpr int COMPAT_REFERENCE = 0, COMPAT_PHYSICS = 1;

// Per-node mask word.  Bits 0..26: the neighbour along c_i is solid (or, on the
// lean path, a no-slip wall); bit 27 solid node; bit 28 bounce-back node (has a
// solid neighbour, drives adsorption); bit 29 node needs explicit face BCs;
// bit 30 node is updated by the face pass, not by the bulk sweep; bit 31 node
// lies one or two layers inside a scalar extrapolation-outflow face (its
// post-stream scalar populations are snapshotted for that face).
constexpr uint32_t M_LINKS = (1u << 27) - 1u;
constexpr uint32_t M_SOLID = 1u << 27;
constexpr uint32_t M_BB = 1u << 28;
constexpr uint32_t M_FACE = 1u << 29;
constexpr uint32_t M_SKIP = 1u << 30;
constexpr uint32_t M_NEAR = 1u << 31;   // 1 or 2 layers inside a scalar outflow face

constexpr int NSLOT = 256;   // partial-sum slots of the FP64 reductions
constexpr int NACC = 8;      // accumulators per slot

// Boundary-condition kinds: the C-ABI values (include/lbflow.h).
enum { BC_NO_SLIP = 0, BC_BOUNCE_BACK = 1, BC_ANTI_BB = 2, BC_ZOU_HE = 3, BC_PERIODIC = 4 };
enum { SBC_ANTI_BB = 0, SBC_ANTI_BB_NO_FLUX = 1, SBC_BB_NO_FLUX = 2, SBC_ZEROTH = 3, SBC_SECOND = 4,
       SBC_PERIODIC = 5 };

struct FaceBC {
    int kind, has_rho;
    int has_u[3];
    int pad;
    double rho;
    double u[3];
};
struct SFaceBC {
    int kind, unknown_only;
    int given_vel;   // 1: wall velocity from the momentum BC of the face; 0: extrapolate
    int pad;
    double value;
    double u[3];
};

// Passive scalars per domain.  They share the momentum lattice (one momentum
// sweep advances all of them, passive_scalar::LatticeVec) and nothing else.
constexpr int NSMAX = 4;

// One passive scalar (same velocity set as the momentum lattice).
struct ScalarParams {
    int coll, inner, has_source, ads;
    double tau, omega, op, om, source;
    double bgk_cb;           // 1 - 1/(2 tau) of the BGK source, computed once
    double ka, kd, qmax;
    double c_solid;          // initial scalar of solid nodes when uniform
    const double* c_init;    // per-node initial scalar, or null
    const void* gsrc;        // plane 0 of g*_{t-1} (g_0 when first); plane i at + i * np elements
    void* gdst;              // plane 0 of g*_t
    void* qads;              // adsorbed amount per node (compute type), in place
    void* cprev;             // scalar value of the previous step per node, in place
    // post-stream scalar populations of layers 1 and 2 inside each outflow face,
    // written by the bulk sweep and read by the face pass of the same step:
    // [layer 0/1][direction][plane node], compute type
    void* snap[6];
    SFaceBC face[6];
};

// The leading fields of a batch member's device state (BatchState): a single-
// domain sweep launched inside a batch's chunk graph skips its launch when the
// domain has stopped or the step (t0 + gate_j) is past its last one.
struct GateView {
    long long t0, last_t, block0, done_t;
};

struct StepParams {
    int nx, ny, nz, dims;
    long long N;
    const uint32_t* mask;
    const void* srcp[27];   // plane pointers of f*_{t-1} (or f_0 when first)
    void* dstp[27];         // plane pointers of f*_t
    int coll, compat, has_force, first;
    double tau, omega, op, om;
    double rates[27];
    double force[3];
    FaceBC face[6];
    int order[6];
    int any_face;
    int observe, write_mom, residual;
    int face_pass, fp_face;   // face pass: update the nodes of face fp_face only
    int* err;                 // set to 1 when a bounded wait gives up
    long long wait_limit;     // polls of a bounded wait before it gives up (< 0: WAIT_LIMIT)
    int pipe_stages, pipe_nc; // pipelined sweep: ring stages, consumer warps
    const uint32_t* list;     // compacted sweep: work entries (see k_step_list)
    long long nlist;
    long long kbeg, kend;     // sparse sweep: the fluid indices it updates (a z-slab: its owned planes)
    double inv_nx, inv_ny;    // 1/nx, 1/ny for index -> coordinate conversion
    int z0, zpad;             // first z plane of the dense sweep (slab domains sweep [z0, z0 + gridDim.z))
    // sparse layout (fluid nodes only, see k_step_sparse): list = fluid node cells,
    // nlist = fluid count, fmask = mask word per fluid node, rw = row words
    const uint32_t* fmask;
    const uint2* rw;
    int rw_w;
    int pf_blocks;            // sparse sweep: a block prefetches into L2 what block + pf_blocks reads first (0: off)
    long long np;             // population plane stride in elements (planes of one buffer are np apart)
    const GateView* gate;     // batch member state, or null outside batches
    int gate_j;               // chunk step of this launch
    int packed;               // sparse list entries are x | y << 11 | z << 22 (else node indices)
    int sweep_mode;           // sparse layout: SWEEP_PULL / SWEEP_PUSH (A/B buffers), SWEEP_AA_EVEN / _ODD (in place)
    int sround;               // 16-bit storage: 1 = stochastic rounding (seeded by node and time step), 0 = nearest
    unsigned tstep;           // time step of the launch (low 32 bits; the rounding seed)
    int tpad;
    long long seed_offset;    // node index of this lattice's node 0 in the whole lattice (z-slabs)
    double bgk_cb;            // 1 - 1/(2 tau) of the momentum BGK source, computed once
    // previous-step moments of the two node layers next to each face:
    // [layer 0/1][field u_0..u_{D-1}, C_0..][plane node], compute type, pb_nf fields
    const void* pb_src[6];
    void* pb_dst[6];
    long long pb_plane[6];
    // per-node moments for residuals: [field][N] (rho, u_0.., C_0..), compute type
    const void* mom_prev;
    void* mom_cur;
    double* accum;   // residual partials: [accumulator][accum_stride] per-block slots
    long long accum_stride, slot0;   // slots per accumulator; first slot of this launch's blocks
    long long res_slots;             // batches: slots a member's residual step fills
    double* obs_rho;
    double* obs_u;
    double* obs_c;           // scalar s at obs_c + s N
    // passive scalars, advanced one after another in the momentum sweep
    int has_scalar, nscalar;   // has_scalar = nscalar > 0
    int pb_nf, ns_pad;         // fields per face layer: D + max(nscalar, 1)
    ScalarParams sc[NSMAX];
};

template <int VS>
struct KParams : StepParams {};
// D3Q27 MRT: population-space collision matrix Lambda = M^-1 S M, built on the host.
template <>
struct KParams<VS_D3Q27> : StepParams {
    float lam32[27 * 27];
    double lam64[27 * 27];
};

// ---- storage formats -----------------------------------------------------
// FP64 storage holds the populations f_i themselves (the reference arithmetic).
// The FP32-compute formats hold the deviation h_i = f_i - w_i ("DDF shifting"):
// at low Mach numbers f_i ~ w_i, so storing and colliding h_i keeps the small
// physical signal instead of rounding it against w_i.
template <int ST>
struct Store;
template <>
struct Store<ST_F64> {
    using T = double;
    using R = double;
    static constexpr bool DEV = false;
    __device__ static __forceinline__ R sc(R v) { return v; }
    __device__ static __forceinline__ R unsc(R v) { return v; }
    __device__ static __forceinline__ R ld(const void* p, int o) { return ((const T*)p)[o]; }
    __device__ static __forceinline__ R cvt(T v) { return v; }
    __device__ static __forceinline__ void st(void* p, int o, R v) { ((T*)p)[o] = v; }
    __device__ static __forceinline__ T enc(R v) { return v; }
};
template <>
struct Store<ST_F32> {
    using T = float;
    using R = float;
    static constexpr bool DEV = true;
    __device__ static __forceinline__ R sc(R v) { return v; }
    __device__ static __forceinline__ R unsc(R v) { return v; }
    __device__ static __forceinline__ R ld(const void* p, int o) { return ((const T*)p)[o]; }
    __device__ static __forceinline__ R cvt(T v) { return v; }
    __device__ static __forceinline__ void st(void* p, int o, R v) { ((T*)p)[o] = v; }
    __device__ static __forceinline__ T enc(R v) { return v; }
};
// FP16 holds h_i * 2^14: at low Mach numbers h_i is 1e-7..1e-4, below FP16's
// smallest normal number (6.1e-5), where the subnormal spacing (6e-8) would cost
// most of the signal; scaled, every |h| > 3.7e-9 is a normal number with 11
// significant bits, and |h| < 4 (it is below 1 for any physical state) stays
// finite.  The scale is a power of two, so scaling itself is exact.
// The step kernels keep the scaled values H = h * 2^14 in registers: ld/cvt/st
// move H, the moments unscale the sums (sc/unsc), and the collision folds the
// scale into its per-node factors.  Every rounding commutes with an exact power
// of two, so the stored bits are those of unscale -> collide -> scale, with 2 x Q
// fewer multiplies per node.
constexpr float F16_SCALE = 16384.0f, F16_UNSCALE = 1.0f / 16384.0f;
template <>
struct Store<ST_F16> {
    using T = __half;
    using R = float;
    static constexpr bool DEV = true;
    __device__ static __forceinline__ R sc(R v) { return v * F16_SCALE; }
    __device__ static __forceinline__ R unsc(R v) { return v * F16_UNSCALE; }
    __device__ static __forceinline__ R ld(const void* p, int o) { return __half2float(((const T*)p)[o]); }
    __device__ static __forceinline__ R cvt(T v) { return __half2float(v); }
    __device__ static __forceinline__ void st(void* p, int o, R v) { ((T*)p)[o] = __float2half_rn(v); }
    __device__ static __forceinline__ T enc(R v) { return __float2half_rn(v); }
    // stochastic rounding: the 13 bits FP16 drops from a normal FP32 significand,
    // plus the top 13 bits of the random word `r`, truncated
    __device__ static __forceinline__ T enc_sr(R v, uint32_t r) {
        return __float2half_rz(__uint_as_float(__float_as_uint(v) + (r >> 19)));
    }
    // two values with the conversion's own stochastic rounding (random bits r):
    // .x = a, .y = b
    __device__ static __forceinline__ void enc_sr2(R a, R b, uint32_t r, T& ta, T& tb) {
        unsigned d;
        asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(r));
        ta = __ushort_as_half((unsigned short)(d >> 16));   // a goes to the upper half
        tb = __ushort_as_half((unsigned short)(d & 0xffffu));
    }
};
template <>
struct Store<ST_BF16> {
    using T = __nv_bfloat16;
    using R = float;
    static constexpr bool DEV = true;
    __device__ static __forceinline__ R sc(R v) { return v; }
    __device__ static __forceinline__ R unsc(R v) { return v; }
    __device__ static __forceinline__ R ld(const void* p, int o) { return __bfloat162float(((const T*)p)[o]); }
    __device__ static __forceinline__ R cvt(T v) { return __bfloat162float(v); }
    __device__ static __forceinline__ void st(void* p, int o, R v) { ((T*)p)[o] = __float2bfloat16_rn(v); }
    __device__ static __forceinline__ T enc(R v) { return __float2bfloat16_rn(v); }
    __device__ static __forceinline__ T enc_sr(R v, uint32_t r) {
        return __float2bfloat16_rz(__uint_as_float(__float_as_uint(v) + (r >> 16)));
    }
    __device__ static __forceinline__ void enc_sr2(R a, R b, uint32_t r, T& ta, T& tb) {
        unsigned d;
        asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(d) : "f"(a), "f"(b), "r"(r));
        ta = __ushort_as_bfloat16((unsigned short)(d >> 16));
        tb = __ushort_as_bfloat16((unsigned short)(d & 0xffffu));
    }
};

// ---- node geometry -----------------------------------------------------------
// Node coordinates, their periodic neighbours, and the 32-bit index offsets of
// the -1/+1 neighbours along each axis (N < 2^31, so one IADD3 per direction).
struct Geo {
    int x, y, z;
    int xm, xp, ym, yp, zm, zp;
    int cell;   // node index x + nx * (y + ny * z)
    int slot;   // index of the node's populations in the planes: the node index (dense
                // layouts) or the fluid-node index (sparse layout)
    int oxm, oxp, oym, oyp, ozm, ozp;
    __device__ __forceinline__ void offsets(const StepParams& P) {
        oxm = xm - x;
        oxp = xp - x;
        oym = (ym - y) * P.nx;
        oyp = (yp - y) * P.nx;
        ozm = (zm - z) * P.nx * P.ny;
        ozp = (zp - z) * P.nx * P.ny;
    }
    __device__ __forceinline__ int at(int dx, int dy, int dz, const StepParams&) const {
        return cell + (dx < 0 ? oxm : (dx > 0 ? oxp : 0)) + (dy < 0 ? oym : (dy > 0 ? oyp : 0)) +
               (dz < 0 ? ozm : (dz > 0 ? ozp : 0));
    }
};

__device__ __forceinline__ bool on_face(const Geo& g, int f, const StepParams& P) {
    switch (f) {
        case 0: return g.x == 0;
        case 1: return g.x == P.nx - 1;
        case 2: return g.y == 0;
        case 3: return g.y == P.ny - 1;
        case 4: return g.z == 0;
        default: return g.z == P.nz - 1;
    }
}
__device__ __forceinline__ int face_dist(const Geo& g, int f, const StepParams& P) {
    switch (f) {
        case 0: return g.x;
        case 1: return P.nx - 1 - g.x;
        case 2: return g.y;
        case 3: return P.ny - 1 - g.y;
        case 4: return g.z;
        default: return P.nz - 1 - g.z;
    }
}
__device__ __forceinline__ long long face_pos(const Geo& g, int f, const StepParams& P) {
    return f < 2 ? (long long)g.y + (long long)P.ny * g.z
                 : (f < 4 ? (long long)g.x + (long long)P.nx * g.z : (long long)g.x + (long long)P.nx * g.y);
}

// ---- reductions ----------------------------------------------------------------
// Per-block partial sums: the block whose slot is `slot` writes its K sums to
// accum[k * stride + slot].  No two blocks share an address and k_finalize adds
// the slots in index order, so a sum does not depend on how the blocks were
// scheduled: residuals, inventories and the steps at which a run stops repeat
// bit for bit from run to run.
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double* accum, long long stride, long long slot) {
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[wid][k] = s;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) accum[k * stride + slot] = s;
        }
    }
}
// The linear index of this block within its launch.
__device__ __forceinline__ long long block_linear() {
    return blockIdx.x + (long long)gridDim.x * (blockIdx.y + (long long)gridDim.y * blockIdx.z);
}
template <int K>
__device__ __forceinline__ void step_partials(double (&v)[K], const StepParams& P, long long local_block) {
    block_partials<K>(v, P.accum, P.accum_stride, P.slot0 + local_block);
}

// Partial sums into NSLOT shared slots with atomics: for a caller-provided
// scratch of fixed size (the allocation-free entry point); the order of the
// additions within a slot is not fixed.
template <int K>
__device__ __forceinline__ void block_accumulate(double (&v)[K], double* accum) {
    __shared__ double red[32][K];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[wid][k] = s;
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) {
                const unsigned long long b = blockIdx.x + (unsigned long long)gridDim.x *
                                                              (blockIdx.y + (unsigned long long)gridDim.y * blockIdx.z);
                atomicAdd(&accum[(b % NSLOT) * NACC + k], s);
            }
        }
    }
}

// ---- equilibrium (src/kernel.rs:3-26) -------------------------------------------
template <class L, class R>
__device__ __forceinline__ R feq_i(int i, R rho, const R* u, R uu) {
    R cu = R(0);
#pragma unroll
    for (int a = 0; a < L::D; ++a) cu += u[a] * R(L::c(i, a));
    return R(L::w(i)) * rho * (R(1) + cu * R(3) + R(0.5) * cu * cu * R(9) - R(0.5) * uu * R(3));
}
// f_eq - w_i = w_i (drho + rho (3 c.u + 4.5 (c.u)^2 - 1.5 u.u)), drho = rho - 1.
template <class L, class R>
__device__ __forceinline__ R heq_i(int i, R rho, R drho, const R* u, R uu) {
    R cu = R(0);
#pragma unroll
    for (int a = 0; a < L::D; ++a) cu += u[a] * R(L::c(i, a));
    return R(L::w(i)) * (drho + rho * (cu * R(3) + R(0.5) * cu * cu * R(9) - R(0.5) * uu * R(3)));
}
// Equilibrium in the register representation of the storage format.
template <class L, bool DEV, class R>
__device__ __forceinline__ R eq_i(int i, R rho, R drho, const R* u, R uu) {
    if constexpr (DEV) return heq_i<L, R>(i, rho, drho, u, uu);
    else return feq_i<L, R>(i, rho, u, uu);
}

// Guo source without the (1 - omega/2) factor (src/kernel.rs:122-154).
template <class L, class R>
__device__ __forceinline__ R guo_i(int i, const R* u, const R* F) {
    R cu = R(0);
#pragma unroll
    for (int a = 0; a < L::D; ++a) cu += u[a] * R(L::c(i, a));
    R s = R(0);
#pragma unroll
    for (int a = 0; a < L::D; ++a) s += (R(3) * R(L::c(i, a)) - R(3) * u[a] + R(9) * cu * R(L::c(i, a))) * F[a];
    return R(L::w(i)) * s;
}

// Reference MRT equilibrium moments, bug for bug
// (src/velocity_set/d2q9.rs:247-264, src/velocity_set/d3q19.rs:550-587).
// With DEV the moments of the weights (M w: [1,-2,1,0..] for D2Q9,
// [1,-11,3,0..] for D3Q19) are subtracted, as the populations are h = f - w.
template <int VS, bool DEV, class R>
__device__ __forceinline__ void meq_reference(R rho, R drho, const R* u, R* m) {
    const R base = DEV ? drho : rho;
    if constexpr (VS == VS_D2Q9) {
        const R s = u[0] * u[0] + u[1] * u[1];
        m[0] = base;
        m[1] = DEV ? (drho + R(3)) - R(3) * rho * s : rho - R(3) * rho * s;
        m[2] = R(9) * rho * u[0] * u[0] * u[1] * u[1] - R(3) * rho * s + base;
        m[3] = rho * u[0];
        m[4] = R(3) * rho * u[0] * u[0] * u[0] - rho * u[0];
        m[5] = rho * u[1];
        m[6] = R(3) * rho * u[1] * u[1] * u[1] - rho * u[1];
        m[7] = rho * s;
        m[8] = rho * u[0] * u[1];
    } else if constexpr (VS == VS_D3Q19) {
        const R s = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const R bug = R(2) * rho * u[0] * u[0] - rho * (u[1] * u[1] + u[2] + u[2]);
        m[0] = base;
        m[1] = R(-11) * base + R(19) * rho * s;
        m[2] = R(3) * base - R(5.5) * rho * s;
        m[3] = rho * u[0];
        m[4] = R(-2.0 / 3.0) * rho * u[0];
        m[5] = rho * u[1];
        m[6] = R(-2.0 / 3.0) * rho * u[1];
        m[7] = rho * u[2];
        m[8] = R(-2.0 / 3.0) * rho * u[2];
        m[9] = bug;
        m[10] = R(-0.5) * bug;
        m[11] = rho * (u[1] * u[1] - u[2] * u[2]);
        m[12] = R(-0.5) * rho * (u[1] * u[1] - u[2] * u[2]);
        m[13] = rho * u[0] * u[1];
        m[14] = rho * u[1] * u[2];
        m[15] = rho * u[0] * u[2];
        m[16] = R(0);
        m[17] = R(0);
        m[18] = R(0);
    }
}

template <int VS, class R>
__device__ __forceinline__ R lam_at(const KParams<VS>& P, int k) {
    if constexpr (VS == VS_D3Q27) {
        if constexpr (sizeof(R) == 8) return P.lam64[k];
        else return P.lam32[k];
    } else {
        return R(0);
    }
}

// Collision in place on f (registers) given feq; src/kernel.rs:28-120 and the
// force source of src/momentum/node.rs:311-333 (BGK) / the physics mode.
template <int VS, int COLL, bool DEV, class R>
__device__ __forceinline__ void collide(const KParams<VS>& P, R (&f)[Lat<VS>::Q], const R (&fe)[Lat<VS>::Q], R rho,
                                        R drho, const R* u, const R* F, bool force, double tau, double omega,
                                        double op, double om, const double* rates, int compat) {
    using L = Lat<VS>;
    constexpr int Q = L::Q;
    if constexpr (COLL == COLL_BGK) {
        const R w1 = R(omega), w0 = R(1) - R(omega);
        const R cb = R(1.0 - 0.5 / tau);
        sfor<Q>([&](auto I) {
            constexpr int i = I;
            R v = w0 * f[i] + w1 * fe[i];
            if (force) v += cb * guo_i<L, R>(i, u, F);
            f[i] = v;
        });
    } else if constexpr (COLL == COLL_TRT) {
        const R wp = R(op), wm = R(om);
        const bool src = force && compat == COMPAT_PHYSICS;
        const R cp = R(1.0 - 0.5 * op), cm = R(1.0 - 0.5 * om);
        R out[Q];
        sfor<Q>([&](auto I) {
            constexpr int i = I;
            constexpr int ib = L::qbar(i);
            const R fp = R(0.5) * (f[i] + f[ib]), fep = R(0.5) * (fe[i] + fe[ib]);
            const R fm = R(0.5) * (f[i] - f[ib]), fem = R(0.5) * (fe[i] - fe[ib]);
            R v = f[i] - wp * (fp - fep) - wm * (fm - fem);
            if (src) {
                const R si = guo_i<L, R>(i, u, F), sb = guo_i<L, R>(ib, u, F);
                v += cp * R(0.5) * (si + sb) + cm * R(0.5) * (si - sb);
            }
            out[i] = v;
        });
        sfor<Q>([&](auto I) { f[I] = out[I]; });
    } else {   // MRT
        if constexpr (VS == VS_D3Q27) {
            const bool src = force && compat == COMPAT_PHYSICS;
            R d[Q], s[Q];
            sfor<Q>([&](auto I) { d[I] = f[I] - fe[I]; });
            if (src) sfor<Q>([&](auto I) { s[I] = guo_i<L, R>(I, u, F); });
            sfor<Q>([&](auto I) {
                constexpr int i = I;
                R acc = R(0), accs = R(0);
                sfor<Q>([&](auto J) {
                    const R lam = lam_at<VS, R>(P, i * Q + J);
                    acc += lam * d[J];
                    if (src) accs += lam * s[J];
                });
                f[i] = f[i] - acc + (src ? s[i] - R(0.5) * accs : R(0));
            });
        } else {
            R m[Q], me[Q];
            sfor<Q>([&](auto K) {
                constexpr int k = K;
                R a = R(0);
                sfor<Q>([&](auto I) {
                    constexpr double c = L::M(k, I);
                    if constexpr (c != 0.0) a += R(c) * f[I];
                });
                m[k] = a;
            });
            if (compat == COMPAT_REFERENCE) {
                meq_reference<VS, DEV, R>(rho, drho, u, me);
            } else {
                sfor<Q>([&](auto K) {
                    constexpr int k = K;
                    R a = R(0);
                    sfor<Q>([&](auto I) {
                        constexpr double c = L::M(k, I);
                        if constexpr (c != 0.0) a += R(c) * fe[I];
                    });
                    me[k] = a;
                });
            }
            const bool src = force && compat == COMPAT_PHYSICS;
            R ms[Q];
            if (src) {
                R s[Q];
                sfor<Q>([&](auto I) { s[I] = guo_i<L, R>(I, u, F); });
                sfor<Q>([&](auto K) {
                    constexpr int k = K;
                    R a = R(0);
                    sfor<Q>([&](auto I) {
                        constexpr double c = L::M(k, I);
                        if constexpr (c != 0.0) a += R(c) * s[I];
                    });
                    ms[k] = (R(1) - R(0.5) * R(rates[k])) * a;
                });
            }
            sfor<Q>([&](auto K) {
                constexpr int k = K;
                m[k] = m[k] - R(rates[k]) * (m[k] - me[k]) + (src ? ms[k] : R(0));
            });
            sfor<Q>([&](auto I) {
                constexpr int i = I;
                R a = R(0);
                sfor<Q>([&](auto K) {
                    constexpr double c = mrt_inv<L>(i, K);
                    if constexpr (c != 0.0) a += R(c) * m[K];
                });
                f[i] = a;
            });
        }
    }
}

// D2Q9 Zou-He, src/velocity_set/d2q9.rs:165-245 (formulas verbatim).
// `one` is 1 when f holds deviations h = f - w (the weights of the known
// populations in each sum add up to 1), 0 otherwise.
template <class R>
__device__ __forceinline__ void zou_he_d2q9(int face, R* f, const FaceBC& b, R one) {
    const bool vel = !b.has_rho;
    R rho, ux, uy;
    switch (face) {
        case 0:
            uy = R(b.u[1]);
            if (vel) { ux = R(b.u[0]); rho = R(1) / (R(1) - ux) * (one + f[0] + f[2] + f[4] + R(2) * (f[3] + f[6] + f[7])); }
            else { rho = R(b.rho); ux = R(1) - R(1) / rho * (one + f[0] + f[2] + f[4] + R(2) * (f[3] + f[6] + f[7])); }
            f[1] = f[3] + R(2.0 / 3.0) * rho * ux;
            f[5] = f[7] - R(0.5) * (f[2] - f[4]) + R(0.5) * rho * uy + R(1.0 / 6.0) * rho * ux;
            f[8] = f[6] + R(0.5) * (f[2] - f[4]) - R(0.5) * rho * uy + R(1.0 / 6.0) * rho * ux;
            break;
        case 1:
            uy = R(b.u[1]);
            if (vel) { ux = R(b.u[0]); rho = R(1) / (R(1) + ux) * (one + f[0] + f[2] + f[4] + R(2) * (f[1] + f[5] + f[8])); }
            else { rho = R(b.rho); ux = R(1) / rho * (one + f[0] + f[2] + f[4] + R(2) * (f[1] + f[5] + f[8])) - R(1); }
            f[3] = f[1] - R(2.0 / 3.0) * rho * ux;
            f[7] = f[5] + R(0.5) * (f[2] - f[4]) - R(0.5) * rho * uy - R(1.0 / 6.0) * rho * ux;
            f[6] = f[8] - R(0.5) * (f[2] - f[4]) + R(0.5) * rho * uy - R(1.0 / 6.0) * rho * ux;
            break;
        case 2:
            ux = R(b.u[0]);
            if (vel) { uy = R(b.u[1]); rho = R(1) / (R(1) - uy) * (one + f[0] + f[1] + f[3] + R(2) * (f[4] + f[7] + f[8])); }
            else { rho = R(b.rho); uy = R(1) - R(1) / rho * (one + f[0] + f[1] + f[3] + R(2) * (f[4] + f[7] + f[8])); }
            f[2] = f[4] + R(2.0 / 3.0) * rho * uy;
            f[5] = f[7] - R(0.5) * (f[1] - f[3]) + R(0.5) * rho * ux + R(1.0 / 6.0) * rho * uy;
            f[6] = f[8] + R(0.5) * (f[1] - f[3]) - R(0.5) * rho * ux + R(1.0 / 6.0) * rho * uy;
            break;
        default:
            ux = R(b.u[0]);
            if (vel) { uy = R(b.u[1]); rho = R(1) / (R(1) + uy) * (one + f[0] + f[1] + f[3] + R(2) * (f[2] + f[5] + f[6])); }
            else { rho = R(b.rho); uy = R(1) / rho * (one + f[0] + f[1] + f[3] + R(2) * (f[2] + f[5] + f[6])) - R(1); }
            f[4] = f[2] - R(2.0 / 3.0) * rho * uy;
            f[7] = f[5] + R(0.5) * (f[1] - f[3]) - R(0.5) * rho * ux - R(1.0 / 6.0) * rho * uy;
            f[8] = f[6] - R(0.5) * (f[1] - f[3]) + R(0.5) * rho * ux - R(1.0 / 6.0) * rho * uy;
            break;
    }
}

// sum of c_A^2 over the directions with c_ax * sgn = +1 (the unknowns of a face)
template <class L, int ax, int sgn, int A>
__host__ __device__ constexpr int zou_he_m() {
    int m = 0;
    for (int i = 0; i < L::Q; ++i)
        if (L::c(i, ax) * sgn == 1) m += L::c(i, A) * L::c(i, A);
    return m;
}

// D3Q19 and D3Q27 Zou-He (engine extension; the reference has none): Hecht &
// Harting (2010), with the transverse correction of each tangential axis shared
// by all unknowns that move along it.
template <class L, int F, class R>
__device__ __forceinline__ void zou_he_3d(R* f, const FaceBC& b, R one) {
    constexpr int ax = F / 2;
    constexpr int sgn = (F & 1) ? -1 : 1;   // inward normal sign along ax
    R s0 = one, sout = R(0);
    sfor<L::Q>([&](auto I) {
        constexpr int cn = L::c(I, ax) * sgn;
        if constexpr (cn == 0) s0 += f[I];
        else if constexpr (cn < 0) sout += f[I];
    });
    R u[3] = {R(0), R(0), R(0)};
    R rho;
    if (!b.has_rho) {
        u[0] = R(b.u[0]); u[1] = R(b.u[1]); u[2] = R(b.u[2]);
        rho = (s0 + R(2) * sout) / (R(1) - R(sgn) * u[ax]);
    } else {
        rho = R(b.rho);
#pragma unroll
        for (int a = 0; a < 3; ++a) if (a != ax) u[a] = R(b.u[a]);
        u[ax] = R(sgn) * (R(1) - (s0 + R(2) * sout) / rho);
    }
    // transverse correction N_t = (S_t - 2 rho u_t / 3) / M, M = sum over the
    // unknowns of c_t^2: 2 for D3Q19 (S_t / 2 - rho u_t / 3), 6 for D3Q27
    R N[3] = {R(0), R(0), R(0)};
    sfor<3>([&](auto A) {
        if constexpr (A != ax) {
            R s = R(0);
            sfor<L::Q>([&](auto I) {
                if constexpr (L::c(I, ax) == 0 && L::c(I, A) != 0) s += R(L::c(I, A)) * f[I];
            });
            constexpr int M = zou_he_m<L, ax, sgn, A>();
            if constexpr (M == 2) N[A] = R(0.5) * s - rho * u[A] / R(3);
            else N[A] = s / R(M) - R(2) * rho * u[A] / R(3 * M);
        }
    });
    sfor<L::Q>([&](auto I) {
        constexpr int i = I;
        if constexpr (L::c(i, ax) * sgn == 1) {
            R cu = R(0), ct = R(0);
            sfor<3>([&](auto A) {
                cu += R(L::c(i, A)) * u[A];
                if constexpr (A != ax) ct += R(L::c(i, A)) * N[A];
            });
            f[i] = f[L::qbar(i)] + R(6.0 * L::w(i)) * rho * cu - ct;
        }
    });
}

// Face BCs on the momentum populations of a node on face F
// (src/momentum/bc.rs:62-149), after streaming and inner bounce-back.
template <int VS, int ST, int F>
__device__ __forceinline__ void momentum_face(const KParams<VS>& P, const Geo& g, typename Store<ST>::R* f) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    const FaceBC& b = P.face[F];
    const int kind = b.kind;
    if (kind == BC_PERIODIC) return;
    if (kind == BC_NO_SLIP || kind == BC_BOUNCE_BACK) {
        const R rw = R(b.rho);
        sfor<L::Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (leaves<L>(i, F)) {
                R v = S::unsc(S::ld(P.srcp[i], g.slot));
                if (kind == BC_BOUNCE_BACK) {
                    R cu = R(0);
#pragma unroll
                    for (int a = 0; a < L::D; ++a) cu += R(b.u[a]) * R(L::c(i, a));
                    v = v - R(2) * R(L::w(i)) * rw * R(3) * cu;
                }
                f[L::qbar(i)] = v;
            }
        });
    } else if (kind == BC_ANTI_BB) {
        // wall velocity 1.5 u(x) - 0.5 u(x + n) from the previous step (bc.rs:86-117)
        const long long pl = P.pb_plane[F], pos = face_pos(g, F, P);
        const R* pb = (const R*)P.pb_src[F];
        const int nf = P.pb_nf;
        R uw[3] = {R(0), R(0), R(0)};
#pragma unroll
        for (int a = 0; a < L::D; ++a)
            uw[a] = R(1.5) * pb[(0 * nf + a) * pl + pos] - R(0.5) * pb[(1 * nf + a) * pl + pos];
        R uu = R(0);
#pragma unroll
        for (int a = 0; a < L::D; ++a) uu += uw[a] * uw[a];
        const R rw = R(b.rho);
        sfor<L::Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (leaves<L>(i, F)) {
                R cu = R(0);
#pragma unroll
                for (int a = 0; a < L::D; ++a) cu += uw[a] * R(L::c(i, a));
                // with h = f - w: h[ibar] = -h*[i] + 2 w (rho_w (...) - 1)
                f[L::qbar(i)] = -S::unsc(S::ld(P.srcp[i], g.slot)) +
                                R(2) * R(L::w(i)) * (rw * (R(1) + R(0.5) * cu * cu * R(9) - R(0.5) * uu * R(3)) -
                                                     (S::DEV ? R(1) : R(0)));
            }
        });
    } else if (kind == BC_ZOU_HE) {
        if constexpr (VS == VS_D2Q9) zou_he_d2q9<R>(F, f, b, S::DEV ? R(1) : R(0));
        else zou_he_3d<L, F, R>(f, b, S::DEV ? R(1) : R(0));
    }
}

// Scalar face BCs of scalar `si` (src/passive_scalar/bc.rs:37-152).
// Extrapolation outflow (zeroth / second order) is applied by the face pass.
template <int VS, int F, class R>
__device__ __forceinline__ void scalar_face(const KParams<VS>& P, int si, const Geo& g, R* gg) {
    using L = Lat<VS>;
    const ScalarParams& sc = P.sc[si];
    const SFaceBC& b = sc.face[F];
    const int kind = b.kind;
    if (kind == SBC_PERIODIC) return;
    const R* gs = (const R*)sc.gsrc;
    const long long np = P.np;
    if (kind == SBC_ZEROTH || kind == SBC_SECOND) {
        // extrapolation from the neighbours along the inward normal
        // (src/passive_scalar/bc.rs:154-199); only the face pass reaches here.
        const long long pl = P.pb_plane[F], pos = face_pos(g, F, P);
        const R* sn = (const R*)sc.snap[F];
        const bool second = kind == SBC_SECOND, all = !b.unknown_only;
        sfor<L::Q>([&](auto J) {
            constexpr int j = J;
            if (all || leaves<L>(L::qbar(j), F)) {
                const R g1 = sn[(0 * L::Q + j) * pl + pos];
                gg[j] = second ? R(2) * g1 - sn[(1 * L::Q + j) * pl + pos] : g1;
            }
        });
        return;
    }
    if (kind == SBC_BB_NO_FLUX) {
        sfor<L::Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (leaves<L>(i, F)) gg[L::qbar(i)] = gs[i * np + g.slot];
        });
        return;
    }
    // anti-bounce-back with the wall equilibrium (bc.rs:107-140)
    const long long pl = P.pb_plane[F], pos = face_pos(g, F, P);
    const R* pb = (const R*)P.pb_src[F];
    const int nf = P.pb_nf;
    R uw[3] = {R(0), R(0), R(0)};
    if (b.given_vel) {
#pragma unroll
        for (int a = 0; a < L::D; ++a) uw[a] = R(b.u[a]);
    } else {
#pragma unroll
        for (int a = 0; a < L::D; ++a)
            uw[a] = R(1.5) * pb[(0 * nf + a) * pl + pos] - R(0.5) * pb[(1 * nf + a) * pl + pos];
    }
    const R sval = kind == SBC_ANTI_BB ? R(b.value) : pb[(0 * nf + L::D + si) * pl + pos];
    R uu = R(0);
#pragma unroll
    for (int a = 0; a < L::D; ++a) uu += uw[a] * uw[a];
    sfor<L::Q>([&](auto I) {
        constexpr int i = I;
        if constexpr (leaves<L>(i, F)) {
            R cu = R(0);
#pragma unroll
            for (int a = 0; a < L::D; ++a) cu += uw[a] * R(L::c(i, a));
            const R ge = R(L::w(i)) * sval * (R(1) + cu * R(3) + R(0.5) * cu * cu * R(9) - R(0.5) * uu * R(3));
            gg[L::qbar(i)] = -gs[i * np + g.slot] + R(2) * ge;
        }
    });
}

// Apply the momentum face BCs of a node in the configured order (P.order).
// Both loops are unrolled: six copies of the face rules, but no loop state live
// across them (a runtime loop over the order positions needs more registers).
// Only nodes on explicit faces run this code; no-slip walls fold into the link
// bits, so in a duct or a packed bed the bulk of the lattice never fetches it.
template <int VS, int ST>
__device__ __forceinline__ void apply_faces(const KParams<VS>& P, const Geo& g, typename Store<ST>::R* f) {
    using L = Lat<VS>;
    sfor<L::NF>([&](auto O) {
        const int fr = P.order[O];
        sfor<L::NF>([&](auto FF) {
            constexpr int F = FF;
            if (fr == F && on_face(g, F, P)) momentum_face<VS, ST, F>(P, g, f);
        });
    });
}

// The face BCs of scalar si in the same order.  The momentum and scalar rules
// touch disjoint populations and read no result of one another, so running all
// momentum faces first changes nothing.
template <int VS, class R>
__device__ __forceinline__ void apply_scalar_faces(const KParams<VS>& P, int si, const Geo& g, R* gg) {
    using L = Lat<VS>;
    sfor<L::NF>([&](auto O) {
        const int fr = P.order[O];
        sfor<L::NF>([&](auto FF) {
            constexpr int F = FF;
            if (fr == F) {
                // snapshot for an outflow face F, taken where F sits in the face order
                R* sn = (R*)P.sc[si].snap[F];
                if (sn) {
                    const int dist = face_dist(g, F, P);
                    if (dist == 1 || dist == 2) {
                        const long long pl = P.pb_plane[F], pos = face_pos(g, F, P);
                        sfor<L::Q>([&](auto J) { sn[((dist - 1) * L::Q + J) * pl + pos] = gg[J]; });
                    }
                }
                if (on_face(g, F, P)) scalar_face<VS, F, R>(P, si, g, gg);
            }
        });
    });
}

// Scalar source of one node (src/passive_scalar/node.rs:258-266 with
// src/passive_scalar/adsorption.rs:50-92).  Updates q when `commit`.
template <class R>
__device__ __forceinline__ bool scalar_source(const ScalarParams& P, bool bb, R c_stored, R& q, bool commit, R& out) {
    if (!P.ads) {
        out = R(P.source);
        return P.has_source != 0;
    }
    R ads = R(0);
    if (bb) {
        const R r = R(P.ka) * c_stored * (R(P.qmax) - q) - R(P.kd) * q;
        ads = -r;
        if (commit) {
            R qn = q + r;
            if (qn < R(0)) qn = R(0);
            else if (qn > R(P.qmax)) qn = R(P.qmax);
            q = qn;
        }
    }
    out = P.has_source ? R(P.source) + ads : ads;
    return true;
}

__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
// Explicitly rounded products and fused multiply-adds: the compiler may not
// contract them differently in different kernels, so every sweep variant of a
// step computes the same bits.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

// Equilibrium, collision and store of the post-collision populations.  BGK and
// TRT are evaluated one direction (BGK) or one opposite pair (TRT) at a time
// and stored at once, so only f[] stays live; MRT needs all moments together.
// ---- central-moment collision (D2Q9, D3Q27: tensor-product velocity sets) ----------
// An engine extension: the reference has no D3Q27 collision at all
// (src/velocity_set.rs:168).  The populations are transformed to central moments
// about the node velocity u by three passes of 3-point transforms, one per axis
// (the factorised "chimera" transform of Geier et al., Comput. Math. Appl. 70
// (2015) 507-547): along an axis with velocities (-1, 0, +1), raw moments
// M0 = f- + f0 + f+, M1 = f+ - f-, M2 = f+ + f-, then central ones k0 = M0,
// k1 = M1 - u M0, k2 = M2 - 2 u M1 + u^2 M0.  The moments relax towards those of
// the product-form equilibrium rho * c(a) c(b) c(c), c = (1, 0, 1/3):
//   order 0 conserved; order 1 reflected (k1 -> -k1: no change without a force,
//   adds F with the half-force velocity shift);
//   order 2: the deviatoric normal parts and the off-diagonal ones at omega = 1/tau
//   (shear viscosity (tau - 1/2) / 3), the trace at omega_bulk;
//   orders 3, 4, 5, 6 at omega_3 .. omega_6 (default 1: full relaxation to the
//   equilibrium, which is what keeps the scheme stable at tau close to 1/2).
// The inverse transform runs the passes backwards: M1 = k1 + u k0,
// M2 = k2 + 2 u k1 + u^2 k0, f+ = (M2 + M1) / 2, f- = (M2 - M1) / 2, f0 = M0 - M2.
// With deviation storage the transform runs on h = f - w: the weights' central
// moments about u are the products of (1, -u_a, 1/3 + u_a^2), subtracted from the
// equilibrium targets, so every quantity stays small (no rounding against w).
template <class L>
__host__ __device__ constexpr int cm_pos(int i) {
    return (L::c(i, 0) + 1) + 3 * (L::c(i, 1) + 1) + (L::D == 3 ? 9 * (L::c(i, 2) + 1) : 0);
}

template <int VS, int ST, class StoreFn>
__device__ __forceinline__ void central_collide(const KParams<VS>& P, typename Store<ST>::R (&f)[Lat<VS>::Q],
                                                typename Store<ST>::R rho, typename Store<ST>::R drho,
                                                const typename Store<ST>::R* u, StoreFn&& store) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int D = L::D, Q = L::Q;
    static_assert(Q == 9 || Q == 27, "central moments need a tensor-product velocity set");
    constexpr bool DEV = S::DEV;
    R v[Q];
    sfor<Q>([&](auto I) { v[cm_pos<L>(I)] = S::unsc(f[I]); });
    // forward passes: axis A (stride 1, 3, 9), velocities -1, 0, +1 at offsets 0, s, 2s
    sfor<D>([&](auto A) {
        constexpr int s = A == 0 ? 1 : (A == 1 ? 3 : 9);
        const R ua = u[A];
        sfor<Q / 3>([&](auto J) {
            constexpr int j = J;
            constexpr int base = (j % s) + (j / s) * 3 * s;   // line j of axis A
            const R fm = v[base], f0 = v[base + s], fp = v[base + 2 * s];
            const R M0 = fm + f0 + fp, M1 = fp - fm, M2 = fp + fm;
            v[base] = M0;
            v[base + s] = M1 - ua * M0;
            v[base + 2 * s] = M2 - R(2) * ua * M1 + ua * ua * M0;
        });
    });
    // relaxation; k(a, b, c) sits at a + 3 b + 9 c (a, b, c = moment order per axis)
    const R om = R(P.omega), ob = R(P.rates[0]);
    const R w3 = R(P.rates[1]), w4 = R(P.rates[2]), w5 = R(P.rates[3]), w6 = R(P.rates[4]);
    // Equilibrium targets.  Without deviations: rho * c(a) c(b) c(c).  With
    // deviations, minus the weights' central moments m(a) m(b) m(c), where
    // m = c + d with d(0) = 0, d(1) = -u, d(2) = u^2; the difference
    // rho c(a)c(b)c(c) - m(a)m(b)m(c) = drho * c(a)c(b)c(c) - Delta is evaluated as
    // Delta_1 = d_1, Delta_k = Delta_{k-1} (c_k + d_k) + (c_1 .. c_{k-1}) d_k, so that
    // no O(1) terms cancel (rho itself is 1 + drho and would lose drho's low bits).
    auto cf = [](int o) -> R { return o == 0 ? R(1) : (o == 1 ? R(0) : R(1.0 / 3.0)); };
    auto df = [&](int o, int ax) -> R { return o == 0 ? R(0) : (o == 1 ? -u[ax] : u[ax] * u[ax]); };
    auto eq = [&](int a, int b, int c) -> R {
        if constexpr (DEV) {
            const int o[3] = {a, b, c};
            R delta = df(a, 0), cprod = cf(a);
            for (int ax = 1; ax < D; ++ax) {
                delta = delta * (cf(o[ax]) + df(o[ax], ax)) + cprod * df(o[ax], ax);
                cprod = cprod * cf(o[ax]);
            }
            return drho * cprod - delta;
        } else {
            return rho * cf(a) * cf(b) * (D == 3 ? cf(c) : R(1));
        }
    };
    // first order: reflection about the equilibrium value (-u with deviations, 0 otherwise)
    sfor<D>([&](auto A) {
        constexpr int pos = A == 0 ? 1 : (A == 1 ? 3 : 9);
        v[pos] = (DEV ? R(2) * u[A] : R(0)) - v[pos];
    });
    // second order
    {
        constexpr int pxx = 2, pyy = 6, pzz = 18;
        const R dxx = v[pxx] - eq(2, 0, 0), dyy = v[pyy] - eq(0, 2, 0);
        if constexpr (D == 3) {
            const R dzz = v[pzz] - eq(0, 0, 2);
            const R tr = (R(1) - ob) * (dxx + dyy + dzz);
            const R dxy = (R(1) - om) * (dxx - dyy), dxz = (R(1) - om) * (dxx - dzz);
            const R nxx = (tr + dxy + dxz) * R(1.0 / 3.0);
            v[pxx] = eq(2, 0, 0) + nxx;
            v[pyy] = eq(0, 2, 0) + (nxx - dxy);
            v[pzz] = eq(0, 0, 2) + (nxx - dxz);
            v[4] = eq(1, 1, 0) + (R(1) - om) * (v[4] - eq(1, 1, 0));      // (1,1,0)
            v[10] = eq(1, 0, 1) + (R(1) - om) * (v[10] - eq(1, 0, 1));    // (1,0,1)
            v[12] = eq(0, 1, 1) + (R(1) - om) * (v[12] - eq(0, 1, 1));    // (0,1,1)
        } else {
            const R tr = (R(1) - ob) * (dxx + dyy), dxy = (R(1) - om) * (dxx - dyy);
            v[pxx] = eq(2, 0, 0) + R(0.5) * (tr + dxy);
            v[pyy] = eq(0, 2, 0) + R(0.5) * (tr - dxy);
            v[4] = eq(1, 1, 0) + (R(1) - om) * (v[4] - eq(1, 1, 0));
        }
    }
    // orders 3..6
    sfor<Q>([&](auto Pp) {
        constexpr int p = Pp;
        constexpr int a = p % 3, b = (p / 3) % 3, c = p / 9;
        constexpr int ord = a + b + c;
        if constexpr (ord >= 3) {
            const R w = ord == 3 ? w3 : (ord == 4 ? w4 : (ord == 5 ? w5 : w6));
            const R e = eq(a, b, c);
            v[p] = e + (R(1) - w) * (v[p] - e);
        }
    });
    // backward passes, last axis first
    sfor<D>([&](auto AA) {
        constexpr int A = D - 1 - AA;
        constexpr int s = A == 0 ? 1 : (A == 1 ? 3 : 9);
        const R ua = u[A];
        sfor<Q / 3>([&](auto J) {
            constexpr int j = J;
            constexpr int base = (j % s) + (j / s) * 3 * s;
            const R k0 = v[base], k1 = v[base + s], k2 = v[base + 2 * s];
            const R M1 = k1 + ua * k0, M2 = k2 + R(2) * ua * k1 + ua * ua * k0;
            v[base] = (M2 - M1) * R(0.5);
            v[base + s] = k0 - M2;
            v[base + 2 * s] = (M2 + M1) * R(0.5);
        });
    });
    sfor<Q>([&](auto I) { store(I, S::sc(v[cm_pos<L>(I)])); });
}

// 32-bit integer hash (two multiply / xor-shift rounds): the seed of a node's
// stochastic rounding in one time step.
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
// Odd multipliers that spread a node's seed over its directions.
__host__ __device__ constexpr uint32_t sr_mult(int i) { return 0x9e3779b1u + 0x632be5abu * (uint32_t)(2 * i); }

// Two 16-bit directions i, j (neither the rest population) with stochastic
// rounding by one paired conversion; returns the mass their rounding added.
template <class S, int I, int J, class Put>
__device__ __forceinline__ typename S::R store_pair_sr(typename S::R vi, typename S::R vj, uint32_t nseed,
                                                       Put&& put) {
    static_assert(I != 0 && J != 0, "the rest population is stored last, with the mass correction");
    typename S::T ti, tj;
    S::enc_sr2(vi, vj, nseed * sr_mult(I), ti, tj);
    put(IC<I>{}, ti);
    put(IC<J>{}, tj);
    return (vi - S::cvt(ti)) + (vj - S::cvt(tj));
}

// `put(IC<i>, t)` stores the post-collision value of direction i, already in the
// storage type.  `nseed` seeds the stochastic rounding of 16-bit storage.
template <int VS, int COLL, int ST, class Put>
__device__ __forceinline__ void collide_store(const KParams<VS>& P, typename Store<ST>::R (&f)[Lat<VS>::Q],
                                              typename Store<ST>::R rho, typename Store<ST>::R dr,
                                              const typename Store<ST>::R* u, typename Store<ST>::R uu,
                                              const typename Store<ST>::R* F, bool force, uint32_t nseed,
                                              Put&& put) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q;
    constexpr bool DEV = S::DEV;
    // 16-bit storage rounds every stored value to 11 (FP16) or 8 (BF16) significant
    // bits.  Two measures keep those roundings from adding up over the steps:
    // - the mass they add or remove is put back into the rest population, stored
    //   last, so the node's outgoing mass carries only the rest population's own
    //   rounding (its value is small, so is its ulp); mass is conserved, nothing
    //   damps a mass error, and density errors drive spurious pressure-gradient flow;
    // - stochastic rounding (P.sround): near a steady state the populations repeat
    //   from step to step, and round-to-nearest then repeats the same error at every
    //   step, a persistent spurious momentum source; rounding up or down with
    //   probability given by the distance makes the error zero-mean, so it averages
    //   out instead of accumulating.
    constexpr bool SIXTEEN = ST == ST_F16 || ST == ST_BF16;
    R merr = R(0), v0 = R(0);
    auto store = [&](auto I, R v) {
        using T = typename S::T;
        if constexpr (SIXTEEN) {
            if constexpr (int(I) == 0) {
                v0 = v;   // stored after the others
                return;
            } else {
                const T t = P.sround ? S::enc_sr(v, nseed * sr_mult(int(I))) : S::enc(v);
                merr += v - S::cvt(t);
                put(I, t);
            }
        } else {
            put(I, S::enc(v));
        }
    };
    if constexpr (COLL == COLL_BGK) {
        // f[] and the result are scaled by the storage scale: so are w1 and cb
        const R w1 = S::sc(R(P.omega)), w0 = R(1) - R(P.omega);
        const R cb = S::sc(R(P.bgk_cb));
        sfor<Q>([&](auto I) {
            constexpr int i = I;
            R v = w0 * f[i] + w1 * eq_i<L, DEV, R>(i, rho, dr, u, uu);
            if (force) v += cb * guo_i<L, R>(i, u, F);
            store(IC<i>{}, v);
        });
    } else if constexpr (COLL == COLL_TRT) {
        const R wp = R(P.op), wm = R(P.om);
        const bool src = force && P.compat == COMPAT_PHYSICS;
        const R cp = S::sc(R(1.0 - 0.5 * P.op)), cm = S::sc(R(1.0 - 0.5 * P.om));
        // for an opposite pair (i, ibar), c_ibar.u = -c_i.u: the symmetric part of the
        // equilibrium is w (base + rho (4.5 (c.u)^2 - 1.5 u.u)), the antisymmetric 3 w rho c.u
        const R base = DEV ? dr : rho;
        const R ruu = mul_rn(mul_rn(R(1.5), rho), uu);
        // f_i - wp (f+_i - feq+_i) - wm (f-_i - feq-_i) in affine form:
        // f*_i = a f_i + b f_ibar + wp feq+_i + wm feq-_i, f*_ibar = a f_ibar + b f_i + wp feq+_i - wm feq-_i,
        // a = 1 - (wp + wm) / 2, b = (wm - wp) / 2; the per-node factors k2, k0, k1 and their
        // products with each weight are shared by every pair of that weight
        const R a = fma_rn(R(-0.5), add_rn(wp, wm), R(1)), bb = mul_rn(R(0.5), add_rn(wm, -wp));
        // f[] and the results are scaled by the storage scale: so are k2, k0, k1 and cp, cm
        const R k2 = S::sc(mul_rn(wp, mul_rn(R(4.5), rho))), k0 = S::sc(mul_rn(wp, add_rn(base, -ruu)));
        const R k1 = S::sc(mul_rn(wm, mul_rn(R(3), rho)));
        sfor<Q>([&](auto I) {
            constexpr int i = I, ib = L::qbar(i);
            if constexpr (i <= ib) {
                R cu = R(0);
                sfor<L::D>([&](auto A) {
                    constexpr int c = L::c(i, A);
                    if constexpr (c == 1) cu += u[A];
                    else if constexpr (c == -1) cu -= u[A];
                });
                const R wi = R(L::w(i));
                const R sym = fma_rn(mul_rn(wi, k2), mul_rn(cu, cu), mul_rn(wi, k0));   // wp feq+_i
                const R asym = mul_rn(mul_rn(wi, k1), cu);                           // wm feq-_i
                R vi = fma_rn(a, f[i], fma_rn(bb, f[ib], add_rn(sym, asym)));
                R vb = fma_rn(a, f[ib], fma_rn(bb, f[i], add_rn(sym, -asym)));
                if (src) {
                    const R si = guo_i<L, R>(i, u, F), sb = guo_i<L, R>(ib, u, F);
                    vi += cp * R(0.5) * (si + sb) + cm * R(0.5) * (si - sb);
                    vb += cp * R(0.5) * (sb + si) + cm * R(0.5) * (sb - si);
                }
                if constexpr (SIXTEEN && i != ib && i != 0) {
                    // the pair rounded stochastically by one paired conversion
                    // (cvt.rs on sm_100a), one random word per pair
                    if (P.sround) merr += store_pair_sr<S, i, ib>(vi, vb, nseed, put);
                    else { store(IC<i>{}, vi); store(IC<ib>{}, vb); }
                } else {
                    store(IC<i>{}, vi);
                    if constexpr (i != ib) store(IC<ib>{}, vb);
                }
            }
        });
    } else if constexpr (COLL == COLL_CENTRAL) {
        if constexpr (L::Q == 9 || L::Q == 27) central_collide<VS, ST>(P, f, rho, dr, u, store);
    } else if constexpr (VS == VS_D3Q27) {
        // population-space MRT, f* = f - Lambda (f - f_eq) (+ the Guo source in physics
        // mode): only the Q deviations e = f - f_eq (+ s/2) stay live through the
        // Q x Q product, and f_eq_i is re-evaluated when row i is stored, so that FP64
        // fits the register budget.  With e_j = d_j + s_j / 2:
        // f_i - sum_j L_ij d_j + s_i - sum_j L_ij s_j / 2 = feq_i + e_i + s_i / 2 - sum_j L_ij e_j
        const bool src = force && P.compat == COMPAT_PHYSICS;
        R e[Q];
        sfor<Q>([&](auto I) {
            constexpr int i = I;
            R v = S::unsc(f[i]) - eq_i<L, DEV, R>(i, rho, dr, u, uu);
            if (src) v += R(0.5) * guo_i<L, R>(i, u, F);
            e[i] = v;
        });
        sfor<Q>([&](auto I) {
            constexpr int i = I;
            R acc = R(0);
            sfor<Q>([&](auto J) { acc += lam_at<VS, R>(P, i * Q + J) * e[J]; });
            R v = eq_i<L, DEV, R>(i, rho, dr, u, uu) + e[i] - acc;
            if (src) v += R(0.5) * guo_i<L, R>(i, u, F);
            store(IC<i>{}, S::sc(v));
        });
    } else {
        R fe[Q];
        sfor<Q>([&](auto I) { fe[I] = eq_i<L, DEV, R>(I, rho, dr, u, uu); });
        sfor<Q>([&](auto I) { f[I] = S::unsc(f[I]); });
        collide<VS, COLL, DEV, R>(P, f, fe, rho, dr, u, F, force, P.tau, P.omega, P.op, P.om, P.rates, P.compat);
        sfor<Q>([&](auto I) { store(I, S::sc(f[I])); });
    }
    if constexpr (SIXTEEN) {
        const R v = v0 + merr;
        put(IC<0>{}, P.sround ? S::enc_sr(v, nseed * sr_mult(0)) : S::enc(v));
    }
}

// ---- bulk-copy staging (cp.async.bulk into shared memory, mbarrier completion)
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// One contiguous global -> shared copy; 16-byte aligned addresses, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll suspends for a
// hardware-chosen interval) and reports failure instead of hanging.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase, long long limit) {
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}
constexpr long long WAIT_LIMIT = 1ll << 22;
// The limit of a step's waits on its copies; the waits that let copies in flight
// land before a block exits always use WAIT_LIMIT.
__device__ __forceinline__ long long wait_limit(const StepParams& P) {
    return P.wait_limit < 0 ? WAIT_LIMIT : P.wait_limit;
}


// A launch that belongs to a stopped batch member, or to a step past its last
// one, does nothing (uniform over the grid).
__device__ __forceinline__ bool gated_off(const StepParams& P) {
    if (!P.gate) return false;
    const GateView g = *P.gate;
    return g.done_t >= 0 || g.t0 + P.gate_j > g.last_t;
}

// Residual accumulators of a sweep: rho, u_0..u_2, then one per scalar.
template <bool SCALAR>
__host__ __device__ constexpr int racc_n() { return SCALAR ? 4 + NSMAX : 5; }

// The momentum part of a fluid node after its populations were pulled: face
// BCs, moments, residual/observe/face-layer outputs, collision + store.
// `madd(J, v)` takes the node's squared residual term J (rho, u_0..) on
// residual steps; `put` stores the post-collision populations (see
// collide_store).  Returns the velocity (force-shifted) and its square, which
// the scalars' equilibria use.
// OUT = false: a step without outputs (not the first step, no residual, moment
// write or observation); those branches are then not compiled in.
template <int VS, int COLL, int ST, bool FACEBC, bool OUT = true, class MAdd, class Put>
__device__ __forceinline__ void momentum_cell(const KParams<VS>& P, const Geo& g, uint32_t mk,
                                              typename Store<ST>::R (&f)[Lat<VS>::Q], MAdd&& madd, Put&& put,
                                              typename Store<ST>::R (&u)[3], typename Store<ST>::R& uu) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q, D = L::D;
    constexpr bool DEV = S::DEV;
    const bool face_node = FACEBC && !P.first && (mk & (M_FACE | M_NEAR));
    // ---- face boundary conditions ------------------------------------------
    if constexpr (FACEBC) {
        if (face_node) {
            // the face rules work on unscaled populations
            sfor<Q>([&](auto I) { f[I] = S::unsc(f[I]); });
            apply_faces<VS, ST>(P, g, f);
            sfor<Q>([&](auto I) { f[I] = S::sc(f[I]); });
        }
    }

    // ---- moments (src/momentum/node.rs:418-457) ------------------------------
    R drho = R(0);
    sfor<Q>([&](auto I) { drho += f[I]; });
    drho = S::unsc(drho);
    const R rho = DEV ? R(1) + drho : drho;   // with h = f - w, sum h = rho - 1
    const R inv_rho = rcp_rn(rho);   // correctly rounded: the same value as 1 / rho
    u[0] = u[1] = u[2] = R(0);
    sfor<D>([&](auto A) {
        R s = R(0);
        sfor<Q>([&](auto I) {
            constexpr int c = L::c(I, A);
            if constexpr (c == 1) s += f[I];
            else if constexpr (c == -1) s -= f[I];
        });
        u[A] = S::unsc(s) * inv_rho;
    });
    R F[3] = {R(P.force[0]), R(P.force[1]), R(P.force[2])};
    const bool force = P.has_force != 0;
    if (force) sfor<D>([&](auto A) { u[A] += R(0.5) * F[A] * inv_rho; });
    const R dr = DEV ? drho : rho - R(1);
    uu = R(0);
    sfor<D>([&](auto A) { uu += u[A] * u[A]; });

    if (OUT && P.observe) {
        P.obs_rho[g.cell] = double(rho);
        sfor<D>([&](auto A) { P.obs_u[(long long)g.cell * D + A] = double(u[A]); });
    } else {
        // ---- residual moments (src/momentum/lattice.rs:369-394) ------------------
        if (OUT && P.residual) {
            const R* mp = (const R*)P.mom_prev;
            const double d0 = double(rho) - double(mp[g.cell]);
            madd(IC<0>{}, d0 * d0);
            sfor<D>([&](auto A) {
                const double du = double(u[A]) - double(mp[(1 + A) * P.N + g.cell]);
                madd(IC<1 + int(A)>{}, du * du);
            });
        }
        if (OUT && P.write_mom) {
            R* mc = (R*)P.mom_cur;
            mc[g.cell] = rho;
            sfor<D>([&](auto A) { mc[(1 + A) * P.N + g.cell] = u[A]; });
        }
        // ---- previous-step layers next to faces (anti-BB, extrapolation) ---------
        if constexpr (FACEBC) {
            if (P.any_face) {
                sfor<L::NF>([&](auto FF) {
                    constexpr int Fc = FF;
                    if (P.pb_dst[Fc]) {
                        const int dist = face_dist(g, Fc, P);
                        if (dist <= 1) {
                            R* pb = (R*)P.pb_dst[Fc];
                            const long long pl = P.pb_plane[Fc], pos = face_pos(g, Fc, P);
                            sfor<D>([&](auto A) { pb[(dist * P.pb_nf + A) * pl + pos] = u[A]; });
                        }
                    }
                });
            }
        }

        // ---- equilibrium + collision --------------------------------------------
        // the seed follows the node (index in the whole lattice), so every layout,
        // streaming scheme and z-slab split rounds a node's values alike
        const uint32_t nseed = (ST == ST_F16 || ST == ST_BF16)
                                   ? mix32((uint32_t)((long long)g.cell + P.seed_offset) ^ (P.tstep * 0x9e3779b9u))
                                   : 0u;
        collide_store<VS, COLL, ST>(P, f, rho, dr, u, uu, F, force, nseed, put);
    }
}

// The scalars of a fluid node, one after another (src/passive_scalar/lattice.rs:
// 241-297, node.rs:258-294), with the momentum velocity u of the same step.
// `gpull(si, gg)` fills gg with the pulled populations of scalar si, inner rule
// applied (the own populations on the first step).  They are pulled after the
// momentum store, so one population set is live at a time.  `radd(si, v)`
// takes the node's squared residual term of scalar si on residual steps.
template <int VS, int ST, bool FACEBC, class GPull, class RAdd>
__device__ __forceinline__ void scalar_cells(const KParams<VS>& P, const Geo& g, uint32_t mk,
                                             const typename Store<ST>::R (&u)[3], typename Store<ST>::R uu,
                                             GPull&& gpull, RAdd&& radd) {
    using L = Lat<VS>;
    using R = typename Store<ST>::R;
    constexpr int Q = L::Q, D = L::D;
    const bool face_node = FACEBC && !P.first && (mk & (M_FACE | M_NEAR));
    const bool bb = (mk & M_BB) != 0;
    {
#pragma unroll 1
        for (int si = 0; si < P.nscalar; ++si) {
            const ScalarParams& sc = P.sc[si];
            R gg[Q];
            gpull(si, gg);
            if constexpr (FACEBC) {
                if (face_node) apply_scalar_faces<VS, R>(P, si, g, gg);
            }
            // scalar value (node.rs:272-279)
            R q = R(0), cst = R(0);
            R cval = R(0);
            sfor<Q>([&](auto I) { cval += gg[I]; });
            if (sc.ads && bb) {
                q = ((const R*)sc.qads)[g.cell];
                cst = ((const R*)sc.cprev)[g.cell];
            }
            {
                R src;
                if (scalar_source<R>(sc, bb, cst, q, !P.observe, src)) cval += R(0.5) * src;
            }
            if (P.observe) {
                P.obs_c[(long long)si * P.N + g.cell] = double(cval);
                continue;
            }
            if (P.residual) {
                const R* mp = (const R*)P.mom_prev;
                const double dc = double(cval) - double(mp[(1 + D + si) * P.N + g.cell]);
                radd(si, dc * dc);
            }
            if (P.write_mom) ((R*)P.mom_cur)[(1 + D + si) * P.N + g.cell] = cval;
            if constexpr (FACEBC) {
                if (P.any_face) {
                    sfor<L::NF>([&](auto FF) {
                        constexpr int Fc = FF;
                        if (P.pb_dst[Fc]) {
                            const int dist = face_dist(g, Fc, P);
                            if (dist <= 1) {
                                R* pb = (R*)P.pb_dst[Fc];
                                const long long pl = P.pb_plane[Fc], pos = face_pos(g, Fc, P);
                                pb[(dist * P.pb_nf + D + si) * pl + pos] = cval;
                            }
                        }
                    });
                }
            }
            // equilibrium with the momentum velocity, then collision (ps/lattice.rs:254-272)
            R ge[Q];
            sfor<Q>([&](auto I) { ge[I] = feq_i<L, R>(I, cval, u, uu); });
            if (sc.coll == COLL_BGK) {
                const R w1 = R(sc.omega), w0 = R(1) - R(sc.omega);
                R src;
                const bool has = scalar_source<R>(sc, bb, cval, q, true, src);
                const R cb = R(sc.bgk_cb);
                sfor<Q>([&](auto I) {
                    R v = w0 * gg[I] + w1 * ge[I];
                    if (has) v += cb * R(L::w(I)) * src;
                    gg[I] = v;
                });
            } else {   // TRT, no source (src/lib.rs:118-127)
                const R wp = R(sc.op), wm = R(sc.om);
                R out[Q];
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    out[i] = gg[i] - wp * (R(0.5) * (gg[i] + gg[ib]) - R(0.5) * (ge[i] + ge[ib])) -
                             wm * (R(0.5) * (gg[i] - gg[ib]) - R(0.5) * (ge[i] - ge[ib]));
                });
                sfor<Q>([&](auto I) { gg[I] = out[I]; });
            }
            R* gd = (R*)sc.gdst;
            sfor<Q>([&](auto I) { gd[(long long)I * P.np + g.slot] = gg[I]; });
            if (sc.ads && bb) {
                ((R*)sc.qads)[g.cell] = q;
                ((R*)sc.cprev)[g.cell] = cval;
            }
        }
    }
}

// Everything a fluid node does after its populations were pulled: the momentum
// part, then the scalars.  Shared by every sweep.
template <int VS, int COLL, int ST, bool FACEBC, bool SCALAR, bool OUT = true, class Put, class GPull, int K>
__device__ __forceinline__ void process_cell_put(const KParams<VS>& P, const Geo& g, uint32_t mk,
                                                 typename Store<ST>::R (&f)[Lat<VS>::Q], double (&racc)[K],
                                                 Put&& put, GPull&& gpull) {
    using R = typename Store<ST>::R;
    R u[3], uu;
    momentum_cell<VS, COLL, ST, FACEBC, OUT>(P, g, mk, f, [&](auto J, double v) { racc[int(J)] += v; }, put, u,
                                             uu);
    if constexpr (SCALAR) {
        // a static index keeps racc in registers
        auto radd = [&](int si, double v) {
            sfor<NSMAX>([&](auto J) {
                if (si == int(J)) racc[4 + J] += v;
            });
        };
        scalar_cells<VS, ST, FACEBC>(P, g, mk, u, uu, gpull, radd);
    }
}

// A gpull for kernels without scalars.
struct NoScalarPull {
    template <class R>
    __device__ __forceinline__ void operator()(int, R*) const {}
};

// The A/B layouts: the post-collision populations go to slot `pidx` of the
// destination planes (the node index for the dense layouts, the fluid-node index
// for the sparse layout).
template <int VS, int COLL, int ST, bool FACEBC, bool SCALAR, bool OUT = true, class GPull, int K>
__device__ __forceinline__ void process_cell_at(const KParams<VS>& P, const Geo& g, uint32_t mk,
                                                typename Store<ST>::R (&f)[Lat<VS>::Q], double (&racc)[K],
                                                long long pidx, GPull&& gpull) {
    using S = Store<ST>;
    process_cell_put<VS, COLL, ST, FACEBC, SCALAR, OUT>(
        P, g, mk, f, racc, [&](auto I, typename S::T v) { ((typename S::T*)P.dstp[I])[pidx] = v; }, gpull);
}

template <int VS, int COLL, int ST, bool FACEBC, bool SCALAR, class GPull, int K>
__device__ __forceinline__ void process_cell(const KParams<VS>& P, const Geo& g, uint32_t mk,
                                             typename Store<ST>::R (&f)[Lat<VS>::Q], double (&racc)[K],
                                             GPull&& gpull) {
    process_cell_at<VS, COLL, ST, FACEBC, SCALAR>(P, g, mk, f, racc, g.cell, gpull);
}

// =================================================================== the step
// FACEBC: explicit face BCs (else no-slip walls are folded into the link bits).
// STAGE: one block per x-row; the Q source rows of the pull (and of the scalar)
// are brought into shared memory by bulk copies issued by one thread, so the
// bytes in flight do not occupy registers and every global read is a full,
// aligned line.  Requires blockDim.x == nx and nx * sizeof(T) % 16 == 0.
// Light kernels (BGK/TRT on D2Q9/D3Q19, FP32 compute, no scalar) are held to 64 registers
// so that at least 1024 threads fit on an SM; the others may use 128.
template <int VS, int COLL, int ST, bool SCALAR>
constexpr int light_kernel() {
    return COLL != COLL_MRT && COLL != COLL_CENTRAL && VS != VS_D3Q27 && !SCALAR && ST != ST_F64 ? 2 : 1;
}

template <int VS, int COLL, int ST, bool FACEBC, bool SCALAR, bool STAGE>
__global__ void __launch_bounds__(STAGE ? 512 : 256, (STAGE ? 1 : 2) * light_kernel<VS, COLL, ST, SCALAR>())
    k_step(const KParams<VS> P) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    using T = typename S::T;
    constexpr int Q = L::Q, D = L::D;
    if (gated_off(P)) return;

    Geo g;
    bool inside;
    const bool staged = STAGE && !P.face_pass && !P.first;
    if (FACEBC && P.face_pass) {
        // one thread per node of face fp_face
        const int F = P.fp_face;
        const long long pos = blockIdx.x * (long long)blockDim.x + threadIdx.x;
        inside = pos < P.pb_plane[F];
        const long long pp = inside ? pos : 0;
        if (F < 2) { g.x = F == 0 ? 0 : P.nx - 1; g.y = (int)(pp % P.ny); g.z = (int)(pp / P.ny); }
        else if (F < 4) { g.y = F == 2 ? 0 : P.ny - 1; g.x = (int)(pp % P.nx); g.z = (int)(pp / P.nx); }
        else { g.z = F == 4 ? 0 : P.nz - 1; g.x = (int)(pp % P.nx); g.y = (int)(pp / P.nx); }
    } else {
        g.x = blockIdx.x * blockDim.x + threadIdx.x;
        g.y = blockIdx.y;
        g.z = blockIdx.z + P.z0;
        inside = g.x < P.nx;
        if (!inside) g.x = 0;
    }
    g.cell = g.x + P.nx * (g.y + P.ny * g.z);
    g.slot = g.cell;
    g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
    g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
    g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
    g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
    g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
    g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
    g.offsets(P);

    // ---- stage the source rows of this x-row ------------------------------------
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* rows = (T*)smem_raw;
    R* grows = (R*)(smem_raw + (size_t)Q * P.nx * sizeof(T));
    if constexpr (STAGE) {
        if (staged) {
            const unsigned rb = (unsigned)(P.nx * sizeof(T));
            const unsigned grb = SCALAR ? (unsigned)(P.nx * sizeof(R)) : 0u;
            uint64_t* bar = (uint64_t*)(smem_raw + (size_t)Q * (rb + grb));
            if (threadIdx.x == 0) mbar_init(bar, 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                mbar_expect_tx(bar, Q * (rb + grb));
                sfor<Q>([&](auto I) {
                    constexpr int i = I;
                    // pull source row of direction i: (y - c_iy, z - c_iz), periodic
                    const int ys = L::c(i, 1) > 0 ? g.ym : (L::c(i, 1) < 0 ? g.yp : g.y);
                    const int zs = D == 3 ? (L::c(i, 2) > 0 ? g.zm : (L::c(i, 2) < 0 ? g.zp : g.z)) : 0;
                    const long long row = (long long)P.nx * ((long long)ys + (long long)P.ny * zs);
                    bulk_g2s(rows + (size_t)i * P.nx, (const T*)P.srcp[i] + row, rb, bar);
                    if constexpr (SCALAR)
                        bulk_g2s(grows + (size_t)i * P.nx, (const R*)P.sc[0].gsrc + (size_t)i * P.np + row, grb, bar);
                });
            }
            if (!mbar_wait_bounded(bar, 0, wait_limit(P))) {
                if (threadIdx.x == 0 && P.err) atomicExch(P.err, 1);
                mbar_wait_bounded(bar, 0, WAIT_LIMIT);   // let the copies in flight land
                return;
            }
        }
    }

    const uint32_t mk = inside ? P.mask[g.cell] : M_SOLID;
    bool active = !(mk & M_SOLID);
    if constexpr (FACEBC) active = active && ((P.face_pass != 0) == ((mk & M_SKIP) != 0));

    double racc[racc_n<SCALAR>()] = {};
    if (active) {
        // ---- stream (pull) + inner bounce-back -------------------------------
        R f[Q];
        if (P.first) {
            sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], g.cell); });
        } else {
            auto nb = [&](auto I) {
                constexpr int i = I;
                return g.at(-L::c(i, 0), -L::c(i, 1), D == 3 ? -L::c(i, 2) : 0, P);
            };
            // a warp whose nodes have no solid or wall links pulls without any test
            const bool nolinks = __all_sync(__activemask(), !(mk & M_LINKS));
            if (STAGE && staged) {
                auto pull = [&](auto I) {
                    constexpr int i = I;
                    const int xs = L::c(i, 0) > 0 ? g.xm : (L::c(i, 0) < 0 ? g.xp : g.x);
                    return S::cvt(rows[i * P.nx + xs]);
                };
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    f[i] = (mk >> ib & 1u) ? S::ld(P.srcp[ib], g.cell) : pull(I);
                });
            } else if (nolinks) {
                sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], nb(I)); });
            } else {
                // branch-free: a linked direction reads f*[ibar] of this node (inner
                // bounce-back / folded wall), the others the pull source
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    const bool lk = (mk >> ib) & 1u;
                    f[i] = S::ld(lk ? P.srcp[ib] : P.srcp[i], lk ? g.cell : nb(I));
                });
            }
        }
        // scalar populations: pull + inner BC (src/passive_scalar/lattice.rs:274-297);
        // the staged rows hold scalar 0
        auto gpull = [&](int si, R* gg) {
            const ScalarParams& sc = P.sc[si];
            const R* gs = (const R*)sc.gsrc;
            const long long np = P.np;
            if (P.first) {
                sfor<Q>([&](auto I) { gg[I] = gs[I * np + g.cell]; });
                return;
            }
            sfor<Q>([&](auto I) {
                constexpr int i = I, ib = L::qbar(i);
                const int n = g.at(-L::c(i, 0), -L::c(i, 1), D == 3 ? -L::c(i, 2) : 0, P);
                if (mk >> ib & 1u) {
                    const R own = gs[ib * np + g.cell];
                    if (sc.inner == 1) {
                        gg[i] = own;   // InnerBounceBack
                    } else {           // InnerAntiBounceBack: -g*[ib] + 2 w C_solid (ps/node.rs:281-294)
                        const R cs = sc.c_init ? R(sc.c_init[n]) : R(sc.c_solid);
                        gg[i] = -own + R(2) * R(L::w(ib)) * cs;
                    }
                } else if (STAGE && staged && si == 0) {
                    const int xs = L::c(i, 0) > 0 ? g.xm : (L::c(i, 0) < 0 ? g.xp : g.x);
                    gg[i] = grows[(size_t)i * P.nx + xs];
                } else {
                    gg[i] = gs[i * np + n];
                }
            });
        };
        process_cell<VS, COLL, ST, FACEBC, SCALAR>(P, g, mk, f, racc, gpull);
    }
    if (!P.observe && !P.face_pass && !P.first) {
        // Solid nodes are never read, but storing them when a node in the same
        // 32-byte sector is fluid turns partial-sector stores (which cost a DRAM
        // read to fill) into full-sector stores.  Lanes map to consecutive x.
        constexpr int per = 32 / (int)sizeof(T);
        const unsigned fl = __ballot_sync(__activemask(), active);
        const int lane = threadIdx.x & 31;
        const unsigned grp = (per >= 32 ? 0xffffffffu : ((1u << per) - 1u) << ((lane / per) * per));
        if (inside && (mk & M_SOLID) && (fl & grp)) {
            sfor<Q>([&](auto I) { S::st(P.dstp[I], g.cell, R(0)); });
            if constexpr (SCALAR) {
#pragma unroll 1
                for (int si = 0; si < P.nscalar; ++si)
                    sfor<Q>([&](auto I) { ((R*)P.sc[si].gdst)[I * P.np + g.cell] = R(0); });
            }
        }
    }
    if (P.residual && !P.observe) step_partials<racc_n<SCALAR>()>(racc, P, block_linear());
}

// =================================================================== compacted sweep
// The hot path of the lean case (periodic / no-slip faces, no scalar, not the
// first step, not observe).  Threads map to a per-domain list of work entries
// instead of to the dense lattice: every fluid node, plus every solid node that
// shares a 32-byte sector of the population planes with a fluid node (those
// store zeros, so that every store covers whole sectors and needs no DRAM read
// to fill).  In a porous medium this keeps all lanes busy with fluid work.
// Entry = node index | (1 << 31) when the node lies on a face of the box (only
// those need the periodic-wrap offsets; the others use constant ones) | (1 << 30)
// when the node is solid or has links (only those read the mask word).
template <int VS, int COLL, int ST>
__global__ void __launch_bounds__(256, ST == ST_F64 ? 2 : 4) k_step_list(const KParams<VS> P) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q, D = L::D;
    if (gated_off(P)) return;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const bool valid = t < P.nlist;
    const uint32_t e = valid ? P.list[t] : 0u;
    Geo g;
    g.cell = (int)(e & 0x3fffffffu);
    g.slot = g.cell;
    if (e >> 31) {
        // coordinates by a double-precision reciprocal plus a +-1 correction
        // (exact for indices < 2^31), much cheaper than integer division
        auto divq = [](int n, int d, double inv) {
            int q = (int)((double)n * inv);
            q -= ((long long)q * d > n);
            q += ((long long)(q + 1) * d <= n);
            return q;
        };
        const int row = divq(g.cell, P.nx, P.inv_nx);
        g.x = g.cell - row * P.nx;
        g.z = divq(row, P.ny, P.inv_ny);
        g.y = row - g.z * P.ny;
        g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
        g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
        g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
        g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
        g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
        g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
        g.offsets(P);
    } else {
        g.oxm = -1;
        g.oxp = 1;
        g.oym = -P.nx;
        g.oyp = P.nx;
        g.ozm = -P.nx * P.ny;
        g.ozp = P.nx * P.ny;
    }
    // plain fluid entries (no links) need neither the mask word nor any test
    const bool special = (e >> 30) & 1u;
    const uint32_t mk = !valid ? M_SOLID : (special ? P.mask[g.cell] : 0u);
    const bool active = !(mk & M_SOLID);
    double racc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (active) {
        R f[Q];
        if (__all_sync(__activemask(), !special)) {
            sfor<Q>([&](auto I) {
                constexpr int i = I;
                f[i] = S::ld(P.srcp[i], g.at(-L::c(i, 0), -L::c(i, 1), D == 3 ? -L::c(i, 2) : 0, P));
            });
        } else {
            sfor<Q>([&](auto I) {
                constexpr int i = I, ib = L::qbar(i);
                const bool lk = (mk >> ib) & 1u;
                f[i] = S::ld(lk ? P.srcp[ib] : P.srcp[i],
                             lk ? g.cell : g.at(-L::c(i, 0), -L::c(i, 1), D == 3 ? -L::c(i, 2) : 0, P));
            });
        }
        process_cell<VS, COLL, ST, false, false>(P, g, mk, f, racc, NoScalarPull{});
    } else if (valid) {
        sfor<Q>([&](auto I) { S::st(P.dstp[I], g.cell, R(0)); });
    }
    if (P.residual) step_partials<5>(racc, P, blockIdx.x);
}

// Marks the work entries of the compacted sweep and encodes them (see k_step_list).
template <int D>
__global__ void k_list_mark(const uint32_t* mask, long long N, int nx, int ny, int nz, int per, uint8_t* keep,
                            uint32_t* val) {
    const long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (cell >= N) return;
    bool k = !(mask[cell] & M_SOLID);
    if (!k) {
        const long long s0 = (cell / per) * per;
        for (long long c = s0; c < s0 + per && c < N; ++c) k = k || !(mask[c] & M_SOLID);
    }
    const int x = (int)(cell % nx), y = (int)((cell / nx) % ny), z = (int)(cell / ((long long)nx * ny));
    const bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1 || (D == 3 && (z == 0 || z == nz - 1));
    const bool special = (mask[cell] & (M_SOLID | M_LINKS)) != 0;
    keep[cell] = k ? 1 : 0;
    val[cell] = (uint32_t)cell | (edge ? 0x80000000u : 0u) | (special ? 0x40000000u : 0u);
}

// =================================================================== pipelined sweep
// Persistent blocks for the lean path (periodic / no-slip faces, no scalar).
// Warp 0 is the producer: one lane streams the Q source rows of each x-row the
// block owns (rows r = blockIdx.x + k * gridDim.x) into a ring of pipe_stages
// shared-memory stages with cp.async.bulk, each stage completing on its `full`
// mbarrier.  Warps 1..pipe_nc consume: wait on `full`, pull from the stage,
// collide, store, and release the stage on its `empty` mbarrier.  Several rows
// of copies are in flight per block at all times without occupying registers.
// Every wait is bounded; a timeout sets P.err and the block stops early.
template <int VS, int COLL, int ST>
__global__ void __launch_bounds__(288, 3) k_step_pipe(const KParams<VS> P) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    using T = typename S::T;
    constexpr int Q = L::Q, D = L::D;
    const int NS = P.pipe_stages, NC = P.pipe_nc;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const unsigned rb = (unsigned)(P.nx * sizeof(T));
    const size_t stage_bytes = (size_t)Q * rb;
    uint64_t* full = (uint64_t*)(smem_raw + NS * stage_bytes);
    uint64_t* empty = full + NS;
    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NC);
        }
    }
    __syncthreads();
    const long long nrows = (long long)P.ny * P.nz;
    double racc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};

    if (warp == 0) {
        if (lane == 0) {
            long long k = 0;
            bool failed = false;
            for (long long r = blockIdx.x; r < nrows; r += gridDim.x, ++k) {
                const int s = (int)(k % NS);
                const long long use = k / NS;
                if (use > 0 && !mbar_wait_bounded(&empty[s], (unsigned)((use - 1) & 1), wait_limit(P))) {
                    failed = true;
                    break;
                }
                mbar_expect_tx(&full[s], Q * rb);
                const int y = (int)(r % P.ny), z = (int)(r / P.ny);
                const int ym = y == 0 ? P.ny - 1 : y - 1, yp = y == P.ny - 1 ? 0 : y + 1;
                const int zm = z == 0 ? P.nz - 1 : z - 1, zp = z == P.nz - 1 ? 0 : z + 1;
                T* st = (T*)(smem_raw + s * stage_bytes);
                sfor<Q>([&](auto I) {
                    constexpr int i = I;
                    const int ys = L::c(i, 1) > 0 ? ym : (L::c(i, 1) < 0 ? yp : y);
                    const int zs = D == 3 ? (L::c(i, 2) > 0 ? zm : (L::c(i, 2) < 0 ? zp : z)) : 0;
                    const long long row = (long long)P.nx * ((long long)ys + (long long)P.ny * zs);
                    bulk_g2s(st + (size_t)i * P.nx, (const T*)P.srcp[i] + row, rb, &full[s]);
                });
            }
            // the copies of the last stages must land before the block may exit
            for (long long j = (k > NS ? k - NS : 0); j < k; ++j)
                mbar_wait_bounded(&full[j % NS], (unsigned)((j / NS) & 1), WAIT_LIMIT);
            if (failed && P.err) atomicExch(P.err, 1);
        }
    } else if (warp <= NC) {
        const int ctid = threadIdx.x - 32;
        long long k = 0;
        for (long long r = blockIdx.x; r < nrows; r += gridDim.x, ++k) {
            const int s = (int)(k % NS);
            const long long use = k / NS;
            if (!mbar_wait_bounded(&full[s], (unsigned)(use & 1), wait_limit(P))) {
                if (lane == 0 && P.err) atomicExch(P.err, 1);
                break;
            }
            const T* st = (const T*)(smem_raw + s * stage_bytes);
            Geo g;
            g.y = (int)(r % P.ny);
            g.z = (int)(r / P.ny);
            g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
            g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
            g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
            g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
            for (int x0 = 0; x0 < P.nx; x0 += NC * 32) {
                g.x = x0 + ctid;
                const bool inside = g.x < P.nx;
                if (!inside) g.x = 0;
                g.cell = g.x + P.nx * (g.y + P.ny * g.z);
                g.slot = g.cell;
                g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
                g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
                g.offsets(P);
                const uint32_t mk = inside ? P.mask[g.cell] : M_SOLID;
                const bool active = !(mk & M_SOLID);
                if (active) {
                    R f[Q];
                    auto src = [&](auto I) {
                        constexpr int i = I;
                        const int xs = L::c(i, 0) > 0 ? g.xm : (L::c(i, 0) < 0 ? g.xp : g.x);
                        return st + (i * P.nx + xs);
                    };
                    if (__all_sync(__activemask(), !(mk & M_LINKS))) {
                        sfor<Q>([&](auto I) { f[I] = S::cvt(*src(I)); });
                    } else {
                        // branch-free: a generic load from this node's own f*[ibar] in global
                        // memory (linked direction) or from the staged row in shared memory
                        sfor<Q>([&](auto I) {
                            constexpr int i = I, ib = L::qbar(i);
                            const T* p = ((mk >> ib) & 1u) ? (const T*)P.srcp[ib] + g.cell : src(I);
                            f[i] = S::cvt(*p);
                        });
                    }
                    process_cell<VS, COLL, ST, false, false>(P, g, mk, f, racc, NoScalarPull{});
                }
                constexpr int per = 32 / (int)sizeof(T);
                const unsigned fl = __ballot_sync(0xffffffffu, active);
                const unsigned grp = ((1u << per) - 1u) << ((lane / per) * per);
                if (inside && (mk & M_SOLID) && (fl & grp)) sfor<Q>([&](auto I) { S::st(P.dstp[I], g.cell, R(0)); });
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
        }
    }
    if (P.residual) step_partials<5>(racc, P, blockIdx.x);
}

// =================================================================== sparse sweep
// The lean path (periodic / no-slip faces, no scalar) over a fluid-only layout:
// the population planes hold the fluid nodes only, in node order (x fastest), so
// a porous medium moves no solid bytes and every lane updates a fluid node.
// Thread k updates fluid node k (cell list[k], link bits fmask[k]).  The pull
// source (x', y', z') = (x, y, z) - c_i, when fluid, is located through the row
// words of its row (y', z'): word w holds the fluid bits of x in [32w, 32w + 32)
// (.x) and the fluid index of the first fluid node at or after x = 32w (.y).
// With p = .y + popc(.x & bits below x), the fluid nodes of that row before x,
// the three directions sharing the row read idx(x - 1) = p - 1, idx(x) = p and
// idx(x + 1) = p + (bit x of the row); the periodic wrap in x (x' = nx - 1 from
// x = 0, x' = 0 from x = nx - 1) reads the first index of the next row, or of
// the row.  A sentinel row after the last holds .y = number of fluid nodes.
// Linked directions (solid source, or a folded no-slip wall) read the node's own
// f*[ibar], as the dense sweeps do.
// The sparse layout's pull source of direction i for fluid node k at g: the
// fluid slot of x - c_i (meaningful unless the link bit of ibar is set).  Word w
// of row (y', z') holds the fluid bits of x in [32w, 32w + 32) (.x) and the fluid
// index of the first fluid node at or after x = 32w (.y); with p = .y + popc(.x &
// bits below x), the three directions sharing the row read idx(x - 1) = p - 1,
// idx(x) = p and idx(x + 1) = p + (bit x of the row); the periodic wrap in x
// (WRAP: some lane of the warp is at a row end) reads the first index of the next
// row, or of the row.
template <class L, int i, bool WRAP>
__device__ __forceinline__ int sparse_source(const StepParams& P, const Geo& g, int k) {
    constexpr int D = L::D;
    constexpr int cx = L::c(i, 0), cy = L::c(i, 1), cz = D == 3 ? L::c(i, 2) : 0;
    const int W = P.rw_w;
    const int w = g.x >> 5, b = g.x & 31;
    const unsigned below = (1u << b) - 1u;
    const int row = g.y + P.ny * g.z;
    int idx;
    if constexpr (cy == 0 && cz == 0) {
        if constexpr (cx == 0) idx = k;
        else if constexpr (cx == 1)
            idx = (WRAP && g.x == 0) ? (int)P.rw[((unsigned)row + 1u) * (unsigned)W].y - 1 : k - 1;
        else idx = (WRAP && g.x == P.nx - 1) ? (int)P.rw[(unsigned)row * (unsigned)W].y : k + 1;
    } else {
        const int ys = cy > 0 ? g.ym : (cy < 0 ? g.yp : g.y);
        const int zs = cz > 0 ? g.zm : (cz < 0 ? g.zp : g.z);
        // row-word indices stay below (rows + 1) * W <= N / 32 + 2 rows + 1 < 2^32
        const unsigned r2 = (unsigned)ys + (unsigned)P.ny * (unsigned)zs;
        const uint2 v = P.rw[r2 * (unsigned)W + (unsigned)w];
        const int p = (int)v.y + __popc(v.x & below);
        if constexpr (cx == 0) idx = p;
        else if constexpr (cx == 1) idx = (WRAP && g.x == 0) ? (int)P.rw[(r2 + 1u) * (unsigned)W].y - 1 : p - 1;
        else idx = (WRAP && g.x == P.nx - 1) ? (int)P.rw[r2 * (unsigned)W].y : p + (int)((v.x >> b) & 1u);
    }
    return idx;
}

// In-place streaming (AA pattern) in the sparse layout: one population buffer A,
// plane i holding direction i per fluid slot.  The state between launches
// alternates between two placements of the post-collision populations f*:
//  - an even step (t even) reads f_i(x) = A[i][x] and stores f*_i(x) into the
//    node's own slot of the opposite plane, A[ibar][x];
//  - an odd step reads f_i(x) = A[ibar][x - c_i] (the value the neighbour x - c_i
//    stored there one step before) and stores f*_i(x) into A[i][x + c_i], where
//    the next even step of node x + c_i reads it.
// A neighbour that is solid (a link) turns both into the node's own slots:
// f_i(x) = A[i][x] (its own f*_ibar of the previous even step) and f*_i(x) goes
// to A[ibar][x] (read as f_ibar(x) by the next even step): half-way bounce-back,
// src/lib.rs:154-165.  In an odd step, the slot that direction i is read from is
// the slot that f*_ibar is stored to, and no other node touches it, so each slot
// is read once and written once per step and no step needs a second buffer.  The
// values pulled and the arithmetic are those of the A/B pull sweep, so both give
// the same bits; an even step needs no neighbour index, mask word or list entry.
//
// Push (SWEEP_PUSH, two buffers): the state between launches is the post-stream
// field f_t itself.  A step reads f_t(x) from the node's own slots (contiguous,
// no neighbour index on the load path), collides, and stores f*_i(x) into slot
// x + c_i of plane i of the other buffer (plane ibar of its own slot when x + c_i
// is solid), which is f_{t+1}.  The values and the arithmetic are again those of
// the pull sweep.
constexpr int SWEEP_PULL = 0, SWEEP_AA_EVEN = 1, SWEEP_AA_ODD = 2, SWEEP_PUSH = 3;
// A kernel form, not a streaming scheme: the pull sweep of a step without outputs
// (not the first step, no residual, moment write or observation), compiled
// without those branches so that its body is shorter.
constexpr int SWEEP_PULL_PLAIN = 4;

// One fluid node of the sparse sweep (k64 = its fluid index; lanes past the
// last fluid node only take part in the block reduction).  `e` and `mk` (its
// list entry and mask word) are read lazily: an in-place even step that writes
// no moments needs neither.
template <int VS, int COLL, int ST, int MODE>
__device__ __forceinline__ void sparse_node_at(const KParams<VS>& P, long long k64, const uint32_t* ep,
                                               const uint32_t* mp, double (&racc)[5]) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    using T = typename S::T;
    constexpr int Q = L::Q;
    const bool valid = k64 < P.nlist;
    const int k = valid ? (int)k64 : (int)(P.nlist - 1);
    // an in-place even step reads the node's own slots: coordinates only for outputs
    constexpr bool SIXTEEN = ST == ST_F16 || ST == ST_BF16;
    const bool need_geo = MODE != SWEEP_AA_EVEN || P.observe || P.residual || P.write_mom || (SIXTEEN && P.sround);
    Geo g;
    g.x = g.y = g.z = g.cell = 0;
    g.slot = k;
    uint32_t mk = 0;
    if (need_geo) {
        const uint32_t e = *ep;
        if (MODE != SWEEP_AA_EVEN) mk = *mp;
        if (P.packed) {   // coordinates packed at set-up: no division
            g.x = (int)(e & 2047u);
            g.y = (int)((e >> 11) & 2047u);
            g.z = (int)(e >> 22);
            g.cell = g.x + P.nx * (g.y + P.ny * g.z);
        } else {
            auto divq = [](int n, int d, double inv) {
                int q = (int)((double)n * inv);
                q -= ((long long)q * d > n);
                q += ((long long)(q + 1) * d <= n);
                return q;
            };
            g.cell = (int)e;
            const int row = divq(g.cell, P.nx, P.inv_nx);
            g.x = g.cell - row * P.nx;
            g.z = divq(row, P.ny, P.inv_ny);
            g.y = row - g.z * P.ny;
        }
        g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
        g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
        g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
        g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
        g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
        g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
    }
    if (!valid) return;
    R f[Q];
    auto pull_index = [&](auto I, auto WRAP) -> int {
        return sparse_source<L, int(I), decltype(WRAP)::value != 0>(P, g, k);
    };
    if constexpr (MODE == SWEEP_AA_EVEN) {
        sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], k); });
        process_cell_put<VS, COLL, ST, false, false>(P, g, mk, f, racc, [&](auto I, T v) {
            ((T*)P.dstp[L::qbar(I)])[k] = v;
        }, NoScalarPull{});
    } else if constexpr (MODE == SWEEP_PUSH) {
        sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], k); });
        auto body = [&](auto WRAP) {
            process_cell_put<VS, COLL, ST, false, false>(P, g, mk, f, racc, [&](auto I, T v) {
                constexpr int i = I, ib = L::qbar(i);
                if constexpr (i == 0) {
                    ((T*)P.dstp[0])[k] = v;
                } else {
                    // x + c_i is the pull source of direction ibar
                    const bool lk = (mk >> i) & 1u;
                    const int idx = sparse_source<L, ib, decltype(WRAP)::value != 0>(P, g, k);
                    ((T*)(lk ? P.dstp[ib] : P.dstp[i]))[lk ? k : idx] = v;
                }
            }, NoScalarPull{});
        };
        if (__any_sync(__activemask(), g.x == 0 || g.x == P.nx - 1)) body(IC<1>{});
        else body(IC<0>{});
    } else if constexpr (MODE == SWEEP_AA_ODD) {
        // element offsets from plane 0: read f_i there, store f*_ibar there (q * np < 2^32)
        unsigned off[Q];
        const unsigned np = (unsigned)P.np;
        auto load = [&](auto WRAP) {
            sfor<Q>([&](auto I) {
                constexpr int i = I, ib = L::qbar(i);
                if constexpr (i == 0) {
                    off[0] = (unsigned)k;
                } else {
                    const bool lk = (mk >> ib) & 1u;
                    const unsigned own = (unsigned)i * np + (unsigned)k;
                    off[i] = lk ? own : (unsigned)ib * np + (unsigned)pull_index(I, WRAP);
                }
                f[i] = S::cvt(((const T*)P.srcp[0])[off[i]]);
            });
        };
        if (__any_sync(__activemask(), g.x == 0 || g.x == P.nx - 1)) load(IC<1>{});
        else load(IC<0>{});
        process_cell_put<VS, COLL, ST, false, false>(P, g, mk, f, racc, [&](auto I, T v) {
            ((T*)P.dstp[0])[off[L::qbar(I)]] = v;
        }, NoScalarPull{});
    } else {
        if (MODE != SWEEP_PULL_PLAIN && P.first) {
            sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], k); });
        } else {
            // WRAP: the periodic wrap in x (x = 0 pulls from x = nx - 1 and x = nx - 1
            // from x = 0) needs the first index of a row; a warp with no lane at a row
            // end pulls without that code
            auto pull = [&](auto WRAP) {
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    const int idx = pull_index(I, WRAP);
                    const bool lk = (mk >> ib) & 1u;
                    f[i] = S::ld(lk ? P.srcp[ib] : P.srcp[i], lk ? k : idx);
                });
            };
            // (a warp-uniform split on the link bits as well measured 3-5 % slower: the
            // branch-free bounce-back select costs less than the extra code)
            if (__any_sync(__activemask(), g.x == 0 || g.x == P.nx - 1)) pull(IC<1>{});
            else pull(IC<0>{});
        }
        process_cell_at<VS, COLL, ST, false, false, MODE != SWEEP_PULL_PLAIN>(P, g, mk, f, racc, k, NoScalarPull{});
    }
}

template <int VS, int COLL, int ST, int MODE = SWEEP_PULL>
__device__ __forceinline__ void sparse_node(const KParams<VS>& P, long long k64, double (&racc)[5]) {
    const int k = k64 < P.nlist ? (int)k64 : (int)(P.nlist - 1);
    sparse_node_at<VS, COLL, ST, MODE>(P, k64, P.list + k, P.fmask + k, racc);
}

// One bulk prefetch of a global range into L2 (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// A node's first load (its list entry and mask word) would wait on DRAM, and
// every later load of the node waits for it.  Thread 0 of each block therefore
// prefetches into L2 the list entries and mask words of the block that starts
// about one wave later (block + pf_blocks), together with its own slots k0 ..
// k0 + n - 1 of the planes it pulls from its own rows (rest and +-x, whose sources
// lie within one slot of those).  A prefetch moves no extra DRAM bytes: the lines
// are read once either way.
template <int VS, int ST>
__device__ __forceinline__ void sparse_prefetch(const KParams<VS>& P) {
    using L = Lat<VS>;
    using T = typename Store<ST>::T;
    if (P.pf_blocks <= 0 || threadIdx.x != 0) return;
    // from a multiple of 16 slots (16-byte aligned for every element size)
    const long long k0 = (P.kbeg + ((long long)blockIdx.x + P.pf_blocks) * blockDim.x) & ~15ll;
    if (k0 >= P.nlist) return;
    const long long want = (long long)blockDim.x + 16;
    const long long n = P.nlist - k0 < want ? P.nlist - k0 : want;
    auto pf = [](const void* p, long long bytes) {   // 16-byte aligned start, size rounded down to 16
        const unsigned b = (unsigned)bytes & ~15u;
        if (b != 0 && ((uintptr_t)p & 15u) == 0) bulk_prefetch_l2(p, b);
    };
    pf(P.list + k0, n * 4);
    pf(P.fmask + k0, n * 4);
    if (!P.first) {
        sfor<L::Q>([&](auto I) {
            constexpr int i = I;
            if constexpr (L::c(i, 1) == 0 && (L::D == 2 || L::c(i, 2) == 0)) {
                pf((const T*)P.srcp[i] + k0, n * (long long)sizeof(T));
                // the scalars' planes of the same directions (compute type)
                for (int si = 0; si < P.nscalar; ++si)
                    pf((const typename Store<ST>::R*)P.sc[si].gsrc + (long long)i * P.np + k0,
                       n * (long long)sizeof(typename Store<ST>::R));
            }
        });
    }
}

// Blocks per SM of the sparse sweeps: 64 registers for the light ones.  (An
// in-place odd step, which keeps the Q slot offsets of its loads for its stores,
// spills 36 B at 64 registers; at 80 registers, three blocks per SM, it measured
// 520 us per launch on the 256^3 headline lattice against 450 us with the spill.)
template <int VS, int COLL, int ST, int MODE>
constexpr int sparse_blocks() {
    return light_kernel<VS, COLL, ST, false>() == 2 ? 4 : 2;
}

template <int VS, int COLL, int ST, int MODE>
__global__ void __launch_bounds__(256, (sparse_blocks<VS, COLL, ST, MODE>())) k_step_sparse(const KParams<VS> P) {
    if (gated_off(P)) return;
    // an in-place even step reads only its own contiguous slots: nothing to prefetch
    if (MODE != SWEEP_AA_EVEN || P.observe || P.residual || P.write_mom || ((ST == ST_F16 || ST == ST_BF16) && P.sround))
        sparse_prefetch<VS, ST>(P);
    double racc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const long long k = P.kbeg + blockIdx.x * (long long)blockDim.x + threadIdx.x;
    sparse_node<VS, COLL, ST, MODE>(P, k < P.kend ? k : P.nlist, racc);   // nlist: no update
    if (MODE != SWEEP_PULL_PLAIN && P.residual && !P.observe) step_partials<5>(racc, P, blockIdx.x);
}

// =================================================================== sparse sweep, faces and scalar
// The sparse layout for lattices with explicit face BCs and/or a passive scalar
// (a packed bed: Zou-He or moving-wall inlet, anti-bounce-back outlet, scalar
// with Langmuir adsorption).  Thread k updates fluid node k as k_step_sparse
// does, with two population buffers; the scalar populations live in the same
// fluid slots and are pulled through the same source indices.  Face nodes run
// apply_faces on their own slots; the nodes of a scalar outflow face are left to
// the face pass (P.face_pass: one thread per position of face fp_face), which
// finds a node's fluid slot through the row words.  Per-node side arrays
// (adsorbed amount, previous scalar value, residual moments, face layers) stay
// indexed by node, as in the dense layout.
// Blocks per SM (ptxas, D3Q19 / D2Q9 BGK and TRT): the FP32 and 16-bit sweeps,
// with or without scalars, fit 80 registers (three blocks); FP64, D3Q27 and MRT
// keep 128 (two), below which they spill.  The scalars' pull reuses the
// momentum's source slots from shared memory, and their residual terms wait
// there for the block reduction, so neither is held in registers across the
// momentum collision.
template <int VS, int COLL, int ST, bool SCALAR>
constexpr int sparse_fs_blocks() {
    return (ST == ST_F64 || VS == VS_D3Q27 || COLL == COLL_MRT) ? 2 : 3;
}

// The node of thread `tid` in a launch of k_step_sparse_fs: its coordinates,
// fluid slot k and mask word (face pass: the tid-th position of face fp_face).
template <bool FACEBC>
__device__ __forceinline__ bool sparse_fs_node(const StepParams& P, long long tid, Geo& g, int& k, uint32_t& mk) {
    bool valid;
    mk = M_SOLID;
    k = 0;
    if (FACEBC && P.face_pass) {
        const int F = P.fp_face;
        valid = tid < P.pb_plane[F];
        const long long pp = valid ? tid : 0;
        if (F < 2) { g.x = F == 0 ? 0 : P.nx - 1; g.y = (int)(pp % P.ny); g.z = (int)(pp / P.ny); }
        else if (F < 4) { g.y = F == 2 ? 0 : P.ny - 1; g.x = (int)(pp % P.nx); g.z = (int)(pp / P.nx); }
        else { g.z = F == 4 ? 0 : P.nz - 1; g.x = (int)(pp % P.nx); g.y = (int)(pp / P.nx); }
        g.cell = g.x + P.nx * (g.y + P.ny * g.z);
        mk = valid ? P.mask[g.cell] : M_SOLID;
        valid = valid && !(mk & M_SOLID) && (mk & M_SKIP);
        if (valid) {
            const uint2 v = P.rw[(unsigned)(g.y + P.ny * g.z) * (unsigned)P.rw_w + (unsigned)(g.x >> 5)];
            k = (int)v.y + __popc(v.x & ((1u << (g.x & 31)) - 1u));
        }
    } else {
        const long long k64 = P.kbeg + tid;
        valid = k64 < P.kend;
        k = valid ? (int)k64 : (int)(P.kend - 1);
        const uint32_t e = P.list[k];
        mk = P.fmask[k];
        if (P.packed) {
            g.x = (int)(e & 2047u);
            g.y = (int)((e >> 11) & 2047u);
            g.z = (int)(e >> 22);
            g.cell = g.x + P.nx * (g.y + P.ny * g.z);
        } else {
            auto divq = [](int n, int d, double inv) {
                int q = (int)((double)n * inv);
                q -= ((long long)q * d > n);
                q += ((long long)(q + 1) * d <= n);
                return q;
            };
            g.cell = (int)e;
            const int row = divq(g.cell, P.nx, P.inv_nx);
            g.x = g.cell - row * P.nx;
            g.z = divq(row, P.ny, P.inv_ny);
            g.y = row - g.z * P.ny;
        }
        if (FACEBC) valid = valid && !(mk & M_SKIP);
    }
    g.slot = k;
    g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
    g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
    g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
    g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
    g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
    g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
    return valid;
}

template <int VS, int COLL, int ST, bool FACEBC, bool SCALAR>
__global__ void __launch_bounds__(256, (sparse_fs_blocks<VS, COLL, ST, SCALAR>())) k_step_sparse_fs(const KParams<VS> P) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    constexpr int Q = L::Q, D = L::D;
    // the pull's source slots for the scalars, [direction][thread]: the fluid slot,
    // or ~k for a linked direction (the node's own slot k of plane ibar)
    __shared__ int sidx[SCALAR ? Q * 256 : 1];
    // with scalars, the squared residual terms of this block's nodes,
    // [rho, u_0..u_2, scalar 0..][thread], kept out of registers until the block
    // reduction
    __shared__ double sres[SCALAR ? (4 + NSMAX) * 256 : 1];
    if (gated_off(P)) return;
    const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int t = threadIdx.x;
    Geo g;
    uint32_t mk;
    int k;
    if (!(FACEBC && P.face_pass)) sparse_prefetch<VS, ST>(P);
    const bool valid = sparse_fs_node<FACEBC>(P, tid, g, k, mk);
    double racc[5] = {};
    if (valid) {
        R f[Q];
        R u[3], uu;
        if (P.first) {
            sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], k); });
        } else {
            // pull + inner bounce-back (src/lib.rs:141-165)
            auto pull = [&](auto WRAP) {
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    const int idx = sparse_source<L, i, decltype(WRAP)::value != 0>(P, g, k);
                    const bool lk = (mk >> ib) & 1u;
                    f[i] = S::ld(lk ? P.srcp[ib] : P.srcp[i], lk ? k : idx);
                    if constexpr (SCALAR) sidx[i * 256 + t] = lk ? ~k : idx;
                });
            };
            // a lane of the warp at a row end: the periodic-wrap form of the source index
            if (__any_sync(__activemask(), g.x == 0 || g.x == P.nx - 1)) pull(IC<1>{});
            else pull(IC<0>{});
        }
        auto put = [&](auto I, typename S::T v) { ((typename S::T*)P.dstp[I])[k] = v; };
        if constexpr (SCALAR) momentum_cell<VS, COLL, ST, FACEBC>(
            P, g, mk, f, [&](auto J, double v) { sres[int(J) * 256 + t] = v; }, put, u, uu);
        else momentum_cell<VS, COLL, ST, FACEBC>(P, g, mk, f, [&](auto J, double v) { racc[int(J)] += v; }, put, u, uu);
        if constexpr (SCALAR) {
            // the scalars: the momentum's source slots (a linked direction reads the
            // node's own g*[ib]) and inner BC (src/passive_scalar/lattice.rs:274-297).
            // The node's coordinates are taken again, so none stay live across the
            // momentum collision.
            Geo gq;
            int kq;
            uint32_t mq;
            sparse_fs_node<FACEBC>(P, tid, gq, kq, mq);
            auto gpull = [&](int si, R* gg) {
                const ScalarParams& sc = P.sc[si];
                const R* gs = (const R*)sc.gsrc;
                const long long np = P.np;
                if (P.first) {
                    sfor<Q>([&](auto I) { gg[I] = gs[I * np + kq]; });
                    return;
                }
                sfor<Q>([&](auto I) {
                    constexpr int i = I, ib = L::qbar(i);
                    const int e = sidx[i * 256 + t];
                    const bool lk = e < 0;
                    const R v = gs[(lk ? ib : i) * np + (lk ? ~e : e)];
                    if (lk && sc.inner != 1) {   // InnerAntiBounceBack: -g*[ib] + 2 w C_solid (ps/node.rs:281-294)
                        R cs = R(sc.c_solid);
                        if (sc.c_init) {   // the solid neighbour's initial value (periodic)
                            const int xs = L::c(i, 0) > 0 ? gq.xm : (L::c(i, 0) < 0 ? gq.xp : gq.x);
                            const int ys = L::c(i, 1) > 0 ? gq.ym : (L::c(i, 1) < 0 ? gq.yp : gq.y);
                            const int zs = D == 3 ? (L::c(i, 2) > 0 ? gq.zm : (L::c(i, 2) < 0 ? gq.zp : gq.z)) : 0;
                            cs = R(sc.c_init[xs + (long long)P.nx * (ys + (long long)P.ny * zs)]);
                        }
                        gg[i] = -v + R(2) * R(L::w(ib)) * cs;
                    } else {
                        gg[i] = v;   // pulled, or InnerBounceBack
                    }
                });
            };
            scalar_cells<VS, ST, FACEBC>(P, gq, mq, u, uu, gpull,
                                         [&](int si, double v) { sres[(4 + si) * 256 + t] = v; });
        }
    }
    if (P.residual && !P.observe) {
        if constexpr (SCALAR) {
            double rall[4 + NSMAX];
            sfor<4 + NSMAX>([&](auto J) {
                const bool has = valid && (int(J) < 1 + D || (int(J) >= 4 && int(J) < 4 + P.nscalar));
                rall[J] = has ? sres[int(J) * 256 + t] : 0.0;
            });
            step_partials<4 + NSMAX>(rall, P, blockIdx.x);
        } else {
            step_partials<5>(racc, P, blockIdx.x);
        }
    }
}

// =================================================================== z-slab halos
// A z-slab domain holds its owned planes plus one ghost plane below and above.
// After a step the owned boundary plane's populations that leave the slab (c_z
// = -1 at the bottom, +1 at the top) are packed into a contiguous buffer for the
// neighbour, and the neighbour's buffer is unpacked into the ghost plane, whose
// entering directions (c_z = +1 below, -1 above) the next step pulls.
// planes[k] = element pointer of direction dirs[k] at the plane's first node.
// In the sparse layout a plane's fluid nodes are `count` consecutive slots (the
// ghost plane holds the same fluid nodes as the neighbour's boundary plane); the
// buffer keeps the dense stride `plane` per direction either way.
struct HaloPlanes {
    void* planes[9];
    int nd;
    long long plane;   // buffer elements per direction (nodes per plane)
    long long count;   // slots copied per direction (plane, or the plane's fluid nodes)
};
template <class T>
__global__ void k_halo_pack(HaloPlanes H, T* buf) {
    const long long n = (long long)H.nd * H.count;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / H.count);
        const long long j = i - k * H.count;
        buf[k * H.plane + j] = ((const T*)H.planes[k])[j];
    }
}
template <class T>
__global__ void k_halo_unpack(HaloPlanes H, const T* buf) {
    const long long n = (long long)H.nd * H.count;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i / H.count);
        const long long j = i - k * H.count;
        ((T*)H.planes[k])[j] = buf[k * H.plane + j];
    }
}

}  // namespace lbf
