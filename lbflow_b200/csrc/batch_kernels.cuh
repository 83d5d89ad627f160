// batch_kernels.cuh -- the batched sweep: many domains, one launch per time step.
//
// A serving mix holds many small lattices (D2Q9 cavities of 64^2..1024^2 nodes,
// D3Q19 channels of 32^3..160^3).  One launch per domain and step leaves most of
// the 148 SMs idle and makes the step launch-bound, so the domains of one kernel
// configuration are laid end to end in one grid: block b belongs to domain
// blk[b] and covers 256 of its nodes in node order.  Each domain's parameters
// are stored once in device memory, laid out for an even time step; a block
// copies them to shared memory and completes them for its domain's time step
// (A/B parity, first step, residual and moment flags).  A domain that has
// stopped, or whose next step is past its last one, costs its blocks one load
// and an early exit.  The per-node work is the same code as the single-domain
// sweep (process_cell), so a domain computes the same values alone and in a
// batch.  Domains with scalars or the central-moment collision run their own
// single-domain sweep inside the batch's chunk graph instead.  Domains in the
// sparse (fluid-only) layout form their own groups, swept by k_step_batch_sparse.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>

#include "batch.cuh"

namespace lbf {

template <int VS, int COLL>
__device__ __forceinline__ void batch_params(KParams<VS>& Ps, const KParams<VS>* tab, int e, long long t, int k) {
    constexpr bool LAM = VS == VS_D3Q27 && COLL == COLL_MRT;
    constexpr int NW = (int)((LAM ? sizeof(KParams<VS>) : sizeof(StepParams)) / 8);
    static_assert(sizeof(StepParams) % 8 == 0 && sizeof(KParams<VS>) % 8 == 0, "8-byte copy");
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(tab + e);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&Ps);
    for (int i = threadIdx.x; i < NW; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    if (threadIdx.x == 0) {
        if (t & 1) {   // odd step: the A/B buffers and the double-buffered layers swap roles
            for (int i = 0; i < Lat<VS>::Q; ++i) {
                const void* a = Ps.srcp[i];
                Ps.srcp[i] = Ps.dstp[i];
                Ps.dstp[i] = const_cast<void*>(a);
            }
            for (int f = 0; f < 6; ++f) {
                const void* a = Ps.pb_src[f];
                Ps.pb_src[f] = Ps.pb_dst[f];
                Ps.pb_dst[f] = const_cast<void*>(a);
            }
            const void* m = Ps.mom_prev;
            Ps.mom_prev = Ps.mom_cur;
            Ps.mom_cur = const_cast<void*>(m);
        }
        Ps.first = t == 0;
        if (Ps.sweep_mode == SWEEP_AA_EVEN || Ps.sweep_mode == SWEEP_AA_ODD)
            Ps.sweep_mode = (t & 1) ? SWEEP_AA_ODD : SWEEP_AA_EVEN;
        Ps.tstep = (unsigned)t;
        Ps.residual = k > 0 && t % k == 0;
        Ps.write_mom = k > 0 && (t % k == 0 || (t + 1) % k == 0);
    }
    __syncthreads();
}

// Block vb of the batched dense sweep, chunk step j (Ps: the block's shared copy
// of its domain's parameters).
template <int VS, int COLL, int ST, bool FACEBC>
__device__ __forceinline__ void batch_dense_block(const KParams<VS>* __restrict__ tab,
                                                  const BatchState* __restrict__ bs, const int* __restrict__ blk,
                                                  int vb, int j, KParams<VS>& Ps) {
    using L = Lat<VS>;
    using S = Store<ST>;
    using R = typename S::R;
    using T = typename S::T;
    constexpr int Q = L::Q, D = L::D;
    const int e = blk[vb];
    const long long t = bs[e].t0 + j;
    if (bs[e].done_t >= 0 || t > bs[e].last_t) return;   // uniform over the block
    batch_params<VS, COLL>(Ps, tab, e, t, bs[e].k);
    const KParams<VS>& P = Ps;

    const long long c64 = (long long)(vb - bs[e].block0) * BATCH_BLOCK + threadIdx.x;
    const bool inside = c64 < P.N;
    Geo g;
    g.cell = inside ? (int)c64 : 0;
    g.slot = g.cell;
    {
        // coordinates by a double-precision reciprocal plus a +-1 correction
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
    }
    g.xm = g.x == 0 ? P.nx - 1 : g.x - 1;
    g.xp = g.x == P.nx - 1 ? 0 : g.x + 1;
    g.ym = g.y == 0 ? P.ny - 1 : g.y - 1;
    g.yp = g.y == P.ny - 1 ? 0 : g.y + 1;
    g.zm = g.z == 0 ? P.nz - 1 : g.z - 1;
    g.zp = g.z == P.nz - 1 ? 0 : g.z + 1;
    g.offsets(P);

    const uint32_t mk = inside ? P.mask[g.cell] : M_SOLID;
    bool active = !(mk & M_SOLID);
    if constexpr (FACEBC) active = active && !(mk & M_SKIP);
    double racc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (active) {
        R f[Q];
        if (P.first) {
            sfor<Q>([&](auto I) { f[I] = S::ld(P.srcp[I], g.cell); });
        } else if (__all_sync(__activemask(), !(mk & M_LINKS))) {
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
        process_cell<VS, COLL, ST, FACEBC, false>(P, g, mk, f, racc, NoScalarPull{});
    }
    if (!P.first) {
        // solid nodes sharing a 32-byte sector with a fluid node store zeros (full-sector stores)
        constexpr int per = 32 / (int)sizeof(T);
        const unsigned fl = __ballot_sync(__activemask(), active);
        const int lane = threadIdx.x & 31;
        const unsigned grp = (per >= 32 ? 0xffffffffu : ((1u << per) - 1u) << ((lane / per) * per));
        if (inside && (mk & M_SOLID) && (fl & grp)) sfor<Q>([&](auto I) { S::st(P.dstp[I], g.cell, R(0)); });
    }
    if (P.residual) step_partials<5>(racc, P, vb - bs[e].block0);
}

template <int VS, int COLL, int ST, bool FACEBC>
__global__ void __launch_bounds__(BATCH_BLOCK, 2 * light_kernel<VS, COLL, ST, false>())
    k_step_batch(const KParams<VS>* __restrict__ tab, const BatchState* __restrict__ bs, const int* __restrict__ blk,
                 int j) {
    __shared__ KParams<VS> Ps;
    batch_dense_block<VS, COLL, ST, FACEBC>(tab, bs, blk, blockIdx.x, j, Ps);
}

// The batched sweep over domains in the sparse (fluid-only) layout: block b
// covers 256 fluid nodes of domain blk[b], in fluid order.
template <int VS, int COLL, int ST>
__device__ __forceinline__ void batch_sparse_block(const KParams<VS>* __restrict__ tab,
                                                   const BatchState* __restrict__ bs, const int* __restrict__ blk,
                                                   int vb, int j, KParams<VS>& Ps) {
    const int e = blk[vb];
    const long long t = bs[e].t0 + j;
    if (bs[e].done_t >= 0 || t > bs[e].last_t) return;   // uniform over the block
    batch_params<VS, COLL>(Ps, tab, e, t, bs[e].k);
    double racc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const long long k = (long long)(vb - bs[e].block0) * BATCH_BLOCK + threadIdx.x;
    // the sweep mode is uniform over the block (one domain per block)
    if (Ps.sweep_mode == SWEEP_AA_EVEN) sparse_node<VS, COLL, ST, SWEEP_AA_EVEN>(Ps, k, racc);
    else if (Ps.sweep_mode == SWEEP_AA_ODD) sparse_node<VS, COLL, ST, SWEEP_AA_ODD>(Ps, k, racc);
    else if (Ps.sweep_mode == SWEEP_PUSH) sparse_node<VS, COLL, ST, SWEEP_PUSH>(Ps, k, racc);
    else sparse_node<VS, COLL, ST, SWEEP_PULL>(Ps, k, racc);
    if (Ps.residual) step_partials<5>(racc, Ps, vb - bs[e].block0);
}

template <int VS, int COLL, int ST>
__global__ void __launch_bounds__(BATCH_BLOCK, 2 * light_kernel<VS, COLL, ST, false>())
    k_step_batch_sparse(const KParams<VS>* __restrict__ tab, const BatchState* __restrict__ bs,
                        const int* __restrict__ blk, int j) {
    __shared__ KParams<VS> Ps;
    batch_sparse_block<VS, COLL, ST>(tab, bs, blk, blockIdx.x, j, Ps);
}

// All k steps of a chunk in one cooperative launch over the group's packed block
// index: block b of the grid takes blocks b, b + gridDim.x, .. of each step, and
// a grid barrier separates the steps (a domain's step j + 1 reads what all its
// blocks wrote in step j).  The grid is at most what fits on the GPU at once,
// which the cooperative launch checks, so every barrier completes.  A domain
// computes the same values as in the one-launch-per-step form: the same blocks,
// the same per-node code.
template <int VS, int COLL, int ST, bool FACEBC, bool SPARSE>
__global__ void __launch_bounds__(BATCH_BLOCK, 2 * light_kernel<VS, COLL, ST, false>())
    k_step_batch_chunk(const KParams<VS>* __restrict__ tab, const BatchState* __restrict__ bs,
                       const int* __restrict__ blk, int nvb, int k) {
    __shared__ KParams<VS> Ps;
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    for (int j = 0; j < k; ++j) {
        for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
            __syncthreads();   // the previous block's parameters are no longer read
            if constexpr (SPARSE) batch_sparse_block<VS, COLL, ST>(tab, bs, blk, vb, j, Ps);
            else batch_dense_block<VS, COLL, ST, FACEBC>(tab, bs, blk, vb, j, Ps);
        }
        if (j + 1 < k) grid.sync();
    }
}

template <int VS, int COLL, int ST, bool FACEBC, bool SPARSE>
cudaError_t launch_batch_chunk_k(const void* tab, const BatchState* bs, const int* blk, int k, unsigned nvb,
                                 cudaStream_t s) {
    auto kern = k_step_batch_chunk<VS, COLL, ST, FACEBC, SPARSE>;
    int per = 0, dev = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, BATCH_BLOCK, 0);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    const unsigned grid = (unsigned)std::min<long long>((long long)nvb, (long long)per * sms);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(BATCH_BLOCK);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, (const KParams<VS>*)tab, bs, blk, (int)nvb, k);
}

// One block of 256 threads per domain: residuals of the chunk's last step (its
// residual step), the stop rule of lbf_domain_run, and t0 += k.
template <int VS>
__global__ void k_batch_finalize(const KParams<VS>* __restrict__ tab, BatchState* __restrict__ bs, int n) {
    const int e = blockIdx.x;
    if (e >= n) return;
    BatchState& s = bs[e];
    if (s.done_t >= 0) return;
    const int k = s.k;
    const long long t_end = s.t0 + k - 1;
    const bool ran = t_end <= s.last_t;
    const double* accum = tab[e].accum;
    const long long stride = tab[e].accum_stride, nslots = tab[e].res_slots;
    __shared__ double r[8];
    __shared__ double part[256];
    // the per-block partials of the residual step, summed in slot order
    const int nacc = s.ns > 0 ? 4 + s.ns : 5;
    for (int a = 0; a < nacc; ++a) {
        double sum = 0.0;
        for (long long jj = threadIdx.x; jj < nslots; jj += blockDim.x) sum += accum[a * stride + jj];
        part[threadIdx.x] = sum;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) r[a] = sqrt(part[0]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (ran) {
            for (int i = 0; i < nacc; ++i) s.res[i] = r[i];
            s.res_t = t_end;
        }
        const bool max_stop = t_end >= s.last_t;   // a step t > max_iterations ran
        if (ran && !max_stop && t_end > 10) {
            bool conv = r[0] <= s.tol[0];
            for (int i = 0; i < s.d; ++i) conv = conv && r[1 + i] <= s.tol[1];
            for (int i = 0; i < s.ns; ++i) conv = conv && r[4 + i] <= s.tol[2];
            if (!isfinite(r[0])) {
                s.status = 3;
                s.done_t = t_end;
            } else if (conv) {
                s.status = 1;
                s.done_t = t_end;
            }
        }
        if (s.done_t < 0 && max_stop) {
            s.status = 2;
            s.done_t = s.last_t;
        }
        s.t0 += k;
    }
}

#define LBF_BATCH_CASE(C_, S_, FB_)                                                                \
    if (coll == C_ && st == S_ && facebc == FB_ && !sparse) {                                      \
        k_step_batch<VS, C_, S_, FB_><<<nblocks, BATCH_BLOCK, 0, s>>>((const KParams<VS>*)tab, bs, blk, j); \
        return cudaGetLastError();                                                                 \
    }
#define LBF_BATCH_SPARSE_CASE(C_, S_)                                                              \
    if (coll == C_ && st == S_ && sparse) {                                                        \
        k_step_batch_sparse<VS, C_, S_><<<nblocks, BATCH_BLOCK, 0, s>>>((const KParams<VS>*)tab, bs, blk, j); \
        return cudaGetLastError();                                                                 \
    }
#define LBF_BATCH_CHUNK_CASE(C_, S_, FB_, SP_)                                                     \
    if (coll == C_ && st == S_ && facebc == FB_ && sparse == SP_)                                  \
        return launch_batch_chunk_k<VS, C_, S_, FB_, SP_>(tab, bs, blk, k, nblocks, s);
#define LBF_BATCH_ST(C_, S_) LBF_BATCH_CASE(C_, S_, false) LBF_BATCH_CASE(C_, S_, true) LBF_BATCH_SPARSE_CASE(C_, S_)
#define LBF_BATCH_CHUNK_ST(C_, S_) LBF_BATCH_CHUNK_CASE(C_, S_, false, false) LBF_BATCH_CHUNK_CASE(C_, S_, true, false) \
    LBF_BATCH_CHUNK_CASE(C_, S_, false, true)
#define LBF_BATCH_CHUNK_COLL(C_) LBF_BATCH_CHUNK_ST(C_, ST_F64) LBF_BATCH_CHUNK_ST(C_, ST_F32) \
    LBF_BATCH_CHUNK_ST(C_, ST_F16) LBF_BATCH_CHUNK_ST(C_, ST_BF16)
#define LBF_BATCH_COLL(C_) LBF_BATCH_ST(C_, ST_F64) LBF_BATCH_ST(C_, ST_F32) LBF_BATCH_ST(C_, ST_F16) LBF_BATCH_ST(C_, ST_BF16)

#define LBF_INSTANTIATE_BATCH(VS_)                                                                 \
    template <>                                                                                    \
    cudaError_t launch_step_batch<VS_>(int coll, int st, bool facebc, bool sparse, const void* tab,     \
                                       const BatchState* bs, const int* blk, int j, unsigned nblocks, \
                                       cudaStream_t s) {                                            \
        constexpr int VS = VS_;                                                                    \
        if (nblocks == 0) return cudaSuccess;                                                      \
        LBF_BATCH_COLL(COLL_BGK) LBF_BATCH_COLL(COLL_TRT) LBF_BATCH_COLL(COLL_MRT)                 \
        return cudaErrorInvalidValue;                                                              \
    }                                                                                              \
    template <>                                                                                    \
    cudaError_t launch_batch_chunk<VS_>(int coll, int st, bool facebc, bool sparse, const void* tab,    \
                                        const BatchState* bs, const int* blk, int k, unsigned nblocks,  \
                                        cudaStream_t s) {                                           \
        constexpr int VS = VS_;                                                                    \
        if (nblocks == 0 || k == 0) return cudaSuccess;                                            \
        LBF_BATCH_CHUNK_COLL(COLL_BGK) LBF_BATCH_CHUNK_COLL(COLL_TRT) LBF_BATCH_CHUNK_COLL(COLL_MRT) \
        return cudaErrorInvalidValue;                                                              \
    }                                                                                              \
    template <>                                                                                    \
    cudaError_t launch_batch_finalize<VS_>(const void* tab, BatchState* bs, int n, cudaStream_t s) { \
        if (n == 0) return cudaSuccess;                                                            \
        k_batch_finalize<VS_><<<n, 256, 0, s>>>((const KParams<VS_>*)tab, bs, n);                  \
        return cudaGetLastError();                                                                 \
    }

}  // namespace lbf
