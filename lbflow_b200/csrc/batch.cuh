// batch.cuh -- device-side state of a batch of domains and the launchers of the
// batched sweep (kernels in batch_kernels.cuh, instantiated by batch_<vs>.cu).
#pragma once

#include <cstddef>

#include "kernels.cuh"

namespace lbf {

// One domain of a batch, in device memory.  The batched sweep reads it; the
// finalize kernel that ends every chunk of k steps evaluates the stop rule of
// lbf_domain_run (src/momentum/lattice.rs:396-418) on the device and advances t0.
struct BatchState {
    long long t0;       // time step of chunk step 0
    long long last_t;   // last time step to run: max_iterations + 1
    long long block0;   // first block of this domain in the batched launch
    long long done_t;   // last time step run once stopped, -1 while running
    long long res_t;    // time step of res[] (-1 = none yet)
    int k;              // residual interval (chunk length)
    int status;         // 0 running, 1 converged, 2 max_iterations, 3 non-finite residual
    int ns;             // scalars (their residuals are accumulators 4 .. 4 + ns - 1)
    int d;
    double tol[3];      // density, velocity, scalar tolerances
    double res[8];      // residuals of res_t: rho, u_0.., scalars from 4, as k_finalize writes them
};

// Launches one time step (chunk step j) of every domain in a batch group: all
// domains of the group share the velocity set VS, the collision, the storage
// and the explicit-face flag.  `tab` holds one KParams<VS> per domain (laid out
// for an even time step), `blk` maps each of the nblocks blocks to its domain.
// `sparse`: the group's domains use the fluid-only layout.
template <int VS>
cudaError_t launch_step_batch(int coll, int st, bool facebc, bool sparse, const void* tab, const BatchState* bs,
                              const int* blk, int j, unsigned nblocks, cudaStream_t s);
// All k steps of a chunk for every domain of a group in one cooperative launch
// (grid barriers between the steps); the same results as k launch_step_batch calls.
template <int VS>
cudaError_t launch_batch_chunk(int coll, int st, bool facebc, bool sparse, const void* tab, const BatchState* bs,
                               const int* blk, int k, unsigned nblocks, cudaStream_t s);
// Residuals + stop rule + t0 += k for each of the n domains of a group.
template <int VS>
cudaError_t launch_batch_finalize(const void* tab, BatchState* bs, int n, cudaStream_t s);

constexpr int BATCH_BLOCK = 256;
static_assert(offsetof(BatchState, t0) == offsetof(GateView, t0) && offsetof(BatchState, last_t) ==
                  offsetof(GateView, last_t) && offsetof(BatchState, done_t) == offsetof(GateView, done_t),
              "GateView mirrors the leading fields of BatchState");
// Members with at least this many nodes (fluid nodes in the sparse layout) run
// their own single-domain sweep inside the chunk graph: they fill the GPU alone,
// and the single-domain kernels read their parameters from the constant bank.
constexpr long long SOLO_UNITS = 1ll << 19;

}  // namespace lbf
