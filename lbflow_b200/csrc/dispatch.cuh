// dispatch.cuh -- host-side launchers, one translation unit per velocity set
// (step_d2q9.cu, step_d3q19.cu, step_d3q27.cu instantiate them).
#pragma once

#include <algorithm>

#include "aux_kernels.cuh"

namespace lbf {

struct Launch {
    dim3 grid, block;
    cudaStream_t stream;
};

template <int VS>
cudaError_t launch_step(int coll, int st, bool facebc, bool scalar, bool stage, const StepParams& base,
                        const double* lam, const Launch& L);
// Dynamic shared memory of the staged kernel: Q rows (+ Q scalar rows) + mbarrier.
inline size_t stage_smem(int q, long long nx, size_t tbytes, size_t rbytes, bool scalar) {
    return (size_t)q * nx * (tbytes + (scalar ? rbytes : 0)) + 16;
}
template <int VS>
cudaError_t launch_init(int st, bool scalar, const StepParams& P, const InitParams& I, void* const* pb,
                        const Launch& L);
template <int VS>
cudaError_t launch_setup(const SetupParams& S, const Launch& L);

template <int VS>
inline void fill_lam(KParams<VS>&, const double*) {}
inline void fill_lam(KParams<VS_D3Q27>& kp, const double* lam) {
    for (int k = 0; k < 27 * 27; ++k) {
        kp.lam64[k] = lam ? lam[k] : 0.0;
        kp.lam32[k] = float(kp.lam64[k]);
    }
}

#define LBF_STEP_CASE(C_, S_, FB_, SC_)                                                                   \
    if (coll == C_ && st == S_ && facebc == FB_ && scalar == SC_) {                                        \
        if (stage) {                                                                                       \
            const size_t sm = stage_smem(Lat<VS>::Q, kp.nx, sizeof(typename Store<S_>::T),                \
                                         sizeof(typename Store<S_>::R), SC_);                              \
            static size_t sm_set = 0;                                                                      \
            if (sm > 48 * 1024 && sm > sm_set) {                                                           \
                cudaError_t e_ = cudaFuncSetAttribute(k_step<VS, C_, S_, FB_, SC_, true>,                  \
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
                if (e_ != cudaSuccess) return e_;                                                          \
                sm_set = sm;                                                                               \
            }                                                                                              \
            k_step<VS, C_, S_, FB_, SC_, true><<<L.grid, L.block, sm, L.stream>>>(kp);                     \
        } else {                                                                                           \
            k_step<VS, C_, S_, FB_, SC_, false><<<L.grid, L.block, 0, L.stream>>>(kp);                     \
        }                                                                                                  \
        return cudaGetLastError();                                                                         \
    }
#define LBF_STEP_ST(C_, S_)            \
    LBF_STEP_CASE(C_, S_, false, false) \
    LBF_STEP_CASE(C_, S_, true, false)
#define LBF_STEP_COLL(C_)                                                                     \
    LBF_STEP_ST(C_, ST_F64) LBF_STEP_ST(C_, ST_F32) LBF_STEP_ST(C_, ST_F16) LBF_STEP_ST(C_, ST_BF16) \
    LBF_STEP_CASE(C_, ST_F64, true, true) LBF_STEP_CASE(C_, ST_F32, true, true)

// Pipelined sweep (lean path only); returns cudaErrorNotSupported when the shape
// does not allow it (the caller then uses k_step).
template <int VS, int COLL>
cudaError_t launch_step_pipe(int st, const StepParams& base, const double* lam, int stages, int nc,
                             cudaStream_t stream);

template <int VS, int COLL, int ST>
cudaError_t launch_pipe_st(const KParams<VS>& kp, int stages, int nc, cudaStream_t stream) {
    using T = typename Store<ST>::T;
    const size_t smem = (size_t)stages * Lat<VS>::Q * kp.nx * sizeof(T) + 2 * stages * sizeof(uint64_t);
    const int threads = 32 * (1 + nc);
    static size_t smem_set = 0;
    if (smem > smem_set) {
        cudaError_t e = cudaFuncSetAttribute(k_step_pipe<VS, COLL, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        smem_set = smem;
    }
    int per_sm = 0, dev = 0, sms = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_pipe<VS, COLL, ST>, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorNotSupported;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long rows = (long long)kp.ny * kp.nz;
    const long long blocks = std::min<long long>(rows, (long long)per_sm * sms);
    k_step_pipe<VS, COLL, ST><<<(unsigned)blocks, threads, smem, stream>>>(kp);
    return cudaGetLastError();
}

// Compacted sweep over the domain's work list (lean path).
template <int VS, int COLL>
cudaError_t launch_step_list(int st, const StepParams& base, const double* lam, cudaStream_t stream);

template <int VS, int COLL, int ST>
cudaError_t launch_list_st(const KParams<VS>& kp, cudaStream_t stream) {
    const unsigned blocks = (unsigned)((kp.nlist + 255) / 256);
    if (blocks == 0) return cudaSuccess;
    k_step_list<VS, COLL, ST><<<blocks, 256, 0, stream>>>(kp);
    return cudaGetLastError();
}

// Sparse (fluid-only) sweep (lean path).
template <int VS, int COLL>
cudaError_t launch_step_sparse(int st, const StepParams& base, const double* lam, cudaStream_t stream);

template <int VS, int COLL, int ST>
cudaError_t launch_sparse_st(KParams<VS>& kp, cudaStream_t stream) {
    const unsigned blocks = (unsigned)((kp.kend - kp.kbeg + 255) / 256);
    if (blocks == 0) return cudaSuccess;
    // prefetch distance: one wave, the blocks that the launch bounds keep resident
    // on every SM (a plain attribute query, also valid during graph capture)
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    kp.pf_blocks = sms * (kp.sweep_mode == SWEEP_AA_ODD ? sparse_blocks<VS, COLL, ST, SWEEP_AA_ODD>()
                                                        : sparse_blocks<VS, COLL, ST, SWEEP_PULL>());
    switch (kp.sweep_mode) {
        case SWEEP_AA_EVEN: k_step_sparse<VS, COLL, ST, SWEEP_AA_EVEN><<<blocks, 256, 0, stream>>>(kp); break;
        case SWEEP_AA_ODD: k_step_sparse<VS, COLL, ST, SWEEP_AA_ODD><<<blocks, 256, 0, stream>>>(kp); break;
        case SWEEP_PUSH: k_step_sparse<VS, COLL, ST, SWEEP_PUSH><<<blocks, 256, 0, stream>>>(kp); break;
        default:
            if (!kp.first && !kp.observe && !kp.residual && !kp.write_mom)
                k_step_sparse<VS, COLL, ST, SWEEP_PULL_PLAIN><<<blocks, 256, 0, stream>>>(kp);
            else
                k_step_sparse<VS, COLL, ST, SWEEP_PULL><<<blocks, 256, 0, stream>>>(kp);
            break;
    }
    return cudaGetLastError();
}
template <int VS>
cudaError_t launch_init_sparse(int st, const StepParams& P, const InitParams& I, cudaStream_t s);

// Sparse sweep with explicit faces and/or a scalar (two buffers); the bulk
// launch covers the fluid slots [kbeg, kend), a face pass the positions of a face.
template <int VS, int COLL>
cudaError_t launch_step_sparse_fs(int st, bool scalar, const StepParams& base, const double* lam, unsigned blocks,
                                  cudaStream_t stream);
#define LBF_SPARSE_FS_CASE(V_, C_, S_, SC_)                                                    \
    if (st == S_ && scalar == SC_) {                                                           \
        /* bulk launches prefetch one wave ahead (the blocks the launch bounds keep    */      \
        /* resident on every SM); the face pass has no wave to look ahead to          */      \
        int dev_ = 0, sms_ = 0;                                                                \
        cudaGetDevice(&dev_);                                                                  \
        cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_);                   \
        kp.pf_blocks = kp.face_pass ? 0 : sms_ * sparse_fs_blocks<V_, C_, S_, SC_>();           \
        k_step_sparse_fs<V_, C_, S_, true, SC_><<<blocks, 256, 0, stream>>>(kp);                \
        return cudaGetLastError();                                                             \
    }

// One translation unit per (velocity set, collision) instantiates the step kernels.
template <int VS, int COLL>
cudaError_t launch_step_c(int st, bool facebc, bool scalar, bool stage, const StepParams& base, const double* lam,
                          const Launch& L);

#define LBF_INSTANTIATE_COLL(VS_, COLL_)                                                               \
    template <>                                                                                        \
    cudaError_t launch_step_c<VS_, COLL_>(int st, bool facebc, bool scalar, bool stage,                \
                                          const StepParams& base, const double* lam, const Launch& L) { \
        constexpr int VS = VS_;                                                                        \
        const int coll = COLL_;                                                                        \
        KParams<VS> kp;                                                                                \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        LBF_STEP_COLL(COLL_)                                                                           \
        return cudaErrorInvalidValue;                                                                  \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_step_list<VS_, COLL_>(int st, const StepParams& base, const double* lam,         \
                                             cudaStream_t stream) {                                    \
        KParams<VS_> kp;                                                                               \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        switch (st) {                                                                                  \
            case ST_F64: return launch_list_st<VS_, COLL_, ST_F64>(kp, stream);                        \
            case ST_F32: return launch_list_st<VS_, COLL_, ST_F32>(kp, stream);                        \
            case ST_F16: return launch_list_st<VS_, COLL_, ST_F16>(kp, stream);                        \
            case ST_BF16: return launch_list_st<VS_, COLL_, ST_BF16>(kp, stream);                      \
            default: return cudaErrorInvalidValue;                                                     \
        }                                                                                              \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_step_sparse<VS_, COLL_>(int st, const StepParams& base, const double* lam,       \
                                               cudaStream_t stream) {                                  \
        KParams<VS_> kp;                                                                               \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        switch (st) {                                                                                  \
            case ST_F64: return launch_sparse_st<VS_, COLL_, ST_F64>(kp, stream);                      \
            case ST_F32: return launch_sparse_st<VS_, COLL_, ST_F32>(kp, stream);                      \
            case ST_F16: return launch_sparse_st<VS_, COLL_, ST_F16>(kp, stream);                      \
            case ST_BF16: return launch_sparse_st<VS_, COLL_, ST_BF16>(kp, stream);                    \
            default: return cudaErrorInvalidValue;                                                     \
        }                                                                                              \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_step_pipe<VS_, COLL_>(int st, const StepParams& base, const double* lam,         \
                                             int stages, int nc, cudaStream_t stream) {                 \
        KParams<VS_> kp;                                                                               \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        kp.pipe_stages = stages;                                                                       \
        kp.pipe_nc = nc;                                                                               \
        switch (st) {                                                                                  \
            case ST_F64: return launch_pipe_st<VS_, COLL_, ST_F64>(kp, stages, nc, stream);            \
            case ST_F32: return launch_pipe_st<VS_, COLL_, ST_F32>(kp, stages, nc, stream);            \
            case ST_F16: return launch_pipe_st<VS_, COLL_, ST_F16>(kp, stages, nc, stream);            \
            case ST_BF16: return launch_pipe_st<VS_, COLL_, ST_BF16>(kp, stages, nc, stream);          \
            default: return cudaErrorInvalidValue;                                                     \
        }                                                                                              \
    }

#define LBF_INSTANTIATE_SPARSE_FS(VS_, COLL_)                                                          \
    template <>                                                                                        \
    cudaError_t launch_step_sparse_fs<VS_, COLL_>(int st, bool scalar, const StepParams& base,         \
                                                  const double* lam, unsigned blocks, cudaStream_t stream) { \
        if (blocks == 0) return cudaSuccess;                                                           \
        KParams<VS_> kp;                                                                               \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        LBF_SPARSE_FS_CASE(VS_, COLL_, ST_F64, false) LBF_SPARSE_FS_CASE(VS_, COLL_, ST_F32, false)    \
        LBF_SPARSE_FS_CASE(VS_, COLL_, ST_F16, false) LBF_SPARSE_FS_CASE(VS_, COLL_, ST_BF16, false)   \
        LBF_SPARSE_FS_CASE(VS_, COLL_, ST_F64, true) LBF_SPARSE_FS_CASE(VS_, COLL_, ST_F32, true)      \
        return cudaErrorInvalidValue;                                                                  \
    }

// The central-moment collision exists for the tensor-product sets only.
#define LBF_CENTRAL_CASE_1(VS_) \
    case COLL_CENTRAL: return launch_step_c<VS_, COLL_CENTRAL>(st, facebc, scalar, stage, base, lam, L);
#define LBF_CENTRAL_CASE_0(VS_)
#define LBF_INSTANTIATE(VS_, CENTRAL_)                                                                 \
    template <>                                                                                        \
    cudaError_t launch_step<VS_>(int coll, int st, bool facebc, bool scalar, bool stage,               \
                                 const StepParams& base, const double* lam, const Launch& L) {         \
        switch (coll) {                                                                                \
            case COLL_BGK: return launch_step_c<VS_, COLL_BGK>(st, facebc, scalar, stage, base, lam, L); \
            case COLL_TRT: return launch_step_c<VS_, COLL_TRT>(st, facebc, scalar, stage, base, lam, L); \
            case COLL_MRT: return launch_step_c<VS_, COLL_MRT>(st, facebc, scalar, stage, base, lam, L); \
            LBF_CENTRAL_CASE_##CENTRAL_(VS_)                                                           \
            default: return cudaErrorInvalidValue;                                                     \
        }                                                                                              \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_init<VS_>(int st, bool scalar, const StepParams& P, const InitParams& I,        \
                                 void* const* pb, const Launch& L) {                                   \
        constexpr int VS = VS_;                                                                        \
        if (scalar) {                                                                                  \
            if (st == ST_F64) k_init<VS, ST_F64, true><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); \
            else if (st == ST_F32) k_init<VS, ST_F32, true><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); \
            else return cudaErrorInvalidValue;                                                         \
        } else {                                                                                       \
            switch (st) {                                                                              \
                case ST_F64: k_init<VS, ST_F64, false><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); break; \
                case ST_F32: k_init<VS, ST_F32, false><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); break; \
                case ST_F16: k_init<VS, ST_F16, false><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); break; \
                case ST_BF16: k_init<VS, ST_BF16, false><<<L.grid, L.block, 0, L.stream>>>(P, I, pb[0], pb[1], pb[2], pb[3], pb[4], pb[5], pb[6], pb[7], pb[8], pb[9], pb[10], pb[11]); break; \
                default: return cudaErrorInvalidValue;                                                 \
            }                                                                                          \
        }                                                                                              \
        return cudaGetLastError();                                                                     \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_init_sparse<VS_>(int st, const StepParams& P, const InitParams& I, cudaStream_t s) { \
        const unsigned nb = (unsigned)((P.nlist + 255) / 256);                                         \
        if (nb == 0) return cudaSuccess;                                                               \
        switch (st) {                                                                                  \
            case ST_F64: k_init_sparse<VS_, ST_F64><<<nb, 256, 0, s>>>(P, I); break;                   \
            case ST_F32: k_init_sparse<VS_, ST_F32><<<nb, 256, 0, s>>>(P, I); break;                   \
            case ST_F16: k_init_sparse<VS_, ST_F16><<<nb, 256, 0, s>>>(P, I); break;                   \
            case ST_BF16: k_init_sparse<VS_, ST_BF16><<<nb, 256, 0, s>>>(P, I); break;                 \
            default: return cudaErrorInvalidValue;                                                     \
        }                                                                                              \
        return cudaGetLastError();                                                                     \
    }                                                                                                  \
    template <>                                                                                        \
    cudaError_t launch_setup<VS_>(const SetupParams& S, const Launch& L) {                             \
        k_setup<VS_><<<L.grid, L.block, 0, L.stream>>>(S);                                             \
        return cudaGetLastError();                                                                     \
    }

}  // namespace lbf
