// dispatch.cuh -- host-side launchers, one translation unit per velocity set
// (step_d2q9.cu, step_d3q19.cu, step_d3q27.cu instantiate them).
#pragma once

#include "aux_kernels.cuh"

namespace lbf {

struct Launch {
    dim3 grid, block;
    cudaStream_t stream;
};

template <int VS>
cudaError_t launch_step(int coll, int st, bool facebc, bool scalar, const StepParams& base, const double* lam,
                        const Launch& L);
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

#define LBF_STEP_CASE(C_, S_, FB_, SC_)                                                 \
    if (coll == C_ && st == S_ && facebc == FB_ && scalar == SC_) {                      \
        k_step<VS, C_, S_, FB_, SC_><<<L.grid, L.block, 0, L.stream>>>(kp);              \
        return cudaGetLastError();                                                      \
    }
#define LBF_STEP_ST(C_, S_)            \
    LBF_STEP_CASE(C_, S_, false, false) \
    LBF_STEP_CASE(C_, S_, true, false)
#define LBF_STEP_COLL(C_)                                                                     \
    LBF_STEP_ST(C_, ST_F64) LBF_STEP_ST(C_, ST_F32) LBF_STEP_ST(C_, ST_F16) LBF_STEP_ST(C_, ST_BF16) \
    LBF_STEP_CASE(C_, ST_F64, true, true) LBF_STEP_CASE(C_, ST_F32, true, true)

#define LBF_INSTANTIATE(VS_)                                                                           \
    template <>                                                                                        \
    cudaError_t launch_step<VS_>(int coll, int st, bool facebc, bool scalar, const StepParams& base,   \
                                 const double* lam, const Launch& L) {                                 \
        constexpr int VS = VS_;                                                                        \
        KParams<VS> kp;                                                                                \
        static_cast<StepParams&>(kp) = base;                                                           \
        fill_lam(kp, lam);                                                                             \
        LBF_STEP_COLL(COLL_BGK)                                                                        \
        LBF_STEP_COLL(COLL_TRT)                                                                        \
        LBF_STEP_COLL(COLL_MRT)                                                                        \
        return cudaErrorInvalidValue;                                                                  \
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
    cudaError_t launch_setup<VS_>(const SetupParams& S, const Launch& L) {                             \
        k_setup<VS_><<<L.grid, L.block, 0, L.stream>>>(S);                                             \
        return cudaGetLastError();                                                                     \
    }

}  // namespace lbf
