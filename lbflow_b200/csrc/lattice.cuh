// lattice.cuh -- compile-time velocity sets for the sm_100a kernels.
//
// The tables of src/velocity_set.rs:28-190 (velocity order, weights, opposite
// directions, outgoing directions per face, inward face normals) and the
// orthogonal MRT bases of src/velocity_set/d2q9.rs:44-156 and
// src/velocity_set/d3q19.rs:69-548 are expressed as constexpr functions of the
// direction index, so that every loop over directions unrolls into straight-line
// code with the table entries folded in as immediates.  Velocity components are
// packed two bits per direction (c+1) into 64-bit constants.
#pragma once

#include <cstdint>
#include <utility>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#endif

namespace lbf {

constexpr int VS_D2Q9 = 1, VS_D3Q19 = 3, VS_D3Q27 = 4;

// Compile-time integer usable from host and device code.
template <int V>
struct IC {
    static constexpr int value = V;
    __host__ __device__ constexpr operator int() const { return V; }
};

// Compile-time loop: f(IC<I>) for I = 0..N-1.
template <typename F, int... Is>
__host__ __device__ __forceinline__ void sfor_impl(F&& f, std::integer_sequence<int, Is...>) {
    (f(IC<Is>{}), ...);
}
template <int N, typename F>
__host__ __device__ __forceinline__ void sfor(F&& f) {
    sfor_impl(f, std::make_integer_sequence<int, N>{});
}

template <int VS>
struct Lat;

// D2Q9, order of src/velocity_set/d2q9.rs:8-18.
template <>
struct Lat<VS_D2Q9> {
    static constexpr int D = 2, Q = 9, NF = 4;
    __host__ __device__ static constexpr int c(int i, int a) {
        return a == 0 ? int((0x20919ull >> (2 * i)) & 3ull) - 1
                      : (a == 1 ? int((0x2865ull >> (2 * i)) & 3ull) - 1 : 0);
    }
    __host__ __device__ static constexpr int qbar(int i) {
        return i == 0 ? 0 : (i < 5 ? ((i + 1) % 4) + 1 : ((i - 3) % 4) + 5);
    }
    __host__ __device__ static constexpr double w(int i) {
        return c2(i) == 0 ? 4.0 / 9.0 : (c2(i) == 1 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
    __host__ __device__ static constexpr int c2(int i) { return c(i, 0) * c(i, 0) + c(i, 1) * c(i, 1); }
    // Lallemand & Luo (2000) moment basis, rows of src/velocity_set/d2q9.rs:44-54.
    __host__ __device__ static constexpr double M(int k, int i) {
        const double x = c(i, 0), y = c(i, 1), s = x * x + y * y;
        return k == 0 ? 1.0
             : k == 1 ? -4.0 + 3.0 * s
             : k == 2 ? 4.0 - 10.5 * s + 4.5 * s * s
             : k == 3 ? x
             : k == 4 ? (-5.0 + 3.0 * s) * x
             : k == 5 ? y
             : k == 6 ? (-5.0 + 3.0 * s) * y
             : k == 7 ? x * x - y * y
             : x * y;
    }
    static constexpr bool has_meq_fn = true;
};

// D3Q19 is the first 19 directions of the D3Q27 ordering
// (src/velocity_set/d3q19.rs:7-27, src/velocity_set/d3q27.rs:7-35).
struct Lat3 {
    __host__ __device__ static constexpr int c(int i, int a) {
        return a == 0 ? int((0x20889489489549ull >> (2 * i)) & 3ull) - 1
             : a == 1 ? int((0xa088960949495ull >> (2 * i)) & 3ull) - 1
                      : int((0x8a0a214894955ull >> (2 * i)) & 3ull) - 1;
    }
    __host__ __device__ static constexpr int qbar(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
    __host__ __device__ static constexpr int c2(int i) {
        return c(i, 0) * c(i, 0) + c(i, 1) * c(i, 1) + c(i, 2) * c(i, 2);
    }
};

template <>
struct Lat<VS_D3Q19> : Lat3 {
    static constexpr int D = 3, Q = 19, NF = 6;
    __host__ __device__ static constexpr double w(int i) {
        return c2(i) == 0 ? 1.0 / 3.0 : (c2(i) == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
    // d'Humieres et al. (2002) basis, rows of src/velocity_set/d3q19.rs:69-...
    __host__ __device__ static constexpr double M(int k, int i) {
        const double x = c(i, 0), y = c(i, 1), z = c(i, 2), s = x * x + y * y + z * z;
        return k == 0 ? 1.0
             : k == 1 ? 19.0 * s - 30.0
             : k == 2 ? (21.0 * s * s - 53.0 * s + 24.0) / 2.0
             : k == 3 ? x
             : k == 4 ? (5.0 * s - 9.0) * x
             : k == 5 ? y
             : k == 6 ? (5.0 * s - 9.0) * y
             : k == 7 ? z
             : k == 8 ? (5.0 * s - 9.0) * z
             : k == 9 ? 3.0 * x * x - s
             : k == 10 ? (3.0 * s - 5.0) * (3.0 * x * x - s)
             : k == 11 ? y * y - z * z
             : k == 12 ? (3.0 * s - 5.0) * (y * y - z * z)
             : k == 13 ? x * y
             : k == 14 ? y * z
             : k == 15 ? x * z
             : k == 16 ? x * (y * y - z * z)
             : k == 17 ? y * (z * z - x * x)
             : z * (x * x - y * y);
    }
    static constexpr bool has_meq_fn = true;
};

template <>
struct Lat<VS_D3Q27> : Lat3 {
    static constexpr int D = 3, Q = 27, NF = 6;
    __host__ __device__ static constexpr double w(int i) {
        return c2(i) == 0 ? 8.0 / 27.0 : (c2(i) == 1 ? 2.0 / 27.0 : (c2(i) == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
    }
    // No compile-time basis: the D3Q27 MRT runs in population space with a
    // collision matrix built on the host (mrt_tables.cpp).
    __host__ __device__ static constexpr double M(int, int) { return 0.0; }
    static constexpr bool has_meq_fn = false;
};

// ---- derived compile-time quantities ------------------------------------
template <class L>
__host__ __device__ constexpr double mrt_norm2(int k) {
    double s = 0.0;
    for (int i = 0; i < L::Q; ++i) s += L::M(k, i) * L::M(k, i);
    return s;
}
// M^-1 of an orthogonal basis: M^T diag(1/|row k|^2).
template <class L>
__host__ __device__ constexpr double mrt_inv(int i, int k) {
    return L::M(k, i) / mrt_norm2<L>(k);
}
// Face f (W,E,S,N,B,T): outward normal along axis f/2 with sign (f odd ? +1 : -1).
template <class L>
__host__ __device__ constexpr int c_out(int i, int f) {
    return L::c(i, f / 2) * ((f & 1) ? 1 : -1);
}
// Direction i leaves the domain through face f (q_faces of the reference).
template <class L>
__host__ __device__ constexpr bool leaves(int i, int f) {
    return c_out<L>(i, f) == 1;
}
// Inward unit normal of face f (face_normal_directions of src/velocity_set.rs).
template <class L>
__host__ __device__ constexpr int inward(int f) {
    int r = -1;
    for (int i = 0; i < L::Q; ++i) {
        bool ok = c_out<L>(i, f) == -1;
        for (int a = 0; a < L::D; ++a)
            if (a != f / 2) ok = ok && L::c(i, a) == 0;
        if (ok) r = i;
    }
    return r;
}

}  // namespace lbf
