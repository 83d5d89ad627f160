// lbf_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A CPU, FP64 restatement of the reference lattice Boltzmann step
// (gilberto-ribeiro/lbflow, Rust).  The reference cannot be built here (no Rust
// toolchain, crates not vendored), so this file follows its source pass by pass,
// with the same floating-point expression order (no FMA contraction:
// compiled with -ffp-contract=off), so that it reproduces the reference
// arithmetic.  It is used only by tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py, as the checker and as the
// timed CPU baseline.  Nothing in the lbflow_b200 product path may call it.
//
// Pinned against the reference's own unit tests (golden vectors in
// tests/golden/, generated by tests/golden/make_golden.py from the reference
// sources).  Arithmetic not covered by a reference test (TRT, MRT, Guo source,
// moving-wall BB, anti-BB, Zou-He, scalar step, adsorption) follows the cited
// source lines; those parts are "unpinned" beyond code reading.
//
// Layout mirrors the reference data model with flat arrays instead of one
// object per node: f, f_eq, f_star [N*Q]; density [N]; velocity [N*D];
// shallow copies for residuals; the fluid / face / bounce-back node lists of
// Lattice::new (src/momentum/lattice.rs:156-191).

#include "../include/lbflow.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

typedef double Float;
// src/constants.rs:1-21
const Float DELTA_T = 1.0;
const Float CS_2_INV = 3.0;
const Float CS_4_INV = 9.0;
const int64_t MIN_ITER = 10;

thread_local std::string g_err;
lbf_status fail(lbf_status s, const std::string& m) { g_err = m; return s; }

// ------------------------------------------------------------ velocity sets
// Tables of src/velocity_set.rs:28-190 and src/velocity_set/{d2q9,d3q19,d3q27}.rs.
struct VS {
    int id = -1, d = 0, q = 0;
    int c[27][3] = {};
    Float w[27] = {};
    int qbar[27] = {};
    int nqf = 0;
    int qfaces[6][9] = {};
    int normal[6] = {};
    bool has_mrt = false;
    Float M[27][27] = {}, Minv[27][27] = {};
    bool has_meq_fn = false;   // mrt_equilibrium_moments_computation is Some
};

// Velocity orderings (src/velocity_set/d2q9.rs:8-18, d3q19.rs:7-27, d3q27.rs:7-35).
const int C_D2Q9[9][2] = {{0,0},{1,0},{0,1},{-1,0},{0,-1},{1,1},{-1,1},{-1,-1},{1,-1}};
const int C_D3Q27[27][3] = {
    {0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1},
    {1,1,0},{-1,-1,0},{1,0,1},{-1,0,-1},{0,1,1},{0,-1,-1},{1,-1,0},{-1,1,0},{1,0,-1},{-1,0,1},{0,1,-1},{0,-1,1},
    {1,1,1},{-1,-1,-1},{1,1,-1},{-1,-1,1},{1,-1,1},{-1,1,-1},{-1,1,1},{1,-1,-1}};

// Outward normal of each face (BoundaryFace order W,E,S,N,B,T).
const int OUTWARD[6][3] = {{-1,0,0},{1,0,0},{0,-1,0},{0,1,0},{0,0,-1},{0,0,1}};

void finish_tables(VS& v) {
    for (int i = 0; i < v.q; ++i)
        for (int j = 0; j < v.q; ++j) {
            bool opp = true;
            for (int a = 0; a < v.d; ++a) opp = opp && (v.c[j][a] == -v.c[i][a]);
            if (opp) v.qbar[i] = j;
        }
    int nf = v.d == 2 ? 4 : 6;
    for (int f = 0; f < nf; ++f) {
        int k = 0;
        for (int i = 0; i < v.q; ++i) {
            int dot = 0;
            for (int a = 0; a < v.d; ++a) dot += v.c[i][a] * OUTWARD[f][a];
            if (dot == 1) v.qfaces[f][k++] = i;     // ascending i, as in Q_WEST.. tables
            bool inward = true;
            for (int a = 0; a < v.d; ++a) inward = inward && (v.c[i][a] == -OUTWARD[f][a]);
            if (inward) v.normal[f] = i;             // face_normal_directions
        }
        v.nqf = k;
    }
}

// Row polynomials of the orthogonal MRT bases.  D2Q9: Lallemand & Luo (2000)
// basis, the rows of src/velocity_set/d2q9.rs:44-54.  D3Q19: d'Humieres et al.
// (2002) basis, the rows of src/velocity_set/d3q19.rs:69-...  Evaluated here
// from their defining polynomials.
Float mrt_row_d2q9(int k, const int* c) {
    Float cx = c[0], cy = c[1], c2 = cx * cx + cy * cy;
    switch (k) {
        case 0: return 1.0;
        case 1: return -4.0 + 3.0 * c2;
        case 2: return 4.0 - 10.5 * c2 + 4.5 * c2 * c2;
        case 3: return cx;
        case 4: return (-5.0 + 3.0 * c2) * cx;
        case 5: return cy;
        case 6: return (-5.0 + 3.0 * c2) * cy;
        case 7: return cx * cx - cy * cy;
        default: return cx * cy;
    }
}
Float mrt_row_d3q19(int k, const int* c) {
    Float x = c[0], y = c[1], z = c[2], c2 = x * x + y * y + z * z;
    switch (k) {
        case 0: return 1.0;
        case 1: return 19.0 * c2 - 30.0;
        case 2: return (21.0 * c2 * c2 - 53.0 * c2 + 24.0) / 2.0;
        case 3: return x;
        case 4: return (5.0 * c2 - 9.0) * x;
        case 5: return y;
        case 6: return (5.0 * c2 - 9.0) * y;
        case 7: return z;
        case 8: return (5.0 * c2 - 9.0) * z;
        case 9: return 3.0 * x * x - c2;
        case 10: return (3.0 * c2 - 5.0) * (3.0 * x * x - c2);
        case 11: return y * y - z * z;
        case 12: return (3.0 * c2 - 5.0) * (y * y - z * z);
        case 13: return x * y;
        case 14: return y * z;
        case 15: return x * z;
        case 16: return x * (y * y - z * z);
        case 17: return y * (z * z - x * x);
        default: return z * (x * x - y * y);
    }
}

// D3Q27 has no usable MRT basis in the reference (src/velocity_set/d3q27.rs:86 is a
// placeholder and src/velocity_set.rs:168 is todo!()).  This engine defines one:
// Gram-Schmidt (plain dot product over the 27 velocities) of the sequence
// 1; cx, cy, cz; |c|^2, 2cx^2-cy^2-cz^2, cy^2-cz^2, cxcy, cycz, cxcz;
// cx^2cy, cx^2cz, cy^2cx, cy^2cz, cz^2cx, cz^2cy, cxcycz;
// cx^2cy^2, cx^2cz^2, cy^2cz^2, cx^2cycz, cy^2cxcz, cz^2cxcy;
// cx^2cy^2cz, cx^2cz^2cy, cy^2cz^2cx; cx^2cy^2cz^2.
Float mono_d3q27(int k, const int* c) {
    Float x = c[0], y = c[1], z = c[2];
    Float x2 = x * x, y2 = y * y, z2 = z * z;
    switch (k) {
        case 0: return 1.0;
        case 1: return x; case 2: return y; case 3: return z;
        case 4: return x2 + y2 + z2;
        case 5: return 2.0 * x2 - y2 - z2;
        case 6: return y2 - z2;
        case 7: return x * y; case 8: return y * z; case 9: return x * z;
        case 10: return x2 * y; case 11: return x2 * z; case 12: return y2 * x;
        case 13: return y2 * z; case 14: return z2 * x; case 15: return z2 * y;
        case 16: return x * y * z;
        case 17: return x2 * y2; case 18: return x2 * z2; case 19: return y2 * z2;
        case 20: return x2 * y * z; case 21: return y2 * x * z; case 22: return z2 * x * y;
        case 23: return x2 * y2 * z; case 24: return x2 * z2 * y; case 25: return y2 * z2 * x;
        default: return x2 * y2 * z2;
    }
}

void build_inverse_from_orthogonal_rows(VS& v) {
    for (int k = 0; k < v.q; ++k) {
        Float n2 = 0.0;
        for (int i = 0; i < v.q; ++i) n2 += v.M[k][i] * v.M[k][i];
        for (int i = 0; i < v.q; ++i) v.Minv[i][k] = v.M[k][i] / n2;
    }
}

VS make_vs(int id) {
    VS v;
    v.id = id;
    if (id == LBF_D2Q9) {
        v.d = 2; v.q = 9;
        for (int i = 0; i < 9; ++i) { v.c[i][0] = C_D2Q9[i][0]; v.c[i][1] = C_D2Q9[i][1]; }
        for (int i = 0; i < 9; ++i) {
            int c2 = v.c[i][0] * v.c[i][0] + v.c[i][1] * v.c[i][1];
            v.w[i] = c2 == 0 ? 4.0 / 9.0 : (c2 == 1 ? 1.0 / 9.0 : 1.0 / 36.0);
        }
        v.has_mrt = true; v.has_meq_fn = true;
        for (int k = 0; k < 9; ++k) for (int i = 0; i < 9; ++i) v.M[k][i] = mrt_row_d2q9(k, v.c[i]);
        build_inverse_from_orthogonal_rows(v);
    } else if (id == LBF_D3Q19 || id == LBF_D3Q27) {
        v.d = 3; v.q = id == LBF_D3Q19 ? 19 : 27;
        for (int i = 0; i < v.q; ++i) for (int a = 0; a < 3; ++a) v.c[i][a] = C_D3Q27[i][a];
        for (int i = 0; i < v.q; ++i) {
            int c2 = v.c[i][0] * v.c[i][0] + v.c[i][1] * v.c[i][1] + v.c[i][2] * v.c[i][2];
            if (id == LBF_D3Q19) v.w[i] = c2 == 0 ? 1.0 / 3.0 : (c2 == 1 ? 1.0 / 18.0 : 1.0 / 36.0);
            else v.w[i] = c2 == 0 ? 8.0 / 27.0 : (c2 == 1 ? 2.0 / 27.0 : (c2 == 2 ? 1.0 / 54.0 : 1.0 / 216.0));
        }
        v.has_mrt = true;
        if (id == LBF_D3Q19) {
            v.has_meq_fn = true;
            for (int k = 0; k < 19; ++k) for (int i = 0; i < 19; ++i) v.M[k][i] = mrt_row_d3q19(k, v.c[i]);
        } else {
            v.has_meq_fn = false;   // m_eq = M f_eq (the None branch of kernel.rs:88-100)
            // classical Gram-Schmidt, row by row, in long double then rounded
            long double R[27][27];
            for (int k = 0; k < 27; ++k) {
                for (int i = 0; i < 27; ++i) R[k][i] = mono_d3q27(k, v.c[i]);
                for (int j = 0; j < k; ++j) {
                    long double num = 0, den = 0;
                    for (int i = 0; i < 27; ++i) { num += R[k][i] * R[j][i]; den += R[j][i] * R[j][i]; }
                    for (int i = 0; i < 27; ++i) R[k][i] -= num / den * R[j][i];
                }
            }
            for (int k = 0; k < 27; ++k) for (int i = 0; i < 27; ++i) v.M[k][i] = (Float)R[k][i];
        }
        build_inverse_from_orthogonal_rows(v);
    } else {
        v.id = -1;
        return v;
    }
    finish_tables(v);
    return v;
}

// ------------------------------------------------------------ kernel.rs
// kernel::equilibrium (src/kernel.rs:3-26)
inline void equilibrium(const VS& v, Float value, const Float* u, Float* feq) {
    Float u_dot_u = 0.0;
    for (int a = 0; a < v.d; ++a) u_dot_u += u[a] * u[a];
    for (int i = 0; i < v.q; ++i) {
        Float u_dot_c = 0.0;
        for (int a = 0; a < v.d; ++a) u_dot_c += u[a] * (Float)v.c[i][a];
        feq[i] = v.w[i] * value *
                 (1.0 + u_dot_c * CS_2_INV + 0.5 * u_dot_c * u_dot_c * CS_4_INV - 0.5 * u_dot_u * CS_2_INV);
    }
}
// kernel::bgk_collision (src/kernel.rs:28-42)
inline void bgk(const VS& v, const Float* f, const Float* feq, Float tau, Float* fs) {
    Float omega = DELTA_T / tau;
    Float omega_prime = 1.0 - omega;
    for (int i = 0; i < v.q; ++i) fs[i] = omega_prime * f[i] + omega * feq[i];
}
// kernel::trt_collision (src/kernel.rs:44-65)
inline void trt(const VS& v, const Float* f, const Float* feq, Float op, Float om, Float* fs) {
    for (int i = 0; i < v.q; ++i) {
        int ib = v.qbar[i];
        Float f_plus = 0.5 * (f[i] + f[ib]);
        Float f_eq_plus = 0.5 * (feq[i] + feq[ib]);
        Float f_minus = 0.5 * (f[i] - f[ib]);
        Float f_eq_minus = 0.5 * (feq[i] - feq[ib]);
        fs[i] = f[i] - op * DELTA_T * (f_plus - f_eq_plus) - om * DELTA_T * (f_minus - f_eq_minus);
    }
}
// velocity_set::{d2q9,d3q19}::mrt_equilibrium_moments_computation
// (src/velocity_set/d2q9.rs:247-264, src/velocity_set/d3q19.rs:550-587), kept bug-for-bug.
void meq_reference(const VS& v, Float density, const Float* u, Float* m) {
    if (v.id == LBF_D2Q9) {
        m[0] = density;
        m[1] = density - 3.0 * density * (u[0] * u[0] + u[1] * u[1]);
        m[2] = 9.0 * density * u[0] * u[0] * u[1] * u[1] - 3.0 * density * (u[0] * u[0] + u[1] * u[1]) + density;
        m[3] = density * u[0];
        m[4] = 3.0 * density * u[0] * u[0] * u[0] - density * u[0];
        m[5] = density * u[1];
        m[6] = 3.0 * density * u[1] * u[1] * u[1] - density * u[1];
        m[7] = density * (u[0] * u[0] + u[1] * u[1]);
        m[8] = density * u[0] * u[1];
    } else {  // D3Q19
        Float uu = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        m[0] = density;
        m[1] = -11.0 * density + 19.0 * density * uu;
        m[2] = 3.0 * density - 5.5 * density * uu;
        m[3] = density * u[0];
        m[4] = -2.0 / 3.0 * density * u[0];
        m[5] = density * u[1];
        m[6] = -2.0 / 3.0 * density * u[1];
        m[7] = density * u[2];
        m[8] = -2.0 / 3.0 * density * u[2];
        m[9] = 2.0 * density * u[0] * u[0] - density * (u[1] * u[1] + u[2] + u[2]);
        m[10] = -0.5 * (2.0 * density * u[0] * u[0] - density * (u[1] * u[1] + u[2] + u[2]));
        m[11] = density * (u[1] * u[1] - u[2] * u[2]);
        m[12] = -0.5 * density * (u[1] * u[1] - u[2] * u[2]);
        m[13] = density * u[0] * u[1];
        m[14] = density * u[1] * u[2];
        m[15] = density * u[0] * u[2];
        m[16] = 0.0; m[17] = 0.0; m[18] = 0.0;
    }
}
// kernel::mrt_collision (src/kernel.rs:67-120)
void mrt(const VS& v, Float value, const Float* u, const Float* f, const Float* feq,
         const Float* relax, int compat, Float* fs) {
    Float m[27], m_eq[27], m_star[27];
    for (int k = 0; k < v.q; ++k) {
        Float s = 0.0;
        for (int i = 0; i < v.q; ++i) s += v.M[k][i] * f[i];
        m[k] = s;
    }
    if (v.has_meq_fn && compat == LBF_COMPAT_REFERENCE) {
        meq_reference(v, value, u, m_eq);
    } else {
        for (int k = 0; k < v.q; ++k) {
            Float s = 0.0;
            for (int i = 0; i < v.q; ++i) s += v.M[k][i] * feq[i];
            m_eq[k] = s;
        }
    }
    for (int k = 0; k < v.q; ++k) m_star[k] = m[k] - relax[k] * DELTA_T * (m[k] - m_eq[k]);
    for (int i = 0; i < v.q; ++i) {
        Float s = 0.0;
        for (int k = 0; k < v.q; ++k) s += v.Minv[i][k] * m_star[k];
        fs[i] = s;
    }
}
// kernel::momentum_source_term (src/kernel.rs:122-154), Guo forcing.
void momentum_source(const VS& v, const Float* u, const Float* F, Float tau, Float* out) {
    Float coeff_b = 1.0 - 0.5 * DELTA_T / tau;
    for (int i = 0; i < v.q; ++i) {
        Float u_dot_c = 0.0;
        for (int a = 0; a < v.d; ++a) u_dot_c += u[a] * (Float)v.c[i][a];
        Float s = 0.0;
        for (int a = 0; a < v.d; ++a) {
            Float ca = (Float)v.c[i][a];
            s += (CS_2_INV * ca - CS_2_INV * u[a] + CS_4_INV * u_dot_c * ca) * F[a];
        }
        out[i] = coeff_b * v.w[i] * s;
    }
}
// Guo source without the (1 - omega/2) factor; used by the physics-fixed mode.
void raw_source(const VS& v, const Float* u, const Float* F, Float* out) {
    for (int i = 0; i < v.q; ++i) {
        Float u_dot_c = 0.0;
        for (int a = 0; a < v.d; ++a) u_dot_c += u[a] * (Float)v.c[i][a];
        Float s = 0.0;
        for (int a = 0; a < v.d; ++a) {
            Float ca = (Float)v.c[i][a];
            s += (CS_2_INV * ca - CS_2_INV * u[a] + CS_4_INV * u_dot_c * ca) * F[a];
        }
        out[i] = v.w[i] * s;
    }
}

// velocity_set::d2q9::zou_he_bc_computation (src/velocity_set/d2q9.rs:165-245).
// Returns false where the reference panics (ZOUHE_ERROR_MESSAGE).
bool zou_he_d2q9(int face, Float* f, bool has_rho, Float rho_in, const int* has_u, const Float* u_in) {
    bool vel = !has_rho && has_u[0] && has_u[1];
    switch (face) {
        case LBF_WEST: {
            Float rho, ux, uy = u_in[1];
            if (vel) {
                ux = u_in[0];
                rho = 1.0 / (1.0 - ux) * (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7]));
            } else if (has_rho && !has_u[0] && has_u[1]) {
                rho = rho_in;
                ux = 1.0 - 1.0 / rho * (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7]));
            } else return false;
            f[1] = f[3] + (2.0 / 3.0) * rho * ux;
            f[5] = f[7] - 0.5 * (f[2] - f[4]) + 0.5 * rho * uy + (1.0 / 6.0) * rho * ux;
            f[8] = f[6] + 0.5 * (f[2] - f[4]) - 0.5 * rho * uy + (1.0 / 6.0) * rho * ux;
            return true;
        }
        case LBF_EAST: {
            Float rho, ux, uy = u_in[1];
            if (vel) {
                ux = u_in[0];
                rho = 1.0 / (1.0 + ux) * (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8]));
            } else if (has_rho && !has_u[0] && has_u[1]) {
                rho = rho_in;
                ux = 1.0 / rho * (f[0] + f[2] + f[4] + 2.0 * (f[1] + f[5] + f[8])) - 1.0;
            } else return false;
            f[3] = f[1] - (2.0 / 3.0) * rho * ux;
            f[7] = f[5] + 0.5 * (f[2] - f[4]) - 0.5 * rho * uy - (1.0 / 6.0) * rho * ux;
            f[6] = f[8] - 0.5 * (f[2] - f[4]) + 0.5 * rho * uy - (1.0 / 6.0) * rho * ux;
            return true;
        }
        case LBF_SOUTH: {
            Float rho, ux = u_in[0], uy;
            if (vel) {
                uy = u_in[1];
                rho = 1.0 / (1.0 - uy) * (f[0] + f[1] + f[3] + 2.0 * (f[4] + f[7] + f[8]));
            } else if (has_rho && has_u[0] && !has_u[1]) {
                rho = rho_in;
                uy = 1.0 - 1.0 / rho * (f[0] + f[1] + f[3] + 2.0 * (f[4] + f[7] + f[8]));
            } else return false;
            f[2] = f[4] + (2.0 / 3.0) * rho * uy;
            f[5] = f[7] - 0.5 * (f[1] - f[3]) + 0.5 * rho * ux + (1.0 / 6.0) * rho * uy;
            f[6] = f[8] + 0.5 * (f[1] - f[3]) - 0.5 * rho * ux + (1.0 / 6.0) * rho * uy;
            return true;
        }
        case LBF_NORTH: {
            Float rho, ux = u_in[0], uy;
            if (vel) {
                uy = u_in[1];
                rho = 1.0 / (1.0 + uy) * (f[0] + f[1] + f[3] + 2.0 * (f[2] + f[5] + f[6]));
            } else if (has_rho && has_u[0] && !has_u[1]) {
                rho = rho_in;
                uy = 1.0 / rho * (f[0] + f[1] + f[3] + 2.0 * (f[2] + f[5] + f[6])) - 1.0;
            } else return false;
            f[4] = f[2] - (2.0 / 3.0) * rho * uy;
            f[7] = f[5] + 0.5 * (f[1] - f[3]) - 0.5 * rho * ux - (1.0 / 6.0) * rho * uy;
            f[8] = f[6] - 0.5 * (f[1] - f[3]) + 0.5 * rho * ux - (1.0 / 6.0) * rho * uy;
            return true;
        }
        default: return false;
    }
}

// Zou-He for D3Q19 and D3Q27 -- an EXTENSION of this engine: the reference has
// no 3-D Zou-He (zou_he_bc_computation is None for D3Q19, src/velocity_set.rs:134-135,
// and calling it panics; D3Q27 is a placeholder).  Hecht & Harting (2010),
// J. Stat. Mech. P01018: rho from the known populations, then for the unknowns
// (c.n = +1, n the inward normal) f_i = f_ibar + 6 w_i rho (c_i.u) - sum_t c_it N_t,
// N_t the transverse momentum correction.  Requiring the tangential momentum
// rho u_t gives N_t = (S_t - 2 rho u_t / 3) / M, with S_t = sum over c.n = 0 of
// c_t f and M = sum over the unknowns of c_t^2 (2 for D3Q19: N_t = S_t / 2 -
// rho u_t / 3, Hecht & Harting's form; 6 for D3Q27, whose corners take a share
// of both tangential corrections).  Mass and normal momentum hold for any N_t,
// since the unknowns' c_t sum to zero.
// Velocity inlet (density None, all velocities Some) or pressure boundary
// (density Some, normal velocity None, tangential velocities Some).
bool zou_he_general(const VS& v, int face, Float* f, bool has_rho, Float rho_in,
                    const int* has_u, const Float* u_in) {
    int ax = face / 2;
    int n_in[3] = {-OUTWARD[face][0], -OUTWARD[face][1], -OUTWARD[face][2]};
    Float sgn = (Float)n_in[ax];
    Float s0 = 0.0, sout = 0.0;
    for (int i = 0; i < v.q; ++i) {
        int cn = v.c[i][0] * n_in[0] + v.c[i][1] * n_in[1] + v.c[i][2] * n_in[2];
        if (cn == 0) s0 += f[i];
        else if (cn < 0) sout += f[i];
    }
    Float u[3] = {0.0, 0.0, 0.0};
    Float rho;
    bool tang_ok = true;
    for (int a = 0; a < v.d; ++a) if (a != ax) tang_ok = tang_ok && has_u[a];
    if (!has_rho && has_u[ax] && tang_ok) {
        for (int a = 0; a < v.d; ++a) u[a] = u_in[a];
        Float un = sgn * u[ax];
        rho = (s0 + 2.0 * sout) / (1.0 - un);
    } else if (has_rho && !has_u[ax] && tang_ok) {
        rho = rho_in;
        for (int a = 0; a < v.d; ++a) if (a != ax) u[a] = u_in[a];
        Float un = 1.0 - (s0 + 2.0 * sout) / rho;
        u[ax] = sgn * un;
    } else {
        return false;
    }
    Float N[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < v.d; ++a) {
        if (a == ax) continue;
        Float s = 0.0;
        int M = 0;
        for (int i = 0; i < v.q; ++i) {
            int cn = v.c[i][0] * n_in[0] + v.c[i][1] * n_in[1] + v.c[i][2] * n_in[2];
            if (cn == 0) s += f[i] * (Float)v.c[i][a];
            if (cn == 1) M += v.c[i][a] * v.c[i][a];
        }
        // M = 2: 0.5 s - rho u / 3 exactly (2 rho u / 6 rounds as rho u / 3)
        N[a] = s / (Float)M - 2.0 * rho * u[a] / (3.0 * (Float)M);
    }
    for (int i = 0; i < v.q; ++i) {
        int cn = v.c[i][0] * n_in[0] + v.c[i][1] * n_in[1] + v.c[i][2] * n_in[2];
        if (cn != 1) continue;
        int ib = v.qbar[i];
        Float cu = 0.0, ct = 0.0;
        for (int a = 0; a < v.d; ++a) {
            cu += (Float)v.c[i][a] * u[a];
            if (a != ax) ct += (Float)v.c[i][a] * N[a];
        }
        f[i] = f[ib] + 6.0 * v.w[i] * rho * cu - ct;
    }
    return true;
}

// ------------------------------------------------------------ lattices
struct Scalar {
    VS vs;
    lbf_collision_desc coll{};
    bool has_source = false;
    Float source = 0.0;
    bool ads = false;
    Float ka = 0, kd = 0, qmax = 0, q0 = 0;
    int inner = LBF_INNER_ANTI_BOUNCE_BACK;
    lbf_scalar_bc_desc bc[6]{};
    std::vector<Float> g, geq, gstar, C, sC, qads;
    Float res = 0.0;
};

struct Domain {
    VS vs;
    int d = 0, q = 0, nfaces = 0;
    int64_t n[3] = {1, 1, 1};
    int64_t N = 0;
    lbf_collision_desc coll{};
    int compat = 0;
    bool has_force = false;
    Float force[3] = {0, 0, 0};
    lbf_bc_desc bc[6]{};
    int order[6] = {0, 1, 2, 3, 4, 5};
    std::vector<uint8_t> type;
    std::vector<Float> f, feq, fstar, rho, u, srho, su;
    std::vector<int64_t> fluid, bbn, face_nodes[6];
    std::vector<uint32_t> links;
    std::vector<uint8_t> is_bb;
    int64_t t = 0;
    Float res[4] = {0, 0, 0, 0};
    Scalar* sc = nullptr;
    bool initialized = false;
    ~Domain() { delete sc; }

    inline int64_t nb(int64_t idx, int i) const {
        int64_t x = idx % n[0], y = (idx / n[0]) % n[1], z = idx / (n[0] * n[1]);
        int64_t xn = x + vs.c[i][0], yn = y + vs.c[i][1], zn = z + (d == 3 ? vs.c[i][2] : 0);
        xn = ((xn % n[0]) + n[0]) % n[0];   // rem_euclid (lattice.rs:138-140)
        yn = ((yn % n[1]) + n[1]) % n[1];
        zn = ((zn % n[2]) + n[2]) % n[2];
        return xn + n[0] * (yn + n[1] * zn);
    }
    inline int64_t coord(int64_t idx, int a) const {
        if (a == 0) return idx % n[0];
        if (a == 1) return (idx / n[0]) % n[1];
        return idx / (n[0] * n[1]);
    }
};

// Node::compute_density + compute_velocity (src/momentum/node.rs:418-457)
inline void node_moments(const Domain& D, const Float* f, Float& rho, Float* u) {
    const VS& v = D.vs;
    Float density = 0.0;
    for (int i = 0; i < v.q; ++i) density += f[i];
    rho = density;
    for (int a = 0; a < v.d; ++a) {
        Float s = 0.0;
        for (int i = 0; i < v.q; ++i) s += f[i] * (Float)v.c[i][a];
        u[a] = s / density;
    }
    if (D.has_force)
        for (int a = 0; a < v.d; ++a) u[a] += 0.5 * DELTA_T * D.force[a] / density;
}

void m_update_density_and_velocity(Domain& D) {
    const int64_t nf = (int64_t)D.fluid.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        node_moments(D, &D.f[idx * D.q], D.rho[idx], &D.u[idx * D.d]);
    }
}
void m_equilibrium(Domain& D) {
    const int64_t nf = (int64_t)D.fluid.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        equilibrium(D.vs, D.rho[idx], &D.u[idx * D.d], &D.feq[idx * D.q]);
    }
}
// Central-moment collision of the tensor-product sets (D2Q9, D3Q27).  No
// reference counterpart (src/velocity_set.rs:168: D3Q27 has no collision): the
// engine's definition, restated here for parity.  Central moments about u are
// built axis by axis from the 3-point raw moments (M0 = f- + f0 + f+, M1 = f+ - f-,
// M2 = f+ + f-; k0 = M0, k1 = M1 - u M0, k2 = M2 - 2 u M1 + u^2 M0); they relax
// towards rho * c(a) c(b) c(c), c = (1, 0, 1/3): order 1 reflected, order 2
// deviatoric and off-diagonal parts at 1/tau, the trace at rates[0], orders 3..6
// at rates[1..4]; then the passes are inverted (M1 = k1 + u k0,
// M2 = k2 + 2 u k1 + u^2 k0, f+ = (M2 + M1)/2, f- = (M2 - M1)/2, f0 = M0 - M2).
void central(const VS& v, Float rho, const Float* u, const Float* f, const lbf_collision_desc& cd, Float* out) {
    const int D = v.d;
    Float k[27] = {};
    auto pos = [&](int i) { return (v.c[i][0] + 1) + 3 * (v.c[i][1] + 1) + (D == 3 ? 9 * (v.c[i][2] + 1) : 0); };
    for (int i = 0; i < v.q; ++i) k[pos(i)] = f[i];
    const int nl = v.q / 3;
    for (int a = 0; a < D; ++a) {
        const int s = a == 0 ? 1 : (a == 1 ? 3 : 9);
        for (int j = 0; j < nl; ++j) {
            const int b = (j % s) + (j / s) * 3 * s;
            const Float fm = k[b], f0 = k[b + s], fp = k[b + 2 * s];
            const Float M0 = fm + f0 + fp, M1 = fp - fm, M2 = fp + fm;
            k[b] = M0;
            k[b + s] = M1 - u[a] * M0;
            k[b + 2 * s] = M2 - 2.0 * u[a] * M1 + u[a] * u[a] * M0;
        }
    }
    const Float om = 1.0 / cd.tau;
    Float r[5];
    for (int i = 0; i < 5; ++i) r[i] = cd.relaxation[i] > 0.0 ? cd.relaxation[i] : 1.0;
    auto cf = [](int o) { return o == 0 ? 1.0 : (o == 1 ? 0.0 : 1.0 / 3.0); };
    auto eq = [&](int a, int b, int c) { return rho * cf(a) * cf(b) * cf(c); };
    // order 1
    k[1] = -k[1];
    k[3] = -k[3];
    if (D == 3) k[9] = -k[9];
    // order 2
    if (D == 3) {
        const Float dxx = k[2] - eq(2, 0, 0), dyy = k[6] - eq(0, 2, 0), dzz = k[18] - eq(0, 0, 2);
        const Float tr = (1.0 - r[0]) * (dxx + dyy + dzz);
        const Float dxy = (1.0 - om) * (dxx - dyy), dxz = (1.0 - om) * (dxx - dzz);
        const Float nxx = (tr + dxy + dxz) / 3.0;
        k[2] = eq(2, 0, 0) + nxx;
        k[6] = eq(0, 2, 0) + (nxx - dxy);
        k[18] = eq(0, 0, 2) + (nxx - dxz);
        for (int p : {4, 10, 12}) k[p] = (1.0 - om) * k[p];
    } else {
        const Float dxx = k[2] - eq(2, 0, 0), dyy = k[6] - eq(0, 2, 0);
        const Float tr = (1.0 - r[0]) * (dxx + dyy), dxy = (1.0 - om) * (dxx - dyy);
        k[2] = eq(2, 0, 0) + 0.5 * (tr + dxy);
        k[6] = eq(0, 2, 0) + 0.5 * (tr - dxy);
        k[4] = (1.0 - om) * k[4];
    }
    // orders 3..6
    for (int p = 0; p < v.q; ++p) {
        const int a = p % 3, b = (p / 3) % 3, c = p / 9, ord = a + b + c;
        if (ord < 3) continue;
        const Float w = r[ord - 2];
        const Float e = eq(a, b, c);
        k[p] = e + (1.0 - w) * (k[p] - e);
    }
    for (int a = D - 1; a >= 0; --a) {
        const int s = a == 0 ? 1 : (a == 1 ? 3 : 9);
        for (int j = 0; j < nl; ++j) {
            const int b = (j % s) + (j / s) * 3 * s;
            const Float k0 = k[b], k1 = k[b + s], k2 = k[b + 2 * s];
            const Float M1 = k1 + u[a] * k0, M2 = k2 + 2.0 * u[a] * k1 + u[a] * u[a] * k0;
            k[b] = (M2 - M1) * 0.5;
            k[b + s] = k0 - M2;
            k[b + 2 * s] = (M2 + M1) * 0.5;
        }
    }
    for (int i = 0; i < v.q; ++i) out[i] = k[pos(i)];
}

// Lattice::collision_step (src/momentum/lattice.rs:343-355)
void m_collision(Domain& D) {
    const int64_t nf = (int64_t)D.fluid.size();
    const VS& v = D.vs;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        const Float* f = &D.f[idx * D.q];
        const Float* feq = &D.feq[idx * D.q];
        Float* fs = &D.fstar[idx * D.q];
        const Float* u = &D.u[idx * D.d];
        if (D.coll.kind == LBF_BGK) {
            bgk(v, f, feq, D.coll.tau, fs);
            if (D.has_force) {     // Node::compute_bgk_collision (node.rs:311-333)
                Float st[27];
                momentum_source(v, u, D.force, D.coll.tau, st);
                for (int i = 0; i < v.q; ++i) fs[i] += st[i];
            }
        } else if (D.coll.kind == LBF_TRT) {
            trt(v, f, feq, D.coll.omega_plus, D.coll.omega_minus, fs);
            if (D.has_force && D.compat == LBF_COMPAT_PHYSICS) {
                Float st[27];
                raw_source(v, u, D.force, st);
                for (int i = 0; i < v.q; ++i) {
                    int ib = v.qbar[i];
                    Float sp = 0.5 * (st[i] + st[ib]), sm = 0.5 * (st[i] - st[ib]);
                    fs[i] += (1.0 - 0.5 * D.coll.omega_plus) * sp + (1.0 - 0.5 * D.coll.omega_minus) * sm;
                }
            }
        } else if (D.coll.kind == LBF_CENTRAL) {
            central(v, D.rho[idx], u, f, D.coll, fs);
        } else {
            mrt(v, D.rho[idx], u, f, feq, D.coll.relaxation, D.compat, fs);
            if (D.has_force && D.compat == LBF_COMPAT_PHYSICS) {
                Float st[27], ms[27];
                raw_source(v, u, D.force, st);
                for (int kk = 0; kk < v.q; ++kk) {
                    Float s = 0.0;
                    for (int i = 0; i < v.q; ++i) s += v.M[kk][i] * st[i];
                    ms[kk] = (1.0 - 0.5 * D.coll.relaxation[kk]) * s;
                }
                for (int i = 0; i < v.q; ++i) {
                    Float s = 0.0;
                    for (int kk = 0; kk < v.q; ++kk) s += v.Minv[i][kk] * ms[kk];
                    fs[i] += s;
                }
            }
        }
    }
}
// NodeLike::compute_streaming (src/lib.rs:141-152): pull f*[ibar] from the
// neighbour along c_i, for every i, periodic wrap on every axis.
void stream(Domain& D, std::vector<Float>& f, const std::vector<Float>& fs, int q, const VS& v) {
    const int64_t nf = (int64_t)D.fluid.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        for (int i = 0; i < q; ++i) {
            int ib = v.qbar[i];
            int64_t nbi = D.nb(idx, i);
            f[idx * q + ib] = fs[nbi * q + ib];
        }
    }
}
// NodeLike::compute_inner_bounce_back (src/lib.rs:154-165)
void inner_bb(Domain& D, std::vector<Float>& f, const std::vector<Float>& fs, int q, const VS& v) {
    const int64_t nb = (int64_t)D.bbn.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nb; ++k) {
        int64_t idx = D.bbn[k];
        uint32_t L = D.links[idx];
        for (int i = 0; i < q; ++i)
            if (L >> i & 1u) f[idx * q + v.qbar[i]] = fs[idx * q + i];
    }
}

// Lattice::boundary_conditions_step (src/momentum/bc.rs:29-58), faces in D.order.
bool m_face_bcs(Domain& D) {
    const VS& v = D.vs;
    bool ok = true;
    for (int o = 0; o < D.nfaces; ++o) {
        int F = D.order[o];
        const lbf_bc_desc& b = D.bc[F];
        const std::vector<int64_t>& nodes = D.face_nodes[F];
        const int64_t nn = (int64_t)nodes.size();
        switch (b.kind) {
            case LBF_BC_NO_SLIP:   // bc.rs:119-129
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    for (int j = 0; j < v.nqf; ++j) {
                        int i = v.qfaces[F][j];
                        D.f[idx * D.q + v.qbar[i]] = D.fstar[idx * D.q + i];
                    }
                }
                break;
            case LBF_BC_BOUNCE_BACK:   // bc.rs:62-84
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    for (int j = 0; j < v.nqf; ++j) {
                        int i = v.qfaces[F][j];
                        Float u_dot_c = 0.0;
                        for (int a = 0; a < v.d; ++a) u_dot_c += b.velocity[a] * (Float)v.c[i][a];
                        D.f[idx * D.q + v.qbar[i]] =
                            D.fstar[idx * D.q + i] - 2.0 * v.w[i] * b.density * CS_2_INV * u_dot_c;
                    }
                }
                break;
            case LBF_BC_ANTI_BOUNCE_BACK:   // bc.rs:86-117
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    int64_t nbi = D.nb(idx, v.normal[F]);
                    Float uw[3];
                    for (int a = 0; a < v.d; ++a) uw[a] = 1.5 * D.u[idx * D.d + a] - 0.5 * D.u[nbi * D.d + a];
                    Float u_dot_u = 0.0;
                    for (int a = 0; a < v.d; ++a) u_dot_u += uw[a] * uw[a];
                    for (int j = 0; j < v.nqf; ++j) {
                        int i = v.qfaces[F][j];
                        Float u_dot_c = 0.0;
                        for (int a = 0; a < v.d; ++a) u_dot_c += uw[a] * (Float)v.c[i][a];
                        D.f[idx * D.q + v.qbar[i]] =
                            -D.fstar[idx * D.q + i] +
                            2.0 * v.w[i] * b.density *
                                (1.0 + 0.5 * u_dot_c * u_dot_c * CS_4_INV - 0.5 * u_dot_u * CS_2_INV);
                    }
                }
                break;
            case LBF_BC_ZOU_HE: {   // bc.rs:131-149
                int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    Float* f = &D.f[idx * D.q];
                    bool r = v.id == LBF_D2Q9
                                 ? zou_he_d2q9(F, f, b.has_density != 0, b.density, b.has_velocity, b.velocity)
                                 : zou_he_general(v, F, f, b.has_density != 0, b.density, b.has_velocity, b.velocity);
                    if (!r) bad += 1;
                }
                if (bad) ok = false;
                break;
            }
            default: break;   // Periodic: no-op
        }
    }
    return ok;
}

// ------------------------------------------------------------ passive scalar
// adsorption::compute_adsorption_source_value (src/passive_scalar/adsorption.rs:50-92),
// including its side effect on q_ads.  `commit` = false evaluates without the update.
inline bool scalar_source(const Domain& D, Scalar& S, int64_t idx, bool commit, Float& out) {
    bool has_user = S.has_source;
    Float user = S.source;
    if (!S.ads) {
        out = user;
        return has_user;
    }
    Float ads_v;
    if (D.is_bb[idx]) {
        Float scalar_value = S.C[idx];
        Float q_ads = S.qads[idx];
        Float r = S.ka * scalar_value * (S.qmax - q_ads) - S.kd * q_ads;
        ads_v = -r;
        if (commit) {   // update_q_ads (adsorption.rs:72-91)
            Float q_new = q_ads + r * DELTA_T;
            if (q_new < 0.0) q_new = 0.0;
            else if (q_new > S.qmax) q_new = S.qmax;
            S.qads[idx] = q_new;
        }
    } else {
        ads_v = 0.0;
    }
    out = has_user ? user + ads_v : ads_v;   // Node::get_source_value (ps/node.rs:258-266)
    return true;
}

void s_main_steps(Domain& D) {
    Scalar& S = *D.sc;
    const VS& v = S.vs;
    const int q = v.q;
    const int64_t nf = (int64_t)D.fluid.size();
    // update_scalar_value_step (ps/node.rs:272-279)
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        Float sv = 0.0;
        for (int i = 0; i < q; ++i) sv += S.g[idx * q + i];
        Float src;
        if (scalar_source(D, S, idx, true, src)) sv += 0.5 * DELTA_T * src;
        S.C[idx] = sv;
    }
    // equilibrium_step with the momentum velocity (lib.rs:107-114, ps/node.rs:133-135)
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        equilibrium(v, S.C[idx], &D.u[idx * D.d], &S.geq[idx * q]);
    }
    // collision_step (ps/lattice.rs:260-272)
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        const Float* g = &S.g[idx * q];
        const Float* geq = &S.geq[idx * q];
        Float* gs = &S.gstar[idx * q];
        if (S.coll.kind == LBF_BGK) {   // ps/node.rs:195-213
            bgk(v, g, geq, S.coll.tau, gs);
            Float src;
            if (scalar_source(D, S, idx, true, src)) {
                Float coeff_b = 1.0 - 0.5 / S.coll.tau;   // kernel.rs:156-169
                for (int i = 0; i < q; ++i) gs[i] += coeff_b * v.w[i] * src;
            }
        } else if (S.coll.kind == LBF_TRT) {
            trt(v, g, geq, S.coll.omega_plus, S.coll.omega_minus, gs);
        } else {
            mrt(v, S.C[idx], &D.u[idx * D.d], g, geq, S.coll.relaxation, D.compat, gs);
        }
    }
    stream(D, S.g, S.gstar, q, v);
    // inner_boundary_condition_step (ps/lattice.rs:280-297)
    if (S.inner == LBF_INNER_BOUNCE_BACK) {
        inner_bb(D, S.g, S.gstar, q, v);
    } else {   // compute_inner_anti_bounce_back (ps/node.rs:281-294)
        const int64_t nb = (int64_t)D.bbn.size();
#pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < nb; ++k) {
            int64_t idx = D.bbn[k];
            uint32_t L = D.links[idx];
            for (int i = 0; i < q; ++i)
                if (L >> i & 1u) {
                    Float wall_scalar_value = S.C[D.nb(idx, i)];
                    S.g[idx * q + v.qbar[i]] = -S.gstar[idx * q + i] + 2.0 * v.w[i] * wall_scalar_value;
                }
        }
    }
    // boundary_conditions_step (ps/bc.rs:37-103)
    for (int o = 0; o < D.nfaces; ++o) {
        int F = D.order[o];
        const lbf_scalar_bc_desc& b = S.bc[F];
        const lbf_bc_desc& mb = D.bc[F];
        bool have_vel = false;
        Float vel[3] = {0, 0, 0};
        switch (mb.kind) {
            case LBF_BC_NO_SLIP: have_vel = true; break;
            case LBF_BC_BOUNCE_BACK: have_vel = true; for (int a = 0; a < D.d; ++a) vel[a] = mb.velocity[a]; break;
            case LBF_BC_ZOU_HE: {
                bool all = true;
                for (int a = 0; a < D.d; ++a) all = all && mb.has_velocity[a];
                if (all) { have_vel = true; for (int a = 0; a < D.d; ++a) vel[a] = mb.velocity[a]; }
                break;
            }
            default: break;
        }
        const std::vector<int64_t>& nodes = D.face_nodes[F];
        const int64_t nn = (int64_t)nodes.size();
        const int inorm = v.normal[F];
        switch (b.kind) {
            case LBF_SBC_ANTI_BOUNCE_BACK:
            case LBF_SBC_ANTI_BB_NO_FLUX:   // ps/bc.rs:107-140
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    Float sval = b.kind == LBF_SBC_ANTI_BOUNCE_BACK ? b.scalar_value : S.C[idx];
                    Float uw[3] = {0, 0, 0};
                    if (have_vel) { for (int a = 0; a < D.d; ++a) uw[a] = vel[a]; }
                    else {   // get_wall_velocity (ps/bc.rs:201-219)
                        int64_t nbi = D.nb(idx, inorm);
                        for (int a = 0; a < D.d; ++a) uw[a] = 1.5 * D.u[idx * D.d + a] - 0.5 * D.u[nbi * D.d + a];
                    }
                    Float u_dot_u = 0.0;
                    for (int a = 0; a < D.d; ++a) u_dot_u += uw[a] * uw[a];
                    for (int j = 0; j < v.nqf; ++j) {
                        int i = v.qfaces[F][j];
                        Float u_dot_c = 0.0;
                        for (int a = 0; a < D.d; ++a) u_dot_c += uw[a] * (Float)v.c[i][a];
                        Float g_eq = v.w[i] * sval *
                                     (1.0 + u_dot_c * CS_2_INV + 0.5 * u_dot_c * u_dot_c * CS_4_INV -
                                      0.5 * u_dot_u * CS_2_INV);
                        S.g[idx * q + v.qbar[i]] = -S.gstar[idx * q + i] + 2.0 * g_eq;
                    }
                }
                break;
            case LBF_SBC_BB_NO_FLUX:   // ps/bc.rs:142-152
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    for (int j = 0; j < v.nqf; ++j) {
                        int i = v.qfaces[F][j];
                        S.g[idx * q + v.qbar[i]] = S.gstar[idx * q + i];
                    }
                }
                break;
            case LBF_SBC_ZEROTH_ORDER_NO_FLUX:   // ps/bc.rs:154-174
            case LBF_SBC_SECOND_ORDER_NO_FLUX: { // ps/bc.rs:176-199
                // Values are read from neighbours that are not on this face, so
                // the per-face parallel loop has no read/write overlap.
                std::vector<Float> newg((size_t)nn * q);
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k) {
                    int64_t idx = nodes[k];
                    int64_t n1 = D.nb(idx, inorm);
                    int64_t n2 = D.nb(n1, inorm);
                    Float* out = &newg[(size_t)k * q];
                    for (int i = 0; i < q; ++i) out[i] = S.g[idx * q + i];
                    bool second = b.kind == LBF_SBC_SECOND_ORDER_NO_FLUX;
                    if (b.unknown_populations_only) {
                        for (int j = 0; j < v.nqf; ++j) {
                            int i = v.qbar[v.qfaces[F][j]];
                            out[i] = second ? 2.0 * S.g[n1 * q + i] - S.g[n2 * q + i] : S.g[n1 * q + i];
                        }
                    } else {
                        for (int i = 0; i < q; ++i)
                            out[i] = second ? 2.0 * S.g[n1 * q + i] - S.g[n2 * q + i] : S.g[n1 * q + i];
                    }
                }
#pragma omp parallel for schedule(static)
                for (int64_t k = 0; k < nn; ++k)
                    for (int i = 0; i < q; ++i) S.g[nodes[k] * q + i] = newg[(size_t)k * q + i];
                break;
            }
            default: break;
        }
    }
}

void m_main_steps_core(Domain& D, bool& ok) {
    m_update_density_and_velocity(D);
    m_equilibrium(D);
    m_collision(D);
    stream(D, D.f, D.fstar, D.q, D.vs);
    inner_bb(D, D.f, D.fstar, D.q, D.vs);
    ok = m_face_bcs(D);
}

// Lattice::compute_lattice_residuals (src/momentum/lattice.rs:369-394) and the
// scalar one (src/passive_scalar/lattice.rs:299-313).
void residuals(Domain& D) {
    const int64_t nf = (int64_t)D.fluid.size();
    Float r0 = 0, r1 = 0, r2 = 0, r3 = 0, rc = 0;
    const int d = D.d;
#pragma omp parallel for schedule(static) reduction(+ : r0, r1, r2, r3, rc)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        Float dr = D.rho[idx] - D.srho[idx];
        r0 += dr * dr;
        Float du0 = D.u[idx * d] - D.su[idx * d];
        Float du1 = D.u[idx * d + 1] - D.su[idx * d + 1];
        r1 += du0 * du0;
        r2 += du1 * du1;
        if (d == 3) { Float du2 = D.u[idx * d + 2] - D.su[idx * d + 2]; r3 += du2 * du2; }
        if (D.sc) { Float dc = D.sc->C[idx] - D.sc->sC[idx]; rc += dc * dc; }
    }
    D.res[0] = std::sqrt(r0);
    D.res[1] = std::sqrt(r1);
    D.res[2] = std::sqrt(r2);
    D.res[3] = std::sqrt(r3);
    if (D.sc) D.sc->res = std::sqrt(rc);
}
void update_shallow(Domain& D) {
    const int64_t nf = (int64_t)D.fluid.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        D.srho[idx] = D.rho[idx];
        for (int a = 0; a < D.d; ++a) D.su[idx * D.d + a] = D.u[idx * D.d + a];
        if (D.sc) D.sc->sC[idx] = D.sc->C[idx];
    }
}

lbf_status one_iteration(Domain& D) {
    bool ok = true;
    m_main_steps_core(D, ok);
    if (!ok) return fail(LBF_EINVAL, "Error: Wrong input of Zou & He (1997) boundary conditions.");
    if (D.sc) s_main_steps(D);
    residuals(D);
    return LBF_OK;
}

bool stop_condition(const Domain& D, int64_t max_it, Float tr, Float tu, Float tc) {
    bool conv = D.res[0] <= tr;
    for (int a = 0; a < D.d; ++a) conv = conv && D.res[1 + a] <= tu;
    if (D.sc) conv = conv && D.sc->res <= tc;
    return (D.t > MIN_ITER && conv) || D.t > max_it;
}

}  // namespace

// ============================================================ C API (oracle)
extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }
int orc_num_threads(void) { return omp_get_max_threads(); }
void orc_set_num_threads(int n) { if (n > 0) omp_set_num_threads(n); }

int orc_velocity_set_tables(int id, int* d, int* q, int* c, double* w, int* qbar, int* qfaces,
                            int* normal, double* M, double* Minv) {
    VS v = make_vs(id);
    if (v.id < 0) return fail(LBF_EUNSUPPORTED, "velocity set not built"), LBF_EUNSUPPORTED;
    if (d) *d = v.d;
    if (q) *q = v.q;
    for (int i = 0; i < v.q; ++i) {
        if (c) for (int a = 0; a < 3; ++a) c[i * 3 + a] = v.c[i][a];
        if (w) w[i] = v.w[i];
        if (qbar) qbar[i] = v.qbar[i];
    }
    int nf = v.d == 2 ? 4 : 6;
    for (int f = 0; f < 6; ++f) {
        for (int j = 0; j < 9; ++j) if (qfaces) qfaces[f * 9 + j] = (f < nf && j < v.nqf) ? v.qfaces[f][j] : -1;
        if (normal) normal[f] = f < nf ? v.normal[f] : -1;
    }
    for (int k = 0; k < v.q; ++k)
        for (int i = 0; i < v.q; ++i) {
            if (M) M[k * v.q + i] = v.M[k][i];
            if (Minv) Minv[k * v.q + i] = v.Minv[k][i];
        }
    return LBF_OK;
}

// --- single-node kernels (for the known-answer tests) ---
int orc_equilibrium(int id, double value, const double* u, double* out) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    equilibrium(v, value, u, out); return LBF_OK;
}
int orc_bgk(int id, const double* f, const double* feq, double tau, double* out) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    bgk(v, f, feq, tau, out); return LBF_OK;
}
int orc_trt(int id, const double* f, const double* feq, double op, double om, double* out) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    trt(v, f, feq, op, om, out); return LBF_OK;
}
int orc_mrt(int id, double value, const double* u, const double* f, const double* feq,
            const double* relax, int compat, double* out) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    mrt(v, value, u, f, feq, relax, compat, out); return LBF_OK;
}
int orc_central(int id, double rho, const double* u, const double* f, double tau, const double* rates5,
                double* out) {
    VS v = make_vs(id); if (v.id < 0 || (v.q != 9 && v.q != 27)) return LBF_EUNSUPPORTED;
    lbf_collision_desc cd{};
    cd.kind = LBF_CENTRAL; cd.tau = tau;
    for (int i = 0; i < 5; ++i) cd.relaxation[i] = rates5[i];
    central(v, rho, u, f, cd, out); return LBF_OK;
}
int orc_momentum_source(int id, const double* u, const double* F, double tau, double* out) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    momentum_source(v, u, F, tau, out); return LBF_OK;
}
int orc_mrt_meq(int id, double rho, const double* u, double* out) {
    VS v = make_vs(id); if (v.id < 0 || !v.has_meq_fn) return LBF_EUNSUPPORTED;
    meq_reference(v, rho, u, out); return LBF_OK;
}
int orc_zou_he(int id, int face, double* f, int has_rho, double rho, const int* has_u, const double* u) {
    VS v = make_vs(id); if (v.id < 0) return LBF_EUNSUPPORTED;
    bool r = v.id == LBF_D2Q9 ? zou_he_d2q9(face, f, has_rho != 0, rho, has_u, u)
                              : zou_he_general(v, face, f, has_rho != 0, rho, has_u, u);
    return r ? LBF_OK : fail(LBF_EINVAL, "Error: Wrong input of Zou & He (1997) boundary conditions.");
}

// --- lattice ---
// Lattice::new (src/momentum/lattice.rs:27-207)
int orc_create(const lbf_domain_desc* ds, void** out) {
    if (!ds || !out) return fail(LBF_EINVAL, "null argument");
    VS v = make_vs(ds->velocity_set);
    if (v.id < 0) return fail(LBF_EUNSUPPORTED, "velocity set not supported");
    Domain* D = new Domain();
    D->vs = v; D->d = v.d; D->q = v.q; D->nfaces = v.d == 2 ? 4 : 6;
    D->n[0] = ds->n[0]; D->n[1] = ds->n[1]; D->n[2] = v.d == 3 ? ds->n[2] : 1;
    if (D->n[0] < 1 || D->n[1] < 1 || D->n[2] < 1) { delete D; return fail(LBF_EINVAL, "bad dimensions"); }
    D->N = D->n[0] * D->n[1] * D->n[2];
    D->coll = ds->collision; D->compat = ds->compat;
    D->has_force = ds->has_force != 0;
    for (int a = 0; a < 3; ++a) D->force[a] = ds->force[a];
    for (int f = 0; f < 6; ++f) D->bc[f] = ds->bc[f];
    bool zero = true;
    for (int f = 0; f < 6; ++f) zero = zero && ds->face_order[f] == 0;
    if (!zero) {
        int seen = 0;
        for (int o = 0; o < D->nfaces; ++o) {
            int F = ds->face_order[o];
            if (F < 0 || F >= D->nfaces || (seen >> F & 1)) { delete D; return fail(LBF_EINVAL, "face_order is not a permutation"); }
            seen |= 1 << F; D->order[o] = F;
        }
    }
    const int64_t N = D->N;
    D->type.assign(N, 0);
    if (ds->node_type) for (int64_t i = 0; i < N; ++i) D->type[i] = ds->node_type[i] ? 1 : 0;
    D->f.assign(N * v.q, 0.0); D->feq.assign(N * v.q, 0.0); D->fstar.assign(N * v.q, 0.0);
    D->rho.assign(N, 0.0); D->u.assign(N * v.d, 0.0);
    for (int64_t i = 0; i < N; ++i) {
        D->rho[i] = ds->initial_density_field ? ds->initial_density_field[i] : ds->initial_density;
        for (int a = 0; a < v.d; ++a)
            D->u[i * v.d + a] = ds->initial_velocity_field ? ds->initial_velocity_field[i * v.d + a] : ds->initial_velocity[a];
    }
    D->srho = D->rho; D->su = D->u;   // ShallowNode::new (node.rs:93,111)
    for (int64_t i = 0; i < N; ++i) if (D->type[i] == 0) D->fluid.push_back(i);
    const int64_t lim[6] = {0, D->n[0] - 1, 0, D->n[1] - 1, 0, D->n[2] - 1};
    for (int F = 0; F < D->nfaces; ++F)
        for (int64_t idx : D->fluid) if (D->coord(idx, F / 2) == lim[F]) D->face_nodes[F].push_back(idx);
    D->links.assign(N, 0u); D->is_bb.assign(N, 0);
    for (int64_t idx : D->fluid) {
        uint32_t L = 0;
        for (int i = 0; i < v.q; ++i) if (D->type[D->nb(idx, i)]) L |= 1u << i;
        D->links[idx] = L;
        if (L) { D->is_bb[idx] = 1; D->bbn.push_back(idx); }
    }
    // Zou-He descriptors are validated up front (the reference panics at the first step).
    for (int F = 0; F < D->nfaces; ++F) {
        if (D->bc[F].kind == LBF_BC_ZOU_HE) {
            double ftest[27];
            for (int i = 0; i < v.q; ++i) ftest[i] = v.w[i];
            bool r = v.id == LBF_D2Q9 ? zou_he_d2q9(F, ftest, D->bc[F].has_density != 0, D->bc[F].density, D->bc[F].has_velocity, D->bc[F].velocity)
                                      : zou_he_general(v, F, ftest, D->bc[F].has_density != 0, D->bc[F].density, D->bc[F].has_velocity, D->bc[F].velocity);
            if (!r) { delete D; return fail(LBF_EINVAL, "Error: Wrong input of Zou & He (1997) boundary conditions."); }
        }
    }
    *out = D;
    return LBF_OK;
}

int orc_scalar_attach(void* h, const lbf_scalar_desc* ds) {
    Domain& D = *(Domain*)h;
    if (D.sc) return fail(LBF_EINVAL, "scalar already attached");
    VS v = make_vs(ds->velocity_set);
    if (v.id < 0 || v.d != D.d) return fail(LBF_EINVAL, "scalar velocity set must match the lattice dimension");
    Scalar* S = new Scalar();
    S->vs = v; S->coll = ds->collision;
    S->has_source = ds->has_source != 0; S->source = ds->source_value;
    S->ads = ds->has_adsorption != 0;
    S->ka = ds->adsorption_rate; S->kd = ds->desorption_rate; S->qmax = ds->q_max; S->q0 = ds->initial_q_ads;
    S->inner = ds->inner_boundary_condition;
    for (int f = 0; f < 6; ++f) S->bc[f] = ds->bc[f];
    const int64_t N = D.N;
    S->g.assign(N * v.q, 0.0); S->geq.assign(N * v.q, 0.0); S->gstar.assign(N * v.q, 0.0);
    S->C.assign(N, 0.0);
    for (int64_t i = 0; i < N; ++i) S->C[i] = ds->initial_scalar_field ? ds->initial_scalar_field[i] : ds->initial_scalar_value;
    S->sC = S->C;
    S->qads.assign(N, 0.0);   // ps/node.rs:77-85
    if (S->ads) for (int64_t i : D.bbn) S->qads[i] = S->q0;
    D.sc = S;
    return LBF_OK;
}

// Lattice::initialize_nodes (lattice.rs:322-328; ps/lattice.rs:241-246)
int orc_init(void* h) {
    Domain& D = *(Domain*)h;
    const int64_t nf = (int64_t)D.fluid.size();
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < nf; ++k) {
        int64_t idx = D.fluid[k];
        equilibrium(D.vs, D.rho[idx], &D.u[idx * D.d], &D.feq[idx * D.q]);
        for (int i = 0; i < D.q; ++i) D.f[idx * D.q + i] = D.feq[idx * D.q + i];
        if (D.sc) {
            Scalar& S = *D.sc;
            equilibrium(S.vs, S.C[idx], &D.u[idx * D.d], &S.geq[idx * S.vs.q]);
            for (int i = 0; i < S.vs.q; ++i) S.g[idx * S.vs.q + i] = S.geq[idx * S.vs.q + i];
        }
    }
    D.t = 0;
    D.initialized = true;
    return LBF_OK;
}

// n iterations of the driver loop body without the stop test:
// main_steps, residuals, update_shallow_nodes, next_time_step.
int orc_step(void* h, int64_t n) {
    Domain& D = *(Domain*)h;
    if (!D.initialized) return fail(LBF_ESTATE, "init first");
    for (int64_t s = 0; s < n; ++s) {
        int st = one_iteration(D);
        if (st) return st;
        update_shallow(D);
        D.t += 1;
    }
    return LBF_OK;
}

// The driver loop (src/momentum.rs:262-293, src/passive_scalar.rs:136-177).
int orc_run(void* h, int64_t max_iterations, double tr, double tu, double tc, int64_t* steps) {
    Domain& D = *(Domain*)h;
    if (!D.initialized) return fail(LBF_ESTATE, "init first");
    for (;;) {
        int st = one_iteration(D);
        if (st) return st;
        if (stop_condition(D, max_iterations, tr, tu, tc)) break;
        update_shallow(D);
        D.t += 1;
    }
    D.t += 1;   // number of main_steps executed
    if (steps) *steps = D.t;
    return LBF_OK;
}

// Moments at the current time step, i.e. what main_steps(t) would write to
// data/<t>/ (src/momentum/io.rs:74-192): computed from the current f and g
// without changing any state (q_ads is not updated).
int orc_observe(void* h, double* rho, double* u, double* c) {
    Domain& D = *(Domain*)h;
    const int64_t N = D.N;
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < N; ++idx) {
        Float r, uu[3] = {0, 0, 0};
        if (D.type[idx] == 0 && D.initialized) {
            node_moments(D, &D.f[idx * D.q], r, uu);
        } else {
            r = D.rho[idx];
            for (int a = 0; a < D.d; ++a) uu[a] = D.u[idx * D.d + a];
        }
        if (rho) rho[idx] = r;
        if (u) for (int a = 0; a < D.d; ++a) u[idx * D.d + a] = uu[a];
        if (c && D.sc) {
            Scalar& S = *D.sc;
            if (D.type[idx] == 0 && D.initialized) {
                Float sv = 0.0;
                for (int i = 0; i < S.vs.q; ++i) sv += S.g[idx * S.vs.q + i];
                Float src;
                if (scalar_source(D, S, idx, false, src)) sv += 0.5 * DELTA_T * src;
                c[idx] = sv;
            } else {
                c[idx] = S.C[idx];
            }
        }
    }
    return LBF_OK;
}

int orc_residuals(void* h, double* out) {
    Domain& D = *(Domain*)h;
    out[0] = D.res[0];
    for (int a = 0; a < D.d; ++a) out[1 + a] = D.res[1 + a];
    if (D.sc) out[1 + D.d] = D.sc->res;
    return LBF_OK;
}
int64_t orc_time_step(void* h) { return ((Domain*)h)->t; }
int64_t orc_num_fluid(void* h) { return (int64_t)((Domain*)h)->fluid.size(); }

int orc_node_class(void* h, uint32_t* cls, uint32_t* links) {
    Domain& D = *(Domain*)h;
    for (int64_t i = 0; i < D.N; ++i) {
        uint32_t c = D.type[i] ? LBF_CLASS_SOLID : 0u;
        if (D.is_bb[i]) c |= LBF_CLASS_BOUNCE_BACK;
        if (cls) cls[i] = c;
        if (links) links[i] = D.links[i];
    }
    if (cls)
        for (int F = 0; F < D.nfaces; ++F)
            for (int64_t idx : D.face_nodes[F]) cls[idx] |= 1u << (LBF_CLASS_FACE_SHIFT + F);
    return LBF_OK;
}

int orc_get_q_ads(void* h, double* out) {
    Domain& D = *(Domain*)h;
    for (int64_t i = 0; i < D.N; ++i) out[i] = D.sc ? D.sc->qads[i] : 0.0;
    return LBF_OK;
}

int orc_inventory(void* h, double* out) {
    Domain& D = *(Domain*)h;
    std::vector<double> r(D.N), u(D.N * D.d), c(D.sc ? D.N : 0);
    orc_observe(h, r.data(), u.data(), D.sc ? c.data() : nullptr);
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int64_t idx : D.fluid) {
        s[0] += r[idx];
        for (int a = 0; a < D.d; ++a) s[1 + a] += r[idx] * u[idx * D.d + a];
        if (D.sc) { s[1 + D.d] += c[idx]; s[2 + D.d] += D.sc->qads[idx]; }
    }
    for (int k = 0; k < 3 + D.d; ++k) out[k] = s[k];
    return LBF_OK;
}

// Raw state access for unit tests that drive single passes, the way the
// reference's tests set f / f_star on a node and call one method.
// which: 0 f, 1 f_eq, 2 f_star, 3 density, 4 velocity, 5 g, 6 g_star, 7 scalar
static std::vector<Float>* pick(Domain& D, int which) {
    switch (which) {
        case 0: return &D.f; case 1: return &D.feq; case 2: return &D.fstar;
        case 3: return &D.rho; case 4: return &D.u;
        case 5: return D.sc ? &D.sc->g : nullptr; case 6: return D.sc ? &D.sc->gstar : nullptr;
        case 7: return D.sc ? &D.sc->C : nullptr;
        default: return nullptr;
    }
}
int orc_get_array(void* h, int which, double* out) {
    std::vector<Float>* a = pick(*(Domain*)h, which);
    if (!a) return LBF_EINVAL;
    std::memcpy(out, a->data(), a->size() * sizeof(Float));
    return LBF_OK;
}
int orc_set_array(void* h, int which, const double* in) {
    std::vector<Float>* a = pick(*(Domain*)h, which);
    if (!a) return LBF_EINVAL;
    std::memcpy(a->data(), in, a->size() * sizeof(Float));
    return LBF_OK;
}
// pass: 0 density+velocity, 1 equilibrium, 2 collision, 3 streaming, 4 inner BB,
// 5 face BCs, 6 residuals, 7 update shallow nodes, 8 scalar main_steps
int orc_pass(void* h, int pass) {
    Domain& D = *(Domain*)h;
    switch (pass) {
        case 0: m_update_density_and_velocity(D); return LBF_OK;
        case 1: m_equilibrium(D); return LBF_OK;
        case 2: m_collision(D); return LBF_OK;
        case 3: stream(D, D.f, D.fstar, D.q, D.vs); return LBF_OK;
        case 4: inner_bb(D, D.f, D.fstar, D.q, D.vs); return LBF_OK;
        case 5: return m_face_bcs(D) ? LBF_OK : LBF_EINVAL;
        case 6: residuals(D); return LBF_OK;
        case 7: update_shallow(D); return LBF_OK;
        case 8: if (!D.sc) return LBF_EINVAL; s_main_steps(D); return LBF_OK;
        default: return LBF_EINVAL;
    }
}
int64_t orc_neighbor(void* h, int64_t idx, int i) { return ((Domain*)h)->nb(idx, i); }

void orc_destroy(void* h) { delete (Domain*)h; }

}  // extern "C"
