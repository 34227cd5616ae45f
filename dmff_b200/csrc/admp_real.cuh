// Real-space multipolar PME pair kernel (sm_100a).
//
// Physics follows dmff/admp/pme.py:633-1173 (calc_e_perm, calc_e_ind, pme_real_kernel,
// pme_real): both sites' global harmonic multipoles are rotated into the quasi-internal (QI)
// frame of the pair (z along r_i - r_j), where the interaction only couples equal-|m|
// components.  Differences from the reference's vectorised JAX are in how, not what:
//   * one thread per pair row, all intermediates in registers (no [Np,9] materialisation);
//   * erf-screened factors are evaluated as (m - 1) + erfc(kr) + ... so FP32 keeps its
//     relative accuracy where 1 - erf(kr) cancels;
//   * forces come from a hand-written derivative: d/dr of every coefficient via a value+slope
//     pair, and the two transverse components from rotational invariance
//     (dE/ddr_perp = (-tau_y, tau_x)/r in the QI frame, tau = total multipole torque), so the
//     QI-frame construction is never differentiated;
//   * per-site torques of the permanent multipoles are accumulated for the local-frame
//     chain rule; i-side sums use a warp segmented reduction (rows sorted by i), j-side sums
//     use atomics; energy and box gradient accumulate in FP64.
#pragma once
#include "common.cuh"

namespace dmffb {

enum { PAIR_FULL = 0, PAIR_FIELD = 1, PAIR_MATVEC = 2 };

template <typename T>
struct PairArgs {
    int n;
    int64_t npairs;
    const int32_t* pairs;  // [npairs*3]
    const T* pos;          // [n*4]
    const double* posd;    // [n*3] FP64 positions (FP64 rows)
    const T* Qg;           // [n*9] permanent multipoles, global harmonic
    const double* Qgd;     // [n*9] the same in FP64
    const double* U;       // [n*3] Cartesian induced dipoles (FULL/FIELD may be null) or CG vector (MATVEC)
    const T* thole;        // [n]
    const T* polsix;       // [n]  pol^(1/6)
    T ms[6], ps[6], dsc[6];
    T kappa;
    Box boxd;
    T* grad;     // [n*3]  dE/dpos
    T* torque;   // [n*3]  global torque of the permanent multipoles
    T* field;    // [n*3]  dE/dU (FIELD, MATVEC)
    double* scal;  // [0] energy, [1..9] box gradient
    int want_box;
    const int32_t* rowmap = nullptr;  // ROWS_SCALED launches: indices of the rows with nbond != 0
    int64_t nrowmap = 0;
};

// row handled by this thread: the thread index, or for a scaled-rows launch with a row map the
// thread's entry of the map (threads past its end get an out-of-range row)
template <int ROWS, typename A>
__device__ __forceinline__ int64_t launch_row(const A& a) {
    int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (ROWS == 2 && a.rowmap) row = row < a.nrowmap ? (int64_t)a.rowmap[row] : a.npairs;
    return row;
}

// l=2 harmonic rotation into frame (ex, ey, ez): local[j] = sum_k C[j][k] global[k]  (multipole.py:155-203)
template <typename T>
__device__ __forceinline__ void quad_rot(const T ex[3], const T ey[3], const T ez[3], T C[5][5]) {
    const T rt3 = T(DMFFB_RT3_REF);
    const T xx = ex[0], xy = ex[1], xz = ex[2];
    const T yx = ey[0], yy = ey[1], yz = ey[2];
    const T zx = ez[0], zy = ez[1], zz = ez[2];
    C[0][0] = (T(3) * zz * zz - T(1)) * T(0.5);
    C[0][1] = rt3 * zx * zz;
    C[0][2] = rt3 * zy * zz;
    C[0][3] = rt3 * (T(-2) * zy * zy - zz * zz + T(1)) * T(0.5);
    C[0][4] = rt3 * zx * zy;
    C[1][0] = rt3 * xz * zz;
    C[1][1] = T(2) * xx * zz - yy;
    C[1][2] = yx + T(2) * xy * zz;
    C[1][3] = T(-2) * xy * zy - xz * zz;
    C[1][4] = xx * zy + zx * xy;
    C[2][0] = rt3 * yz * zz;
    C[2][1] = T(2) * yx * zz + xy;
    C[2][2] = -xx + T(2) * yy * zz;
    C[2][3] = T(-2) * yy * zy - yz * zz;
    C[2][4] = yx * zy + zx * yy;
    C[3][0] = rt3 * (T(-2) * yz * yz - zz * zz + T(1)) * T(0.5);
    C[3][1] = T(-2) * yx * yz - zx * zz;
    C[3][2] = T(-2) * yy * yz - zy * zz;
    C[3][3] = (T(4) * yy * yy + T(2) * zy * zy + T(2) * yz * yz + zz * zz - T(3)) * T(0.5);
    C[3][4] = T(-2) * yx * yy - zx * zy;
    C[4][0] = rt3 * xz * yz;
    C[4][1] = xx * yz + yx * xz;
    C[4][2] = xy * yz + yy * xz;
    C[4][3] = T(-2) * xy * yy - xz * yz;
    C[4][4] = xx * yy + yx * xy;
}

// rotate a global harmonic multipole (9) into the frame
template <typename T>
__device__ __forceinline__ void rot9(const T* Q, const T ex[3], const T ey[3], const T ez[3], const T C[5][5], T q[9]) {
    q[0] = Q[0];
    const T dx = Q[2], dy = Q[3], dz = Q[1];  // harmonic (z, x, y) -> Cartesian
    q[1] = ez[0] * dx + ez[1] * dy + ez[2] * dz;
    q[2] = ex[0] * dx + ex[1] * dy + ex[2] * dz;
    q[3] = ey[0] * dx + ey[1] * dy + ey[2] * dz;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        T s = T(0);
#pragma unroll
        for (int k = 0; k < 5; ++k) s += C[j][k] * Q[4 + k];
        q[4 + j] = s;
    }
}

// torque (active-rotation generator contraction) of a 9-component multipole q with gradient g
template <typename T>
__device__ __forceinline__ void torque9(const T q[9], const T g[9], T t[3]) {
    const T s3 = T(DMFFB_SQRT3);
    const T dx = q[2], dy = q[3], dz = q[1];
    const T gx = g[2], gy = g[3], gz = g[1];
    t[0] = dy * gz - dz * gy;
    t[1] = dz * gx - dx * gz;
    t[2] = dx * gy - dy * gx;
    const T Q0 = q[4], Q1 = q[5], Q2 = q[6], Q3 = q[7], Q4 = q[8];
    const T g0 = g[4], g1 = g[5], g2 = g[6], g3 = g[7], g4 = g[8];
    t[0] += g0 * (s3 * Q2) + g1 * Q4 + g2 * (-s3 * Q0 - Q3) + g3 * Q2 - g4 * Q1;
    t[1] += g0 * (-s3 * Q1) + g1 * (s3 * Q0 - Q3) - g2 * Q4 + g3 * Q1 + g4 * Q2;
    t[2] += -g1 * Q2 + g2 * Q1 - T(2) * g3 * Q4 + T(2) * g4 * Q3;
}

// quasi-internal frame for unit vector z
template <typename T>
__device__ __forceinline__ void qi_frame(const T ez[3], T ex[3], T ey[3]) {
    if (fabs((double)ez[0]) < 0.7) {
        T s = d_rsqrt(T(1) - ez[0] * ez[0]);
        ex[0] = (T(1) - ez[0] * ez[0]) * s;
        ex[1] = -ez[0] * ez[1] * s;
        ex[2] = -ez[0] * ez[2] * s;
    } else {
        T s = d_rsqrt(T(1) - ez[1] * ez[1]);
        ex[0] = -ez[1] * ez[0] * s;
        ex[1] = (T(1) - ez[1] * ez[1]) * s;
        ex[2] = -ez[1] * ez[2] * s;
    }
    ey[0] = ez[1] * ex[2] - ez[2] * ex[1];
    ey[1] = ez[2] * ex[0] - ez[0] * ex[2];
    ey[2] = ez[0] * ex[1] - ez[1] * ex[0];
}

// Per-pair physics in arithmetic TC.  dr: minimum-image r_i - r_j; QI/QJ: global harmonic
// multipoles; UI/UJ: Cartesian induced dipoles (POL); scales for this row; thole width Ath and
// distance scale dmp.  Outputs: FULL: oi = dE/ddr (3) + torque_i (3), oj = -dE/ddr + torque_j;
// FIELD/MATVEC: oi/oj = dE/dU_i, dE/dU_j.  e = pair energy (FULL).
template <typename TC, bool POL, int MODE>
__device__ __forceinline__ void pair_eval(const TC dr[3], const TC* QIg, const TC* QJg, const TC UI[3], const TC UJ[3],
                                          TC m, TC pp, TC dsv, TC Ath, TC dmp, TC kap, TC oi[6], TC oj[6], double& e) {
    const TC D = TC(DMFFB_DIELECTRIC);
    const TC r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
    const TC rinv = d_rsqrt(r2);
    const TC r = r2 * rinv;
    TC ez[3] = {dr[0] * rinv, dr[1] * rinv, dr[2] * rinv};
    // ---------------- shared Ewald pieces (value + d/dr)
    const TC av = kap * r;
    const TC a2v = av * av;
    const TC Xv = TC(DMFFB_TWO_OVER_SQRTPI) * d_exp(-a2v);
    const Dl<TC> A1(av, kap);
    const Dl<TC> A2(a2v, TC(2) * av * kap);
    const Dl<TC> X(Xv, TC(-2) * av * kap * Xv);
    const Dl<TC> ERFC(d_erfc(av), -kap * Xv);
    const Dl<TC> t2 = A1 * X;
    const Dl<TC> a3X = A2 * t2;
    const Dl<TC> t3 = TC(2.0 / 3.0) * a3X;
    const Dl<TC> a5X = A2 * a3X;
    const Dl<TC> t4 = TC(4.0 / 15.0) * a5X;
    const Dl<TC> R1(rinv, -rinv * rinv);
    const Dl<TC> R2 = R1 * R1;
    const Dl<TC> R3 = R2 * R1;

    if (MODE == PAIR_MATVEC) {
        // induced-induced only: T_ij = udud1 I + (udud0 - udud1) z z^T  (pme.py:872-878)
        TC u = r / dmp;
        u = u < TC(1e8) ? u : TC(1e8);
        const TC au = Ath * u;
        const TC ev = au < TC(50) ? d_exp(-au) : TC(0);
        const TC Pc = TC(1) + au + TC(0.5) * au * au;
        const TC Pd0 = Pc + au * au * au * TC(0.25);
        const TC base = ERFC.v + t2.v + t3.v;
        const TC bd0 = (dsv - TC(1)) - dsv * ev * Pd0 + base;
        const TC bd1 = (dsv - TC(1)) - dsv * ev * Pc + base;
        const TC udud0 = TC(-2.0 / 3.0) * D * R3.v * (TC(3) * bd0 + a3X.v);
        const TC udud1 = D * R3.v * (bd1 - TC(2.0 / 3.0) * a3X.v);
        const TC zUI = ez[0] * UI[0] + ez[1] * UI[1] + ez[2] * UI[2];
        const TC zUJ = ez[0] * UJ[0] + ez[1] * UJ[1] + ez[2] * UJ[2];
        const TC dd = udud0 - udud1;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            oi[c] = udud1 * UJ[c] + dd * zUJ * ez[c];
            oj[c] = udud1 * UI[c] + dd * zUI * ez[c];
        }
        return;
    }
    TC ex[3], ey[3];
    qi_frame(ez, ex, ey);
    TC C[5][5];
    quad_rot(ex, ey, ez, C);
    TC qI[9], qJ[9];
    rot9(QIg, ex, ey, ez, C, qI);
    rot9(QJg, ex, ey, ez, C, qJ);
    const Dl<TC> R4 = R2 * R2;
    const Dl<TC> R5 = R4 * R1;
    // permanent coefficients (pme.py:656-710, erfc form)
    const Dl<TC> b2m = (m - TC(1)) + (ERFC + t2);
    const Dl<TC> b3m = b2m + t3;
    const Dl<TC> b4m = b3m + t4;
    const Dl<TC> cc = D * (R1 * ((m - TC(1)) + ERFC));
    const Dl<TC> cd = D * (R2 * b2m);
    const Dl<TC> dd0 = TC(-2.0 / 3.0 * DMFFB_DIELECTRIC) * (R3 * (TC(3) * b3m + a3X));
    const Dl<TC> dd1 = D * (R3 * (b3m - TC(2.0 / 3.0) * a3X));
    const Dl<TC> cq = D * (R3 * b3m);
    const Dl<TC> dq0 = D * (R4 * (TC(3) * b3m + TC(4.0 / 3.0) * a5X));
    const Dl<TC> dq1 = TC(-DMFFB_SQRT3 * DMFFB_DIELECTRIC) * (R4 * b3m);
    const Dl<TC> qq0 = D * (R5 * (TC(6) * b4m + TC(4.0 / 45.0) * ((TC(-3) + TC(10) * A2) * a5X)));
    const Dl<TC> qq1 = TC(-4.0 / 15.0 * DMFFB_DIELECTRIC) * (R5 * (TC(15) * b4m + a5X));
    const Dl<TC> qq2 = D * (R5 * (b4m - TC(4.0 / 15.0) * a5X));

    TC uI[3] = {TC(0), TC(0), TC(0)}, uJ[3] = {TC(0), TC(0), TC(0)};
    Dl<TC> cud, dud0, dud1, udq0, udq1, udud0, udud1;
    if (POL) {
        uI[0] = ez[0] * UI[0] + ez[1] * UI[1] + ez[2] * UI[2];
        uI[1] = ex[0] * UI[0] + ex[1] * UI[1] + ex[2] * UI[2];
        uI[2] = ey[0] * UI[0] + ey[1] * UI[1] + ey[2] * UI[2];
        uJ[0] = ez[0] * UJ[0] + ez[1] * UJ[1] + ez[2] * UJ[2];
        uJ[1] = ex[0] * UJ[0] + ex[1] * UJ[1] + ex[2] * UJ[2];
        uJ[2] = ey[0] * UJ[0] + ey[1] * UJ[1] + ey[2] * UJ[2];
        // Thole-damped coefficients (pme.py:766-879)
        Dl<TC> u(r / dmp, TC(1) / dmp);
        if (u.v >= TC(1e8)) u = Dl<TC>(TC(1e8), TC(0));
        const Dl<TC> au = Ath * u;
        Dl<TC> ee(TC(0), TC(0));
        if (au.v < TC(50)) {
            const TC ev = d_exp(-au.v);
            ee = Dl<TC>(ev, -au.d * ev);
        }
        const Dl<TC> au2 = au * au;
        const Dl<TC> au3 = au2 * au;
        const Dl<TC> Pc = TC(1) + (au + TC(0.5) * au2);
        const Dl<TC> Pd0 = Pc + TC(0.25) * au3;
        const Dl<TC> Pq1 = Pc + TC(1.0 / 6.0) * au3;
        const Dl<TC> Pq0 = Pq1 + TC(1.0 / 18.0) * (au3 * au);
        const Dl<TC> base2 = ERFC + t2;
        const Dl<TC> base3 = base2 + t3;
        const Dl<TC> eP_c = ee * Pc, eP_d0 = ee * Pd0, eP_q0 = ee * Pq0, eP_q1 = ee * Pq1;
        const Dl<TC> bc2 = (pp - TC(1)) + (base2 - pp * eP_c);
        const Dl<TC> bc3 = (pp - TC(1)) + (base3 - pp * eP_c);
        const Dl<TC> bd0 = (pp - TC(1)) + (base3 - pp * eP_d0);
        const Dl<TC> bq0 = (pp - TC(1)) + (base3 - pp * eP_q0);
        const Dl<TC> bq1 = (pp - TC(1)) + (base3 - pp * eP_q1);
        const Dl<TC> ed0 = (dsv - TC(1)) + (base3 - dsv * eP_d0);
        const Dl<TC> ed1 = (dsv - TC(1)) + (base3 - dsv * eP_c);
        cud = TC(2 * DMFFB_DIELECTRIC) * (R2 * bc2);
        dud0 = TC(-4.0 / 3.0 * DMFFB_DIELECTRIC) * (R3 * (TC(3) * bd0 + a3X));
        dud1 = TC(2 * DMFFB_DIELECTRIC) * (R3 * (bc3 - TC(2.0 / 3.0) * a3X));
        udq0 = TC(2 * DMFFB_DIELECTRIC) * (R4 * (TC(3) * bq0 + TC(4.0 / 3.0) * a5X));
        udq1 = TC(-2 * DMFFB_SQRT3 * DMFFB_DIELECTRIC) * (R4 * bq1);
        udud0 = TC(-2.0 / 3.0 * DMFFB_DIELECTRIC) * (R3 * (TC(3) * ed0 + a3X));
        udud1 = D * (R3 * (ed1 - TC(2.0 / 3.0) * a3X));
    }

    if (MODE == PAIR_FIELD) {
        // dE/du of the permanent-induced terms (the P^T q part; U-U is MATVEC)
        const TC guI0 = TC(0.5) * (-cud.v * qJ[0] + dud0.v * qJ[1] - udq0.v * qJ[4]);
        const TC guI1 = TC(0.5) * (dud1.v * qJ[2] - udq1.v * qJ[5]);
        const TC guI2 = TC(0.5) * (dud1.v * qJ[3] - udq1.v * qJ[6]);
        const TC guJ0 = TC(0.5) * (cud.v * qI[0] + dud0.v * qI[1] + udq0.v * qI[4]);
        const TC guJ1 = TC(0.5) * (dud1.v * qI[2] + udq1.v * qI[5]);
        const TC guJ2 = TC(0.5) * (dud1.v * qI[3] + udq1.v * qI[6]);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            oi[c] = guI0 * ez[c] + guI1 * ex[c] + guI2 * ey[c];
            oj[c] = guJ0 * ez[c] + guJ1 * ex[c] + guJ2 * ey[c];
        }
        return;
    }
    // ---- energy and gradients in the QI frame: V = A qI (seen by J), W = A^T qJ
    Dl<TC> V[9];
    V[0] = cc * Dl<TC>(qI[0], 0) - cd * Dl<TC>(qI[1], 0) + cq * Dl<TC>(qI[4], 0);
    V[1] = cd * Dl<TC>(qI[0], 0) + dd0 * Dl<TC>(qI[1], 0) + dq0 * Dl<TC>(qI[4], 0);
    V[2] = dd1 * Dl<TC>(qI[2], 0) + dq1 * Dl<TC>(qI[5], 0);
    V[3] = dd1 * Dl<TC>(qI[3], 0) + dq1 * Dl<TC>(qI[6], 0);
    V[4] = cq * Dl<TC>(qI[0], 0) - dq0 * Dl<TC>(qI[1], 0) + qq0 * Dl<TC>(qI[4], 0);
    V[5] = qq1 * Dl<TC>(qI[5], 0) - dq1 * Dl<TC>(qI[2], 0);
    V[6] = qq1 * Dl<TC>(qI[6], 0) - dq1 * Dl<TC>(qI[3], 0);
    V[7] = qq2 * Dl<TC>(qI[7], 0);
    V[8] = qq2 * Dl<TC>(qI[8], 0);
    TC gI[9], gJ[9];
    gI[0] = cc.v * qJ[0] + cd.v * qJ[1] + cq.v * qJ[4];
    gI[1] = -cd.v * qJ[0] + dd0.v * qJ[1] - dq0.v * qJ[4];
    gI[2] = dd1.v * qJ[2] - dq1.v * qJ[5];
    gI[3] = dd1.v * qJ[3] - dq1.v * qJ[6];
    gI[4] = cq.v * qJ[0] + dq0.v * qJ[1] + qq0.v * qJ[4];
    gI[5] = dq1.v * qJ[2] + qq1.v * qJ[5];
    gI[6] = dq1.v * qJ[3] + qq1.v * qJ[6];
    gI[7] = qq2.v * qJ[7];
    gI[8] = qq2.v * qJ[8];
    TC Ev = TC(0), Ed = TC(0);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        gJ[k] = V[k].v;
        Ev += qJ[k] * V[k].v;
        Ed += qJ[k] * V[k].d;
    }
    TC tsum[2];
    TC guI[3] = {TC(0), TC(0), TC(0)}, guJ[3] = {TC(0), TC(0), TC(0)};
    if (POL) {
        // 1/2 P uI (contracted with qJ) and 1/2 P' uJ (contracted with qI)
        const Dl<TC> hJ[7] = {TC(-0.5) * (cud * Dl<TC>(uI[0], 0)), TC(0.5) * (dud0 * Dl<TC>(uI[0], 0)),
                              TC(0.5) * (dud1 * Dl<TC>(uI[1], 0)), TC(0.5) * (dud1 * Dl<TC>(uI[2], 0)),
                              TC(-0.5) * (udq0 * Dl<TC>(uI[0], 0)), TC(-0.5) * (udq1 * Dl<TC>(uI[1], 0)),
                              TC(-0.5) * (udq1 * Dl<TC>(uI[2], 0))};
        const Dl<TC> hI[7] = {TC(0.5) * (cud * Dl<TC>(uJ[0], 0)), TC(0.5) * (dud0 * Dl<TC>(uJ[0], 0)),
                              TC(0.5) * (dud1 * Dl<TC>(uJ[1], 0)), TC(0.5) * (dud1 * Dl<TC>(uJ[2], 0)),
                              TC(0.5) * (udq0 * Dl<TC>(uJ[0], 0)), TC(0.5) * (udq1 * Dl<TC>(uJ[1], 0)),
                              TC(0.5) * (udq1 * Dl<TC>(uJ[2], 0))};
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            Ev += qJ[k] * hJ[k].v + qI[k] * hI[k].v;
            Ed += qJ[k] * hJ[k].d + qI[k] * hI[k].d;
            gJ[k] += hJ[k].v;
            gI[k] += hI[k].v;
        }
        guI[0] = TC(0.5) * (-cud.v * qJ[0] + dud0.v * qJ[1] - udq0.v * qJ[4]) + udud0.v * uJ[0];
        guI[1] = TC(0.5) * (dud1.v * qJ[2] - udq1.v * qJ[5]) + udud1.v * uJ[1];
        guI[2] = TC(0.5) * (dud1.v * qJ[3] - udq1.v * qJ[6]) + udud1.v * uJ[2];
        guJ[0] = TC(0.5) * (cud.v * qI[0] + dud0.v * qI[1] + udq0.v * qI[4]) + udud0.v * uI[0];
        guJ[1] = TC(0.5) * (dud1.v * qI[2] + udq1.v * qI[5]) + udud1.v * uI[1];
        guJ[2] = TC(0.5) * (dud1.v * qI[3] + udq1.v * qI[6]) + udud1.v * uI[2];
        Ev += udud0.v * uI[0] * uJ[0] + udud1.v * (uI[1] * uJ[1] + uI[2] * uJ[2]);
        Ed += udud0.d * uI[0] * uJ[0] + udud1.d * (uI[1] * uJ[1] + uI[2] * uJ[2]);
    }
    TC tI[3], tJ[3];
    torque9(qI, gI, tI);
    torque9(qJ, gJ, tJ);
    tsum[0] = tI[0] + tJ[0];
    tsum[1] = tI[1] + tJ[1];
    if (POL) {
        // induced dipoles (harmonic z,x,y -> Cartesian x,y,z = u1,u2,u0)
        tsum[0] += (uI[2] * guI[0] - uI[0] * guI[2]) + (uJ[2] * guJ[0] - uJ[0] * guJ[2]);
        tsum[1] += (uI[0] * guI[1] - uI[1] * guI[0]) + (uJ[0] * guJ[1] - uJ[1] * guJ[0]);
    }
    const TC G0 = -tsum[1] * rinv, G1 = tsum[0] * rinv, G2 = Ed;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const TC g = G0 * ex[c] + G1 * ey[c] + G2 * ez[c];
        oi[c] = g;
        oj[c] = -g;
        oi[3 + c] = tI[0] * ex[c] + tI[1] * ey[c] + tI[2] * ez[c];
        oj[3 + c] = tJ[0] * ex[c] + tJ[1] * ey[c] + tJ[2] * ez[c];
    }
    e = (double)Ev;
}

// transpose of rot9: the global-frame gradient G of a function of the frame components q
template <typename T>
__device__ __forceinline__ void rot9T(const T* g, const T ex[3], const T ey[3], const T ez[3], const T C[5][5], T G[9]) {
    G[0] = g[0];
    // q1 = ez.d, q2 = ex.d, q3 = ey.d with d = (Q2, Q3, Q1) Cartesian
    const T cx = ez[0] * g[1] + ex[0] * g[2] + ey[0] * g[3];
    const T cy = ez[1] * g[1] + ex[1] * g[2] + ey[1] * g[3];
    const T cz = ez[2] * g[1] + ex[2] * g[2] + ey[2] * g[3];
    G[1] = cz;
    G[2] = cx;
    G[3] = cy;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        T s = T(0);
#pragma unroll
        for (int j = 0; j < 5; ++j) s += C[j][k] * g[4 + j];
        G[4 + k] = s;
    }
}

// Parameter adjoints of one pair at fixed (converged) induced dipoles: dE/dQ_global of both
// sites (9 each), and for the Thole damping dE/d(au) times au (-> dE/dpol through
// dmp = (pol_i pol_j)^(1/6)) and times u (-> dE/dthole when the width is thole_i + thole_j).
// The damped coefficients are differentiated in au with value+slope pairs: d/dau of
// e^-au P(au) = e^-au (P' - P).
template <typename TC, bool POL>
__device__ __forceinline__ void pair_eval_pgrad(const TC dr[3], const TC* QIg, const TC* QJg, const TC UI[3],
                                                const TC UJ[3], TC m, TC pp, TC dsv, TC Ath, TC dmp, TC kap,
                                                TC GI[9], TC GJ[9], TC& dau_au, TC& dau_u) {
    const TC D = TC(DMFFB_DIELECTRIC);
    const TC r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
    const TC rinv = d_rsqrt(r2);
    const TC r = r2 * rinv;
    TC ez[3] = {dr[0] * rinv, dr[1] * rinv, dr[2] * rinv};
    const TC av = kap * r;
    const TC a2v = av * av;
    const TC Xv = TC(DMFFB_TWO_OVER_SQRTPI) * d_exp(-a2v);
    const TC ERFC = d_erfc(av);
    const TC t2 = av * Xv;
    const TC a3X = a2v * t2;
    const TC t3 = TC(2.0 / 3.0) * a3X;
    const TC a5X = a2v * a3X;
    const TC t4 = TC(4.0 / 15.0) * a5X;
    const TC R1 = rinv, R2 = rinv * rinv, R3 = R2 * rinv, R4 = R2 * R2, R5 = R4 * rinv;
    TC ex[3], ey[3];
    qi_frame(ez, ex, ey);
    TC C[5][5];
    quad_rot(ex, ey, ez, C);
    TC qI[9], qJ[9];
    rot9(QIg, ex, ey, ez, C, qI);
    rot9(QJg, ex, ey, ez, C, qJ);
    const TC b2m = (m - TC(1)) + (ERFC + t2);
    const TC b3m = b2m + t3;
    const TC b4m = b3m + t4;
    const TC cc = D * (R1 * ((m - TC(1)) + ERFC));
    const TC cd = D * (R2 * b2m);
    const TC dd0 = TC(-2.0 / 3.0 * DMFFB_DIELECTRIC) * (R3 * (TC(3) * b3m + a3X));
    const TC dd1 = D * (R3 * (b3m - TC(2.0 / 3.0) * a3X));
    const TC cq = D * (R3 * b3m);
    const TC dq0 = D * (R4 * (TC(3) * b3m + TC(4.0 / 3.0) * a5X));
    const TC dq1 = TC(-DMFFB_SQRT3 * DMFFB_DIELECTRIC) * (R4 * b3m);
    const TC qq0 = D * (R5 * (TC(6) * b4m + TC(4.0 / 45.0) * ((TC(-3) + TC(10) * a2v) * a5X)));
    const TC qq1 = TC(-4.0 / 15.0 * DMFFB_DIELECTRIC) * (R5 * (TC(15) * b4m + a5X));
    const TC qq2 = D * (R5 * (b4m - TC(4.0 / 15.0) * a5X));
    TC gI[9], gJ[9];
    gI[0] = cc * qJ[0] + cd * qJ[1] + cq * qJ[4];
    gI[1] = -cd * qJ[0] + dd0 * qJ[1] - dq0 * qJ[4];
    gI[2] = dd1 * qJ[2] - dq1 * qJ[5];
    gI[3] = dd1 * qJ[3] - dq1 * qJ[6];
    gI[4] = cq * qJ[0] + dq0 * qJ[1] + qq0 * qJ[4];
    gI[5] = dq1 * qJ[2] + qq1 * qJ[5];
    gI[6] = dq1 * qJ[3] + qq1 * qJ[6];
    gI[7] = qq2 * qJ[7];
    gI[8] = qq2 * qJ[8];
    gJ[0] = cc * qI[0] - cd * qI[1] + cq * qI[4];
    gJ[1] = cd * qI[0] + dd0 * qI[1] + dq0 * qI[4];
    gJ[2] = dd1 * qI[2] + dq1 * qI[5];
    gJ[3] = dd1 * qI[3] + dq1 * qI[6];
    gJ[4] = cq * qI[0] - dq0 * qI[1] + qq0 * qI[4];
    gJ[5] = qq1 * qI[5] - dq1 * qI[2];
    gJ[6] = qq1 * qI[6] - dq1 * qI[3];
    gJ[7] = qq2 * qI[7];
    gJ[8] = qq2 * qI[8];
    dau_au = dau_u = TC(0);
    if (POL) {
        TC uI[3], uJ[3];
        uI[0] = ez[0] * UI[0] + ez[1] * UI[1] + ez[2] * UI[2];
        uI[1] = ex[0] * UI[0] + ex[1] * UI[1] + ex[2] * UI[2];
        uI[2] = ey[0] * UI[0] + ey[1] * UI[1] + ey[2] * UI[2];
        uJ[0] = ez[0] * UJ[0] + ez[1] * UJ[1] + ez[2] * UJ[2];
        uJ[1] = ex[0] * UJ[0] + ex[1] * UJ[1] + ex[2] * UJ[2];
        uJ[2] = ey[0] * UJ[0] + ey[1] * UJ[1] + ey[2] * UJ[2];
        TC u = r / dmp;
        const bool u_live = u < TC(1e8);
        if (!u_live) u = TC(1e8);
        const Dl<TC> au(Ath * u, TC(1));
        Dl<TC> ee(TC(0), TC(0));
        if (au.v < TC(50)) {
            const TC ev = d_exp(-au.v);
            ee = Dl<TC>(ev, -ev);
        }
        const Dl<TC> au2 = au * au;
        const Dl<TC> au3 = au2 * au;
        const Dl<TC> Pc = TC(1) + (au + TC(0.5) * au2);
        const Dl<TC> Pd0 = Pc + TC(0.25) * au3;
        const Dl<TC> Pq1 = Pc + TC(1.0 / 6.0) * au3;
        const Dl<TC> Pq0 = Pq1 + TC(1.0 / 18.0) * (au3 * au);
        const TC base2 = ERFC + t2, base3 = base2 + t3;
        const Dl<TC> eP_c = ee * Pc, eP_d0 = ee * Pd0, eP_q0 = ee * Pq0, eP_q1 = ee * Pq1;
        const Dl<TC> bc2 = Dl<TC>((pp - TC(1)) + base2, TC(0)) - pp * eP_c;
        const Dl<TC> bc3 = Dl<TC>((pp - TC(1)) + base3, TC(0)) - pp * eP_c;
        const Dl<TC> bd0 = Dl<TC>((pp - TC(1)) + base3, TC(0)) - pp * eP_d0;
        const Dl<TC> bq0 = Dl<TC>((pp - TC(1)) + base3, TC(0)) - pp * eP_q0;
        const Dl<TC> bq1 = Dl<TC>((pp - TC(1)) + base3, TC(0)) - pp * eP_q1;
        const Dl<TC> ed0 = Dl<TC>((dsv - TC(1)) + base3, TC(0)) - dsv * eP_d0;
        const Dl<TC> ed1 = Dl<TC>((dsv - TC(1)) + base3, TC(0)) - dsv * eP_c;
        const Dl<TC> cud = TC(2 * DMFFB_DIELECTRIC) * R2 * bc2;
        const Dl<TC> dud0 = TC(-4.0 / 3.0 * DMFFB_DIELECTRIC) * R3 * (TC(3) * bd0 + a3X);
        const Dl<TC> dud1 = TC(2 * DMFFB_DIELECTRIC) * R3 * (bc3 - TC(2.0 / 3.0) * a3X);
        const Dl<TC> udq0 = TC(2 * DMFFB_DIELECTRIC) * R4 * (TC(3) * bq0 + TC(4.0 / 3.0) * a5X);
        const Dl<TC> udq1 = TC(-2 * DMFFB_SQRT3 * DMFFB_DIELECTRIC) * R4 * bq1;
        const Dl<TC> udud0 = TC(-2.0 / 3.0 * DMFFB_DIELECTRIC) * R3 * (TC(3) * ed0 + a3X);
        const Dl<TC> udud1 = D * R3 * (ed1 - TC(2.0 / 3.0) * a3X);
        const Dl<TC> hJ[7] = {TC(-0.5) * (cud * uI[0]), TC(0.5) * (dud0 * uI[0]), TC(0.5) * (dud1 * uI[1]),
                              TC(0.5) * (dud1 * uI[2]), TC(-0.5) * (udq0 * uI[0]), TC(-0.5) * (udq1 * uI[1]),
                              TC(-0.5) * (udq1 * uI[2])};
        const Dl<TC> hI[7] = {TC(0.5) * (cud * uJ[0]), TC(0.5) * (dud0 * uJ[0]), TC(0.5) * (dud1 * uJ[1]),
                              TC(0.5) * (dud1 * uJ[2]), TC(0.5) * (udq0 * uJ[0]), TC(0.5) * (udq1 * uJ[1]),
                              TC(0.5) * (udq1 * uJ[2])};
        TC dEd = TC(0);
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            gJ[k] += hJ[k].v;
            gI[k] += hI[k].v;
            dEd += qJ[k] * hJ[k].d + qI[k] * hI[k].d;
        }
        dEd += udud0.d * uI[0] * uJ[0] + udud1.d * (uI[1] * uJ[1] + uI[2] * uJ[2]);
        if (u_live) {
            dau_au = dEd * au.v;
            dau_u = dEd * u;
        }
    }
    rot9T(gI, ex, ey, ez, C, GI);
    rot9T(gJ, ex, ey, ez, C, GJ);
}

// load one row's inputs in arithmetic TC and evaluate it
template <typename TC, typename T, bool POL, int MODE>
__device__ __forceinline__ void pair_row(const PairArgs<T>& a, int i, int j, int nb, TC oi[6], TC oj[6], double& e,
                                         TC nimg[3]) {
    TC dr[3];
    if (sizeof(TC) > sizeof(T)) {
        dr[0] = (TC)(a.posd[3 * i] - a.posd[3 * j]);
        dr[1] = (TC)(a.posd[3 * i + 1] - a.posd[3 * j + 1]);
        dr[2] = (TC)(a.posd[3 * i + 2] - a.posd[3 * j + 2]);
    } else {
        dr[0] = (TC)(a.pos[4 * i] - a.pos[4 * j]);
        dr[1] = (TC)(a.pos[4 * i + 1] - a.pos[4 * j + 1]);
        dr[2] = (TC)(a.pos[4 * i + 2] - a.pos[4 * j + 2]);
    }
    BoxT<TC> bx;
#pragma unroll
    for (int k = 0; k < 9; ++k) { bx.h[k] = (TC)a.boxd.h[k]; bx.hinv[k] = (TC)a.boxd.hinv[k]; }
    pbc_shift(bx, dr[0], dr[1], dr[2], nimg);
    int sidx = nb - 1;  // scale index nbond-1, Python-style wrap (nbond 0 -> trailing 1.0), clamped
    if (sidx < 0) sidx += 6;
    sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
    TC QI[9], QJ[9];
    if (MODE != PAIR_MATVEC) {
        if (sizeof(TC) > sizeof(T)) {
#pragma unroll
            for (int k = 0; k < 9; ++k) { QI[k] = (TC)a.Qgd[9 * i + k]; QJ[k] = (TC)a.Qgd[9 * j + k]; }
        } else {
#pragma unroll
            for (int k = 0; k < 9; ++k) { QI[k] = (TC)a.Qg[9 * i + k]; QJ[k] = (TC)a.Qg[9 * j + k]; }
        }
    }
    TC UI[3] = {TC(0), TC(0), TC(0)}, UJ[3] = {TC(0), TC(0), TC(0)};
    if (POL && a.U) {
#pragma unroll
        for (int c = 0; c < 3; ++c) { UI[c] = (TC)a.U[3 * i + c]; UJ[c] = (TC)a.U[3 * j + c]; }
    }
    TC Ath = TC(0), dmp = TC(1);
    const TC pp = (TC)a.ps[sidx], dsv = (TC)a.dsc[sidx];
    if (POL) {
        Ath = pp > TC(0) ? TC(5.0) : (TC)a.thole[i] + (TC)a.thole[j];
        dmp = (TC)a.polsix[i] * (TC)a.polsix[j];
        dmp = dmp < TC(1e-8) ? TC(1e-8) : dmp;
    }
    pair_eval<TC, POL, MODE>(dr, QI, QJ, UI, UJ, (TC)a.ms[sidx], pp, dsv, Ath, dmp, (TC)a.kappa, oi, oj, e);
}

// One thread per pair row.  Rows with a topological scale (nbond != 0: excluded / scaled
// intramolecular pairs, which carry the large Ewald corrections that cancel the self energy)
// are evaluated in FP64 even in the FP32 instantiation.
enum { ROWS_ALL = 0, ROWS_UNSCALED = 1, ROWS_SCALED = 2 };

// ROWS selects which rows this launch evaluates: all of them, only nbond == 0 rows (FP32
// arithmetic) or only nbond != 0 rows (always FP64); the FP32 engine launches the last two so
// that no warp mixes the two arithmetic paths.
template <typename T, bool POL, int MODE, int ROWS = ROWS_ALL>
__global__ void __launch_bounds__(128, (sizeof(T) == 4 && ROWS == ROWS_UNSCALED && MODE == PAIR_FULL) ? 6 : 0) k_admp_pair(PairArgs<T> a) {
    const int64_t row = launch_row<ROWS>(a);
    int i = -1, j = -1, nb = 0;
    if (row < a.npairs) {
        i = a.pairs[3 * row];
        j = a.pairs[3 * row + 1];
        nb = a.pairs[3 * row + 2];
    }
    const bool valid = (row < a.npairs) && i >= 0 && i < j && j < a.n &&
                       (ROWS == ROWS_ALL || (ROWS == ROWS_UNSCALED) == (nb == 0));
    const int key = valid ? i : -1;

    T oi[6], oj[6];  // FULL: grad(3) + torque(3); FIELD/MATVEC: field(3)
#pragma unroll
    for (int k = 0; k < 6; ++k) { oi[k] = T(0); oj[k] = T(0); }
    double eacc = 0.0;
    double nimg[3] = {0.0, 0.0, 0.0};
    if (valid) {
        if (sizeof(T) < sizeof(double) && nb != 0) {
            double di[6], dj[6], ni[3];
#pragma unroll
            for (int k = 0; k < 6; ++k) { di[k] = 0.0; dj[k] = 0.0; }
            pair_row<double, T, POL, MODE>(a, i, j, nb, di, dj, eacc, ni);
#pragma unroll
            for (int k = 0; k < 6; ++k) { oi[k] = (T)di[k]; oj[k] = (T)dj[k]; }
#pragma unroll
            for (int k = 0; k < 3; ++k) nimg[k] = ni[k];
        } else {
            T ni[3];
            pair_row<T, T, POL, MODE>(a, i, j, nb, oi, oj, eacc, ni);
#pragma unroll
            for (int k = 0; k < 3; ++k) nimg[k] = (double)ni[k];
        }
    }

    // ---- accumulate
    const int nout = (MODE == PAIR_FULL) ? 6 : 3;
    T* outp = (MODE == PAIR_FULL) ? a.grad : a.field;
    const bool head = seg_head(key);
    const int run = seg_run_id(key);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (k >= nout) break;
        T s = seg_sum(oi[k], run);
        if (head && key >= 0) {
            T* dst = (k < 3) ? (outp + 3 * key + k) : (a.torque + 3 * key + (k - 3));
            atomicAdd(dst, s);
        }
    }
    if (valid) {
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            if (k >= nout) break;
            T* dst = (k < 3) ? (outp + 3 * j + k) : (a.torque + 3 * j + (k - 3));
            atomicAdd(dst, oj[k]);
        }
    }
    if (MODE == PAIR_FULL) {
        double red[10];
        red[0] = eacc;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) red[1 + 3 * k + c] = a.want_box ? -nimg[k] * (double)oi[c] : 0.0;
        block_reduce_add<10>(red, a.scal);
    }
}


// Parameter-adjoint pass (param grads requested): per pair, dE/dQ_global of both sites and the
// Thole damping sums; at the converged dipoles E is stationary in U, so these partials are the
// total derivatives.  Outputs (FP64 atomics): dQ [n*9] += dE/dQ_global; dpa [n] += sum of
// dE/d(au) au over the atom's pairs (dE/dpol_i = -dpa_i / (6 pol_i), zero where dmp or u is
// clamped); dth [n] += sum of dE/d(au) u over pairs whose Thole width is thole_i + thole_j.
template <typename T>
struct PgradArgs {
    PairArgs<T> p;
    double* dQ;
    double* dpa;
    double* dth;
};

template <typename TC, typename T, bool POL>
__device__ __forceinline__ void pgrad_row(const PairArgs<T>& a, int i, int j, int nb, double oi[11], double oj[11]) {
    TC dr[3];
    if (sizeof(TC) > sizeof(T)) {
        for (int c = 0; c < 3; ++c) dr[c] = (TC)(a.posd[3 * i + c] - a.posd[3 * j + c]);
    } else {
        for (int c = 0; c < 3; ++c) dr[c] = (TC)(a.pos[4 * i + c] - a.pos[4 * j + c]);
    }
    BoxT<TC> bx;
#pragma unroll
    for (int k = 0; k < 9; ++k) { bx.h[k] = (TC)a.boxd.h[k]; bx.hinv[k] = (TC)a.boxd.hinv[k]; }
    TC nimg[3];
    pbc_shift(bx, dr[0], dr[1], dr[2], nimg);
    int sidx = nb - 1;
    if (sidx < 0) sidx += 6;
    sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
    TC QI[9], QJ[9];
    if (sizeof(TC) > sizeof(T)) {
        for (int k = 0; k < 9; ++k) { QI[k] = (TC)a.Qgd[9 * i + k]; QJ[k] = (TC)a.Qgd[9 * j + k]; }
    } else {
        for (int k = 0; k < 9; ++k) { QI[k] = (TC)a.Qg[9 * i + k]; QJ[k] = (TC)a.Qg[9 * j + k]; }
    }
    TC UI[3] = {TC(0), TC(0), TC(0)}, UJ[3] = {TC(0), TC(0), TC(0)};
    if (POL && a.U)
        for (int c = 0; c < 3; ++c) { UI[c] = (TC)a.U[3 * i + c]; UJ[c] = (TC)a.U[3 * j + c]; }
    TC Ath = TC(0), dmp = TC(1);
    bool dmp_live = true;
    const TC pp = (TC)a.ps[sidx], dsv = (TC)a.dsc[sidx];
    if (POL) {
        Ath = pp > TC(0) ? TC(5.0) : (TC)a.thole[i] + (TC)a.thole[j];
        dmp = (TC)a.polsix[i] * (TC)a.polsix[j];
        if (dmp < TC(1e-8)) { dmp = TC(1e-8); dmp_live = false; }
    }
    TC GI[9], GJ[9], dau_au, dau_u;
    pair_eval_pgrad<TC, POL>(dr, QI, QJ, UI, UJ, (TC)a.ms[sidx], pp, dsv, Ath, dmp, (TC)a.kappa, GI, GJ, dau_au, dau_u);
    for (int k = 0; k < 9; ++k) { oi[k] = (double)GI[k]; oj[k] = (double)GJ[k]; }
    oi[9] = oj[9] = dmp_live ? (double)dau_au : 0.0;
    oi[10] = oj[10] = (POL && !(pp > TC(0))) ? (double)dau_u : 0.0;
}

template <typename T, bool POL, int ROWS = ROWS_ALL>
__global__ void __launch_bounds__(128) k_admp_pgrad(PgradArgs<T> g) {
    const PairArgs<T>& a = g.p;
    const int64_t row = launch_row<ROWS>(a);
    int i = -1, j = -1, nb = 0;
    if (row < a.npairs) {
        i = a.pairs[3 * row];
        j = a.pairs[3 * row + 1];
        nb = a.pairs[3 * row + 2];
    }
    const bool valid = (row < a.npairs) && i >= 0 && i < j && j < a.n &&
                       (ROWS == ROWS_ALL || (ROWS == ROWS_UNSCALED) == (nb == 0));
    const int key = valid ? i : -1;
    double oi[11], oj[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) { oi[k] = 0.0; oj[k] = 0.0; }
    if (valid) {
        if (sizeof(T) < sizeof(double) && nb != 0) pgrad_row<double, T, POL>(a, i, j, nb, oi, oj);
        else pgrad_row<T, T, POL>(a, i, j, nb, oi, oj);
    }
    const bool head = seg_head(key);
    const int run = seg_run_id(key);
#pragma unroll
    for (int k = 0; k < 11; ++k) {
        if (!POL && k >= 9) break;
        const double s = seg_sum(oi[k], run);
        if (head && key >= 0) {
            double* dst = k < 9 ? g.dQ + 9 * key + k : (k == 9 ? g.dpa + key : g.dth + key);
            atomicAdd(dst, s);
        }
        if (valid) {
            double* dst = k < 9 ? g.dQ + 9 * j + k : (k == 9 ? g.dpa + j : g.dth + j);
            atomicAdd(dst, oj[k]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Induced-dipole matrix-vector product for the CG solve, atomics-free: a full (both-direction)
// CSR neighbour list, one warp per atom, FP32 pair tensors accumulated in FP64 registers.
//   dE/dU_i += sum_j [udud1 I + (udud0 - udud1) z z^T] U_j      (pme.py:872-878)
// CSR entries pack j in bits 0..27 and the scale index (nbond-1, wrapped) in bits 28..30.
struct CsrArgs {
    int n;
    const int64_t* off;   // [n+1]
    const int32_t* ent;   // packed (j, scale index)
};

__device__ __forceinline__ int scale_index(int nb) {
    int sidx = nb - 1;
    if (sidx < 0) sidx += 6;
    return sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
}

__global__ void k_csr_count(int64_t npairs, const int32_t* pairs, int n, int32_t* deg) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= npairs) return;
    const int i = pairs[3 * r], j = pairs[3 * r + 1];
    if (i < 0 || i >= j || j >= n) return;
    atomicAdd(deg + i, 1);
    atomicAdd(deg + j, 1);
}

__global__ void k_csr_fill(int64_t npairs, const int32_t* pairs, int n, const int64_t* off, int32_t* cursor,
                           int32_t* ent) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= npairs) return;
    const int i = pairs[3 * r], j = pairs[3 * r + 1];
    if (i < 0 || i >= j || j >= n) return;
    const int s = scale_index(pairs[3 * r + 2]);
    const int ki = atomicAdd(cursor + i, 1);
    const int kj = atomicAdd(cursor + j, 1);
    ent[off[i] + ki] = j | (s << 28);
    ent[off[j] + kj] = i | (s << 28);
}

template <typename T>
__global__ void __launch_bounds__(256) k_matvec_csr(PairArgs<T> a, CsrArgs c, double* out) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= c.n) return;
    const int i = w;
    const T D = T(DMFFB_DIELECTRIC);
    BoxT<T> bx;
#pragma unroll
    for (int k = 0; k < 9; ++k) { bx.h[k] = (T)a.boxd.h[k]; bx.hinv[k] = (T)a.boxd.hinv[k]; }
    const T xi = a.pos[4 * i], yi = a.pos[4 * i + 1], zi = a.pos[4 * i + 2];
    const T thi = a.thole[i], psi = a.polsix[i];
    const T kap = a.kappa;
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    const int64_t beg = c.off[i], end = c.off[i + 1];
    for (int64_t k = beg + lane; k < end; k += 32) {
        const int e = c.ent[k];
        const int j = e & 0x0FFFFFFF;
        const int sidx = (e >> 28) & 7;
        T dx = xi - a.pos[4 * j], dy = yi - a.pos[4 * j + 1], dz = zi - a.pos[4 * j + 2];
        pbc_shift(bx, dx, dy, dz, (T*)nullptr);
        const T r2 = dx * dx + dy * dy + dz * dz;
        const T rinv = d_rsqrt(r2);
        const T r = r2 * rinv;
        const T ez0 = dx * rinv, ez1 = dy * rinv, ez2 = dz * rinv;
        const T av = kap * r;
        const T a2 = av * av;
        const T X = T(DMFFB_TWO_OVER_SQRTPI) * d_exp(-a2);
        const T t2 = av * X;
        const T a3X = a2 * t2;
        const T base = d_erfc(av) + t2 + T(2.0 / 3.0) * a3X;
        const T pp = a.ps[sidx], dsv = a.dsc[sidx];
        const T Ath = pp > T(0) ? T(5.0) : thi + a.thole[j];
        T dmp = psi * a.polsix[j];
        dmp = dmp < T(1e-8) ? T(1e-8) : dmp;
        T u = r / dmp;
        u = u < T(1e8) ? u : T(1e8);
        const T au = Ath * u;
        const T ev = au < T(50) ? d_exp(-au) : T(0);
        const T Pc = T(1) + au + T(0.5) * au * au;
        const T Pd0 = Pc + au * au * au * T(0.25);
        const T bd0 = (dsv - T(1)) - dsv * ev * Pd0 + base;
        const T bd1 = (dsv - T(1)) - dsv * ev * Pc + base;
        const T r3 = rinv * rinv * rinv;
        const T udud0 = T(-2.0 / 3.0) * D * r3 * (T(3) * bd0 + a3X);
        const T udud1 = D * r3 * (bd1 - T(2.0 / 3.0) * a3X);
        const double* U = a.U + 3 * j;
        const T u0 = (T)U[0], u1 = (T)U[1], u2 = (T)U[2];
        const T zu = ez0 * u0 + ez1 * u1 + ez2 * u2;
        const T dd = (udud0 - udud1) * zu;
        acc0 += (double)(udud1 * u0 + dd * ez0);
        acc1 += (double)(udud1 * u1 + dd * ez1);
        acc2 += (double)(udud1 * u2 + dd * ez2);
    }
    acc0 = warp_sum(acc0);
    acc1 = warp_sum(acc1);
    acc2 = warp_sum(acc2);
    if (lane == 0) {
        out[3 * i] = acc0;
        out[3 * i + 1] = acc1;
        out[3 * i + 2] = acc2;
    }
}


// Matvec split in two: the pair tensors [udud1, udud0 - udud1, z] of every CSR entry are fixed
// during one dipole solve, so they are evaluated once (k_matvec_coef) and each CG iteration only
// streams them (k_matvec_apply).
template <typename T>
struct MvCoef {
    T c[2];  // udud1, udud0 - udud1 (the pair direction is recomputed from the positions)
};

template <typename T>
__global__ void __launch_bounds__(256) k_matvec_coef(PairArgs<T> a, CsrArgs c, MvCoef<T>* coef) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= c.n) return;
    const int i = w;
    const T D = T(DMFFB_DIELECTRIC);
    BoxT<T> bx;
#pragma unroll
    for (int k = 0; k < 9; ++k) { bx.h[k] = (T)a.boxd.h[k]; bx.hinv[k] = (T)a.boxd.hinv[k]; }
    const T xi = a.pos[4 * i], yi = a.pos[4 * i + 1], zi = a.pos[4 * i + 2];
    const T thi = a.thole[i], psi = a.polsix[i];
    const T kap = a.kappa;
    const int64_t beg = c.off[i], end = c.off[i + 1];
    for (int64_t k = beg + lane; k < end; k += 32) {
        const int e = c.ent[k];
        const int j = e & 0x0FFFFFFF;
        const int sidx = (e >> 28) & 7;
        T dx = xi - a.pos[4 * j], dy = yi - a.pos[4 * j + 1], dz = zi - a.pos[4 * j + 2];
        pbc_shift(bx, dx, dy, dz, (T*)nullptr);
        const T r2 = dx * dx + dy * dy + dz * dz;
        const T rinv = d_rsqrt(r2);
        const T r = r2 * rinv;
        const T av = kap * r;
        const T a2 = av * av;
        const T X = T(DMFFB_TWO_OVER_SQRTPI) * d_exp(-a2);
        const T t2 = av * X;
        const T a3X = a2 * t2;
        const T base = d_erfc(av) + t2 + T(2.0 / 3.0) * a3X;
        const T pp = a.ps[sidx], dsv = a.dsc[sidx];
        const T Ath = pp > T(0) ? T(5.0) : thi + a.thole[j];
        T dmp = psi * a.polsix[j];
        dmp = dmp < T(1e-8) ? T(1e-8) : dmp;
        T u = r / dmp;
        u = u < T(1e8) ? u : T(1e8);
        const T au = Ath * u;
        const T ev = au < T(50) ? d_exp(-au) : T(0);
        const T Pc = T(1) + au + T(0.5) * au * au;
        const T Pd0 = Pc + au * au * au * T(0.25);
        const T bd0 = (dsv - T(1)) - dsv * ev * Pd0 + base;
        const T bd1 = (dsv - T(1)) - dsv * ev * Pc + base;
        const T r3 = rinv * rinv * rinv;
        const T udud0 = T(-2.0 / 3.0) * D * r3 * (T(3) * bd0 + a3X);
        const T udud1 = D * r3 * (bd1 - T(2.0 / 3.0) * a3X);
        MvCoef<T> cf;
        cf.c[0] = udud1;
        cf.c[1] = udud0 - udud1;
        coef[k] = cf;
    }
}

// The CG matvec streams 12 bytes per CSR entry (packed j + two coefficients); the pair
// direction z is recomputed from the positions, which like U stay cache-resident.  One warp per
// atom i: out_i = sum_j A_ij U_j; returns U_i . out_i in lane 0 (0 elsewhere).
template <typename T>
__device__ __forceinline__ double matvec_atom(const CsrArgs& c, const MvCoef<T>* coef, const T* pos4,
                                              const BoxT<T>& bx, const double* U, double* out, int i, int lane) {
    const T xi = pos4[4 * i], yi = pos4[4 * i + 1], zi = pos4[4 * i + 2];
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0;
    const int64_t beg = c.off[i], end = c.off[i + 1];
    for (int64_t k = beg + lane; k < end; k += 32) {
        const int j = c.ent[k] & 0x0FFFFFFF;
        const MvCoef<T> cf = coef[k];
        T dx = xi - pos4[4 * j], dy = yi - pos4[4 * j + 1], dz = zi - pos4[4 * j + 2];
        pbc_shift(bx, dx, dy, dz, (T*)nullptr);
        const T rinv = d_rsqrt(dx * dx + dy * dy + dz * dz);
        const T ex = dx * rinv, ey = dy * rinv, ez = dz * rinv;
        const double* Uj = U + 3 * j;
        const T u0 = (T)Uj[0], u1 = (T)Uj[1], u2 = (T)Uj[2];
        const T dd = cf.c[1] * (ex * u0 + ey * u1 + ez * u2);
        acc0 += (double)(cf.c[0] * u0 + dd * ex);
        acc1 += (double)(cf.c[0] * u1 + dd * ey);
        acc2 += (double)(cf.c[0] * u2 + dd * ez);
    }
    acc0 = warp_sum(acc0);
    acc1 = warp_sum(acc1);
    acc2 = warp_sum(acc2);
    if (lane != 0) return 0.0;
    out[3 * i] = acc0;
    out[3 * i + 1] = acc1;
    out[3 * i + 2] = acc2;
    return U[3 * i] * acc0 + U[3 * i + 1] * acc1 + U[3 * i + 2] * acc2;
}

// With dot_out, sum_i U_i . out_i is reduced into *dot_out.
template <typename T>
__global__ void __launch_bounds__(256) k_matvec_apply(CsrArgs c, const MvCoef<T>* coef, const T* pos4, BoxT<T> bx,
                                                      const double* U, double* out, double* dot_out = nullptr) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const bool active = w < c.n;
    if (!active && !dot_out) return;
    double d[1] = {0.0};
    if (active) d[0] = matvec_atom<T>(c, coef, pos4, bx, U, out, w, lane);
    if (dot_out) block_reduce_add<1>(d, dot_out);
}

}  // namespace dmffb
