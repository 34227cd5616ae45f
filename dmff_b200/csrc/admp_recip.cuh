// Reciprocal-space smooth PME for multipoles up to quadrupoles (sm_100a).
//
// Follows dmff/admp/recip.py:9-471: order-6 cardinal B-splines on a K1 x K2 x K3 mesh, the
// multipole "gradient operator" spread (recip.py:254-349), an FFT, the influence function
// C_k / theta_k^2 (recip.py:438-466, Ck_1 at :474) and the energy sum.  The reference gets
// forces by autodiff; here the gather is explicit: the convolved mesh phi is interpolated
// with B-spline derivatives up to third order (20 sums per atom), giving dE/dpos, dE/dQ,
// torques and the box gradient in one pass.
//
// Layout: each atom's 6x6x6 stencil is split into 36 (x, y) lines of 6 contiguous z points;
// one warp owns one atom, lanes own lines.  The multipole is first mapped to mesh-derivative
// coefficients c_abc (mu^u = -B mu, Theta^u = B Theta B^T with B the reference's derivative
// operator, recip.py:213/251), so the per-point work is a 3-term dot product.  Spreading uses
// FP32/FP64 atomics on the mesh (it lives in L2); the gather is atomics-free.
#pragma once
#include "common.cuh"

namespace dmffb {

struct MeshGeom {
    double NA[9];   // grid coordinates x_j = sum_c NA[j][c] R_c  (NA = diag(K) h^-T)
    double B[9];    // derivative operator used by the reference: B = NA^T
    int K[3];
};

// order-6 B-spline values and derivatives at u = w + j, j = 0..5, w in [0, 1]
template <typename T>
__device__ __forceinline__ void bspline6(T w, T M0[6], T M1[6], T M2[6], T M3[6]) {
    T m2[2] = {w, T(1) - w};
    T m3[3], m4[4], m5[5];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        T a = j < 2 ? m2[j] : T(0);
        T b = j > 0 ? m2[j - 1] : T(0);
        m3[j] = ((w + T(j)) * a + (T(3) - w - T(j)) * b) * T(0.5);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        T a = j < 3 ? m3[j] : T(0);
        T b = j > 0 ? m3[j - 1] : T(0);
        m4[j] = ((w + T(j)) * a + (T(4) - w - T(j)) * b) * T(1.0 / 3.0);
    }
#pragma unroll
    for (int j = 0; j < 5; ++j) {
        T a = j < 4 ? m4[j] : T(0);
        T b = j > 0 ? m4[j - 1] : T(0);
        m5[j] = ((w + T(j)) * a + (T(5) - w - T(j)) * b) * T(0.25);
    }
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        T a = j < 5 ? m5[j] : T(0);
        T b = j > 0 ? m5[j - 1] : T(0);
        M0[j] = ((w + T(j)) * a + (T(6) - w - T(j)) * b) * T(0.2);
        M1[j] = a - b;
        T c0 = j < 4 ? m4[j] : T(0), c1 = (j >= 1 && j - 1 < 4) ? m4[j - 1] : T(0), c2 = j >= 2 ? m4[j - 2] : T(0);
        M2[j] = c0 - T(2) * c1 + c2;
        T e0 = j < 3 ? m3[j] : T(0), e1 = (j >= 1 && j - 1 < 3) ? m3[j - 1] : T(0);
        T e2 = (j >= 2 && j - 2 < 3) ? m3[j - 2] : T(0), e3 = j >= 3 ? m3[j - 3] : T(0);
        M3[j] = e0 - T(3) * e1 + T(3) * e2 - e3;
    }
}

__device__ __forceinline__ int wrapi(int g, int K) {
    g %= K;
    return g < 0 ? g + K : g;
}

// mesh-derivative coefficients of one site: c[0]=000, 1..3 = e_x,e_y,e_z, 4..9 = xx,yy,zz,xy,xz,yz
// (second-order entries hold Theta^u_jk summed over both orders for j != k).
template <typename T>
__device__ __forceinline__ void site_coefs(const double* B, T q, const T mu[3], const T Th[3][3], T c[10]) {
    c[0] = q;
#pragma unroll
    for (int j = 0; j < 3; ++j) c[1 + j] = -(T(B[3 * j]) * mu[0] + T(B[3 * j + 1]) * mu[1] + T(B[3 * j + 2]) * mu[2]);
    T BT[3][3];  // (B Theta)
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int d = 0; d < 3; ++d) BT[j][d] = T(B[3 * j]) * Th[0][d] + T(B[3 * j + 1]) * Th[1][d] + T(B[3 * j + 2]) * Th[2][d];
    T Tu[3][3];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int k = 0; k < 3; ++k) Tu[j][k] = BT[j][0] * T(B[3 * k]) + BT[j][1] * T(B[3 * k + 1]) + BT[j][2] * T(B[3 * k + 2]);
    c[4] = Tu[0][0];
    c[5] = Tu[1][1];
    c[6] = Tu[2][2];
    c[7] = Tu[0][1] + Tu[1][0];
    c[8] = Tu[0][2] + Tu[2][0];
    c[9] = Tu[1][2] + Tu[2][1];
}

// harmonic quadrupole (Q4..Q8, recip.py:317-349 with the /3) -> Cartesian coefficient matrix
template <typename T>
__device__ __forceinline__ void quad_cart(const T* Qq, T Th[3][3]) {
    const T s = T(DMFFB_SQRT3 / 6.0);
    Th[2][2] = Qq[0] * T(1.0 / 3.0);
    Th[0][0] = -Qq[0] * T(1.0 / 6.0) + Qq[3] * s;
    Th[1][1] = -Qq[0] * T(1.0 / 6.0) - Qq[3] * s;
    Th[0][2] = Th[2][0] = Qq[1] * s;
    Th[1][2] = Th[2][1] = Qq[2] * s;
    Th[0][1] = Th[1][0] = Qq[4] * s;
}

template <typename T>
struct SpreadArgs {
    int n;
    const double* pos;  // [n*3]
    const T* Qg;        // [n*9] permanent (may be null)
    const double* U;    // [n*3] Cartesian dipoles (may be null)
    const T* q1;        // [n] plain charges for charge-only channels (may be null)
    int lmax;           // 0: charge only, 1: up to dipole, 2: up to quadrupole
    MeshGeom g;
    T* grid;
    int perm_mul;  // warps visit atoms in the order (w * perm_mul) mod n, gcd(perm_mul, n) = 1
    double* zero_scal[3] = {nullptr, nullptr, nullptr};  // scalars thread 0 of block 0 sets to 0 (may be null)
    unsigned long long* ctr_inc = nullptr;                // counter thread 0 of block 0 advances (may be null)
};

template <typename T>
__device__ __forceinline__ void site_multipole(const SpreadArgs<T>& a, int at, T& q, T mu[3], T Th[3][3]) {
    q = T(0);
    mu[0] = mu[1] = mu[2] = T(0);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Th[r][c] = T(0);
    if (a.q1) q = a.q1[at];
    if (a.Qg) {
        const T* Q = a.Qg + 9 * at;
        q += Q[0];
        if (a.lmax >= 1) { mu[0] = Q[2]; mu[1] = Q[3]; mu[2] = Q[1]; }
        if (a.lmax >= 2) quad_cart(Q + 4, Th);
    }
    if (a.U) {
        mu[0] += (T)a.U[3 * at];
        mu[1] += (T)a.U[3 * at + 1];
        mu[2] += (T)a.U[3 * at + 2];
    }
}

template <typename T>
__device__ __forceinline__ void stencil_setup(const MeshGeom& g, const double* pos, int at, int m0[3], T Mx[4][6],
                                              T My[4][6], T Mz[4][6]) {
    const double R0 = pos[3 * at], R1 = pos[3 * at + 1], R2 = pos[3 * at + 2];
    T (*Ms[3])[6] = {Mx, My, Mz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double x = g.NA[3 * d] * R0 + g.NA[3 * d + 1] * R1 + g.NA[3 * d + 2] * R2;
        const double c = ceil(x);
        m0[d] = (int)c;
        bspline6<T>((T)(c - x), Ms[d][0], Ms[d][1], Ms[d][2], Ms[d][3]);
    }
}

// one warp per site; lanes cover the 36 (x, y) lines of the 6^3 stencil
template <typename T>
__global__ void __launch_bounds__(256) k_spread(SpreadArgs<T> a) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= a.n) return;
    // concurrently running warps take atoms far apart in the box, which keeps them off the same
    // mesh addresses (atoms are usually stored in spatial order)
    const int at = (int)(((int64_t)warp * a.perm_mul) % a.n);
    int m0[3];
    T Mx[4][6], My[4][6], Mz[4][6];
    stencil_setup<T>(a.g, a.pos, at, m0, Mx, My, Mz);
    T q, mu[3], Th[3][3];
    site_multipole(a, at, q, mu, Th);
    T c[10];
    site_coefs<T>(a.g.B, q, mu, Th, c);
    const int K0 = a.g.K[0], K1 = a.g.K[1], K2 = a.g.K[2];
    int gz[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) gz[t] = wrapi(m0[2] - 3 + t, K2);
    for (int L = lane; L < 36; L += 32) {
        const int ix = L / 6, iy = L % 6;
        const T x0 = Mx[0][ix], x1 = Mx[1][ix], x2 = Mx[2][ix];
        const T y0 = My[0][iy], y1 = My[1][iy], y2 = My[2][iy];
        const T s0 = c[0] * x0 * y0 + c[1] * x1 * y0 + c[2] * x0 * y1 + c[4] * x2 * y0 + c[5] * x0 * y2 + c[7] * x1 * y1;
        const T s1 = c[3] * x0 * y0 + c[8] * x1 * y0 + c[9] * x0 * y1;
        const T s2 = c[6] * x0 * y0;
        const int gx = wrapi(m0[0] - 3 + ix, K0), gy = wrapi(m0[1] - 3 + iy, K1);
        T* line = a.grid + ((size_t)gx * K1 + gy) * K2;
#pragma unroll
        for (int t = 0; t < 6; ++t) {
            const T v = s0 * Mz[0][t] + s1 * Mz[1][t] + s2 * Mz[2][t];
            atomicAdd(line + gz[t], v);
        }
    }
}

enum { CK_COUL = 0, CK_DISP6 = 1, CK_DISP8 = 2, CK_DISP10 = 3 };

template <typename T>
struct ConvArgs {
    int K[3];
    int Kh;              // K3/2 + 1
    T* S;                // [K1*K2*Kh] interleaved complex (re, im), overwritten by G*S
    const double* bmod;  // [K1 + K2 + K3] per-dimension B-spline moduli (recip.py:440-448)
    double hinv[9];
    double V;
    double kappa;
    double escale;       // DIELECTRIC for Coulomb, 1 for dispersion
    int kind;
    double* scal;        // [0] energy, [1..6] sum E_k (dlnC/dk2) k k  (xx,yy,zz,xy,xz,yz)
    int want_energy;
    T* zero_real = nullptr;  // real grid of nzero elements the kernel sets to 0 (may be null)
    int64_t nzero = 0;
};

// influence function C(k^2) and d ln C / d k^2
__device__ __forceinline__ void influence(int kind, double ksq, double kappa, double V, double& C, double& dlnC) {
    const double SQRT_PI = 1.7724538509055159;
    const double PI = 3.141592653589793;
    if (kind == CK_COUL) {
        C = 2.0 * PI / V / ksq * exp(-ksq / 4.0 / (kappa * kappa));
        dlnC = -1.0 / ksq - 1.0 / (4.0 * kappa * kappa);
        return;
    }
    // dispersion (recip.py:477-508): ksq thresholded at 1e-16
    const double ks = ksq < 1e-16 ? 1e-16 : ksq;
    const double x2 = ks / 4.0 / (kappa * kappa);
    const double x = sqrt(x2);
    const double ex = exp(-x2);
    const double ec = erfc(x);
    double f, dfdx, pref;
    if (kind == CK_DISP6) {
        const double x3 = x2 * x;
        f = (1 - 2 * x2) * ex + 2 * x3 * SQRT_PI * ec;
        // d/dx: (-4x)e + (1-2x^2)(-2x)e + 6x^2 sqrt(pi) erfc - 2x^3 * 2 e
        dfdx = -4 * x * ex - 2 * x * (1 - 2 * x2) * ex + 6 * x2 * SQRT_PI * ec - 4 * x3 * ex;
        pref = SQRT_PI * PI / 2 / V * kappa * kappa * kappa / 3;
    } else if (kind == CK_DISP8) {
        const double x4 = x2 * x2, x5 = x4 * x;
        f = (3 - 2 * x2 + 4 * x4) * ex - 4 * x5 * SQRT_PI * ec;
        dfdx = (-4 * x + 16 * x2 * x) * ex - 2 * x * (3 - 2 * x2 + 4 * x4) * ex - 20 * x4 * SQRT_PI * ec + 8 * x5 * ex;
        pref = SQRT_PI * PI / 2 / V * pow(kappa, 5) / 45;
    } else {
        const double x4 = x2 * x2, x6 = x4 * x2, x7 = x6 * x;
        f = (15 - 6 * x2 + 4 * x4 - 8 * x6) * ex + 8 * x7 * SQRT_PI * ec;
        dfdx = (-12 * x + 16 * x2 * x - 48 * x4 * x) * ex - 2 * x * (15 - 6 * x2 + 4 * x4 - 8 * x6) * ex + 56 * x6 * SQRT_PI * ec - 16 * x7 * ex;
        pref = SQRT_PI * PI / 2 / V * pow(kappa, 7) / 1260;
    }
    C = pref * f;
    // d/dk2 = dx/dk2 d/dx, x = sqrt(k2)/(2 kappa) -> dx/dk2 = 1/(8 kappa^2 x)
    dlnC = (ksq < 1e-16) ? 0.0 : dfdx / f / (8.0 * kappa * kappa * x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_conv(ConvArgs<T> a) {
    const int64_t total = (int64_t)a.K[0] * a.K[1] * a.Kh;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double red[7] = {0, 0, 0, 0, 0, 0, 0};
    if (idx < total) {
        const int k3 = (int)(idx % a.Kh);
        const int k2 = (int)((idx / a.Kh) % a.K[1]);
        const int k1 = (int)(idx / ((int64_t)a.Kh * a.K[1]));
        const int m1 = k1 < (a.K[0] + 1) / 2 ? k1 : k1 - a.K[0];
        const int m2 = k2 < (a.K[1] + 1) / 2 ? k2 : k2 - a.K[1];
        const int m3 = k3 < (a.K[2] + 1) / 2 ? k3 : k3 - a.K[2];
        const double TWO_PI = 6.283185307179586;
        double kv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) kv[c] = TWO_PI * (a.hinv[3 * c] * m1 + a.hinv[3 * c + 1] * m2 + a.hinv[3 * c + 2] * m3);
        const double ksq = kv[0] * kv[0] + kv[1] * kv[1] + kv[2] * kv[2];
        const double th = a.bmod[k1] * a.bmod[a.K[0] + k2] * a.bmod[a.K[0] + a.K[1] + k3];
        double G = 0.0, dlnC = 0.0;
        const bool zero = (m1 == 0 && m2 == 0 && m3 == 0);
        if (!(zero && a.kind == CK_COUL)) {
            double C;
            influence(a.kind, ksq, a.kappa, a.V, C, dlnC);
            G = C / (th * th);
        }
        T* s = a.S + 2 * idx;
        const double re = (double)s[0], im = (double)s[1];
        if (a.want_energy) {
            const bool self_conj = (k3 == 0) || ((a.K[2] % 2 == 0) && k3 == a.K[2] / 2);
            const double w = self_conj ? 1.0 : 2.0;
            const double Ek = a.escale * w * G * (re * re + im * im);
            red[0] = Ek;
            const double f = Ek * dlnC;
            red[1] = f * kv[0] * kv[0];
            red[2] = f * kv[1] * kv[1];
            red[3] = f * kv[2] * kv[2];
            red[4] = f * kv[0] * kv[1];
            red[5] = f * kv[0] * kv[2];
            red[6] = f * kv[1] * kv[2];
        }
        s[0] = (T)(re * G);
        s[1] = (T)(im * G);
    }
    // the spread input of this pass has been transformed: clear it for the next spread
    for (int64_t i = idx; i < a.nzero; i += (int64_t)gridDim.x * blockDim.x) a.zero_real[i] = T(0);
    if (a.want_energy) block_reduce_add<7>(red, a.scal);
}

enum { GATHER_FULL = 0, GATHER_FIELD = 1 };

template <typename T>
struct GatherArgs {
    int n;
    const double* pos;
    const T* Qg;          // permanent multipoles (torque and coefficients), may be null
    const double* U;      // induced dipoles added to the spread multipole, may be null
    const T* q1;          // plain charges (charge-only channel), may be null
    int lmax;
    MeshGeom g;
    const T* phi;         // convolved mesh (real)
    double scale;         // dE/dmesh = scale * phi   (2*DIELECTRIC or 2)
    double* grad;         // [n*3] += dE/dpos
    T* torque;            // [n*3] += torque of permanent multipoles (may be null)
    double* field;        // [n*3] dE/dU (Cartesian); written (FIELD) or accumulated
    int field_accumulate;
    double* gQ;           // [n*9] += dE/dQ_global (may be null)
    double* dq1;          // [n] += dE/dq for the charge channel (may be null)
    double* scal;         // [0] energy (1/2 sum c P), [1..9] X_NA
    int want_box;
    int mode;
};

template <typename T>
__global__ void __launch_bounds__(256) k_gather(GatherArgs<T> a) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const bool active = warp < a.n;
    const int at = active ? warp : 0;
    int m0[3];
    T Mx[4][6], My[4][6], Mz[4][6];
    stencil_setup<T>(a.g, a.pos, at, m0, Mx, My, Mz);
    const int K0 = a.g.K[0], K1 = a.g.K[1], K2 = a.g.K[2];
    int gz[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) gz[t] = wrapi(m0[2] - 3 + t, K2);
    // partial sums P_abc, a+b+c <= 3, order: index via table below
    // 0:000 1:100 2:010 3:001 4:200 5:020 6:002 7:110 8:101 9:011
    // 10:300 11:030 12:003 13:210 14:201 15:120 16:021 17:102 18:012 19:111
    T P[20];
#pragma unroll
    for (int k = 0; k < 20; ++k) P[k] = T(0);
    const int maxo = (a.mode == GATHER_FIELD) ? 2 : 3;
    if (active) {
        for (int L = lane; L < 36; L += 32) {
            const int ix = L / 6, iy = L % 6;
            const int gx = wrapi(m0[0] - 3 + ix, K0), gy = wrapi(m0[1] - 3 + iy, K1);
            const T* line = a.phi + ((size_t)gx * K1 + gy) * K2;
            T s[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const T v = line[gz[t]];
                s[0] += v * Mz[0][t];
                s[1] += v * Mz[1][t];
                s[2] += v * Mz[2][t];
                s[3] += v * Mz[3][t];
            }
            const T x0 = Mx[0][ix], x1 = Mx[1][ix], x2 = Mx[2][ix], x3 = Mx[3][ix];
            const T y0 = My[0][iy], y1 = My[1][iy], y2 = My[2][iy], y3 = My[3][iy];
            P[0] += x0 * y0 * s[0];
            P[1] += x1 * y0 * s[0];
            P[2] += x0 * y1 * s[0];
            P[3] += x0 * y0 * s[1];
            P[4] += x2 * y0 * s[0];
            P[5] += x0 * y2 * s[0];
            P[6] += x0 * y0 * s[2];
            P[7] += x1 * y1 * s[0];
            P[8] += x1 * y0 * s[1];
            P[9] += x0 * y1 * s[1];
            if (maxo == 3) {
                P[10] += x3 * y0 * s[0];
                P[11] += x0 * y3 * s[0];
                P[12] += x0 * y0 * s[3];
                P[13] += x2 * y1 * s[0];
                P[14] += x2 * y0 * s[1];
                P[15] += x1 * y2 * s[0];
                P[16] += x0 * y2 * s[1];
                P[17] += x1 * y0 * s[2];
                P[18] += x0 * y1 * s[2];
                P[19] += x1 * y1 * s[1];
            }
        }
    }
    // reduce only the sums this mode uses (field: first derivatives; full: all 20)
    if (maxo == 2) {
#pragma unroll
        for (int k = 1; k < 4; ++k) P[k] = warp_sum(P[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 20; ++k) P[k] = warp_sum(P[k]);
    }

    double red[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) red[k] = 0.0;
    if (active && lane == 0) {
        const double sc = a.scale;
        double Pd[20];
#pragma unroll
        for (int k = 0; k < 20; ++k) Pd[k] = sc * (double)P[k];
        // site multipole (the one that was spread)
        SpreadArgs<T> sa;
        sa.Qg = a.Qg; sa.U = a.U; sa.q1 = a.q1; sa.lmax = a.lmax;
        T q, mu[3], Th[3][3];
        site_multipole(sa, at, q, mu, Th);
        T cT[10];
        site_coefs<T>(a.g.B, q, mu, Th, cT);
        double c[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) c[k] = (double)cT[k];
        const double* B = a.g.B;
        // dE/dmu^u_j and dE/dTheta^u_jk
        const double Pu[3] = {Pd[1], Pd[2], Pd[3]};
        const double P2[3][3] = {{Pd[4], Pd[7], Pd[8]}, {Pd[7], Pd[5], Pd[9]}, {Pd[8], Pd[9], Pd[6]}};
        double dmu[3];
#pragma unroll
        for (int cc = 0; cc < 3; ++cc) dmu[cc] = -(Pu[0] * B[cc] + Pu[1] * B[3 + cc] + Pu[2] * B[6 + cc]);
        if (a.mode == GATHER_FIELD) {
            double* f = a.field + 3 * at;
            if (a.field_accumulate) { f[0] += dmu[0]; f[1] += dmu[1]; f[2] += dmu[2]; }
            else { f[0] = dmu[0]; f[1] = dmu[1]; f[2] = dmu[2]; }
        } else {
            // dE/dx_j = -sum_abc c_abc P_{abc + e_j}
            // coefficient -> (a,b,c) exponents; index of abc+e_j in P
            const int up[10][3] = {{1, 2, 3},   {4, 7, 8},   {7, 5, 9},   {8, 9, 6},    {10, 13, 14},
                                   {15, 11, 16}, {17, 18, 12}, {13, 15, 19}, {14, 19, 17}, {19, 16, 18}};
            double Y[3] = {0, 0, 0};
#pragma unroll
            for (int k = 0; k < 10; ++k)
#pragma unroll
                for (int j = 0; j < 3; ++j) Y[j] -= c[k] * Pd[up[k][j]];
            double* gr = a.grad + 3 * at;
            const double* NA = a.g.NA;
#pragma unroll
            for (int cc = 0; cc < 3; ++cc) gr[cc] += NA[cc] * Y[0] + NA[3 + cc] * Y[1] + NA[6 + cc] * Y[2];
            double e = 0.0;
#pragma unroll
            for (int k = 0; k < 10; ++k) e += c[k] * Pd[k];
            red[0] = 0.5 * e;
            // dE/dTheta (Cartesian) = B^T P2 B
            double BP[3][3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int k = 0; k < 3; ++k) BP[cc][k] = B[cc] * P2[0][k] + B[3 + cc] * P2[1][k] + B[6 + cc] * P2[2][k];
            double dTh[3][3];
#pragma unroll
            for (int cc = 0; cc < 3; ++cc)
#pragma unroll
                for (int d = 0; d < 3; ++d) dTh[cc][d] = BP[cc][0] * B[d] + BP[cc][1] * B[3 + d] + BP[cc][2] * B[6 + d];
            double g[9];
            g[0] = Pd[0];
            g[1] = dmu[2];
            g[2] = dmu[0];
            g[3] = dmu[1];
            const double s6 = DMFFB_SQRT3 / 6.0;
            g[4] = dTh[2][2] / 3.0 - dTh[0][0] / 6.0 - dTh[1][1] / 6.0;
            g[5] = (dTh[0][2] + dTh[2][0]) * s6;
            g[6] = (dTh[1][2] + dTh[2][1]) * s6;
            g[7] = (dTh[0][0] - dTh[1][1]) * s6;
            g[8] = (dTh[0][1] + dTh[1][0]) * s6;
            if (a.field) {
                double* f = a.field + 3 * at;
                if (a.field_accumulate) { f[0] += dmu[0]; f[1] += dmu[1]; f[2] += dmu[2]; }
                else { f[0] = dmu[0]; f[1] = dmu[1]; f[2] = dmu[2]; }
            }
            if (a.gQ) {
#pragma unroll
                for (int k = 0; k < 9; ++k) a.gQ[9 * at + k] += g[k];
            }
            if (a.dq1) a.dq1[at] += g[0];
            if (a.torque && a.Qg) {
                T qp[9], gT[9], t[3];
#pragma unroll
                for (int k = 0; k < 9; ++k) { qp[k] = a.Qg[9 * at + k]; gT[k] = (T)g[k]; }
                if (a.lmax < 2) { for (int k = 4; k < 9; ++k) qp[k] = T(0); }
                if (a.lmax < 1) { qp[1] = qp[2] = qp[3] = T(0); }
                torque9(qp, gT, t);
                // atomics: the real-space FULL pass may add to the same torques concurrently
                atomicAdd(a.torque + 3 * at, t[0]);
                atomicAdd(a.torque + 3 * at + 1, t[1]);
                atomicAdd(a.torque + 3 * at + 2, t[2]);
            }
            if (a.want_box) {
                // X_NA = Y (x) R + (dE/dB)^T,  dE/dB = -Pu (x) mu + 2 P2 B Theta
                const double R[3] = {a.pos[3 * at], a.pos[3 * at + 1], a.pos[3 * at + 2]};
                double PB[3][3];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int k = 0; k < 3; ++k) PB[j][k] = P2[j][0] * B[k] + P2[j][1] * B[3 + k] + P2[j][2] * B[6 + k];
#pragma unroll
                for (int j = 0; j < 3; ++j)
#pragma unroll
                    for (int cc = 0; cc < 3; ++cc) {
                        double dB = -Pu[j] * (double)mu[cc];
                        dB += 2.0 * (PB[j][0] * (double)Th[0][cc] + PB[j][1] * (double)Th[1][cc] + PB[j][2] * (double)Th[2][cc]);
                        // (dE/dB)^T[cc][j] adds to X_NA[cc][j]; Y (x) R adds to X_NA[j][cc]
                        red[1 + 3 * cc + j] += dB;
                        red[1 + 3 * j + cc] += Y[j] * R[cc];
                    }
            }
        }
    }
    if (a.mode == GATHER_FULL) block_reduce_add<10>(red, a.scal);
}


// ---------------------------------------------------------------------------------------------
// Lean kernels for the CG loop, where only induced dipoles are spread and only the first
// derivatives of the convolved mesh are gathered: value + first-derivative splines, 3 mesh
// coefficients, 3 sums; small register footprint for occupancy.
template <typename T>
__device__ __forceinline__ void bspline6_01(T w, T M0[6], T M1[6]) {
    T m2[2] = {w, T(1) - w};
    T m3[3], m4[4], m5[5];
#pragma unroll
    for (int j = 0; j < 3; ++j)
        m3[j] = ((w + T(j)) * (j < 2 ? m2[j] : T(0)) + (T(3) - w - T(j)) * (j > 0 ? m2[j - 1] : T(0))) * T(0.5);
#pragma unroll
    for (int j = 0; j < 4; ++j)
        m4[j] = ((w + T(j)) * (j < 3 ? m3[j] : T(0)) + (T(4) - w - T(j)) * (j > 0 ? m3[j - 1] : T(0))) * T(1.0 / 3.0);
#pragma unroll
    for (int j = 0; j < 5; ++j)
        m5[j] = ((w + T(j)) * (j < 4 ? m4[j] : T(0)) + (T(5) - w - T(j)) * (j > 0 ? m4[j - 1] : T(0))) * T(0.25);
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const T a = j < 5 ? m5[j] : T(0), b = j > 0 ? m5[j - 1] : T(0);
        M0[j] = ((w + T(j)) * a + (T(6) - w - T(j)) * b) * T(0.2);
        M1[j] = a - b;
    }
}

template <typename T>
__device__ __forceinline__ void stencil01(const MeshGeom& g, const double* pos, int at, int m0[3], T Mx[2][6],
                                          T My[2][6], T Mz[2][6]) {
    const double R0 = pos[3 * at], R1 = pos[3 * at + 1], R2 = pos[3 * at + 2];
    T (*Ms[3])[6] = {Mx, My, Mz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double x = g.NA[3 * d] * R0 + g.NA[3 * d + 1] * R1 + g.NA[3 * d + 2] * R2;
        const double c = ceil(x);
        m0[d] = (int)c;
        bspline6_01<T>((T)(c - x), Ms[d][0], Ms[d][1]);
    }
}

// v[k] for a runtime k in 0..5 without indexing a register array (a select chain keeps the
// stencil in registers instead of the stack)
template <typename T>
__device__ __forceinline__ T sel6(const T v[6], int k) {
    T r = v[0];
#pragma unroll
    for (int t = 1; t < 6; ++t) r = (k == t) ? v[t] : r;
    return r;
}

// dE/dmu (Cartesian) of every site from the convolved mesh: out = scale * (-B^T grad_u phi).
// Lanes take whole (x, y) stencil columns and read their six z points in sequence (one cache
// line, L1 hits after the first); sel6 keeps the column weights in registers.
template <typename T>
__global__ void __launch_bounds__(256) k_gather_field(int n, const double* pos, MeshGeom g, const T* phi, double scale,
                                                      double* out) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n) return;
    const int at = warp;
    int m0[3];
    T Mx[2][6], My[2][6], Mz[2][6];
    stencil01<T>(g, pos, at, m0, Mx, My, Mz);
    const int K0 = g.K[0], K1 = g.K[1], K2 = g.K[2];
    T p1 = T(0), p2 = T(0), p3 = T(0);
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
        const int L = lane + 32 * pass;
        if (L < 36) {
            const int ix = L / 6, iy = L - 6 * ix;
            const int gx = wrapi(m0[0] - 3 + ix, K0), gy = wrapi(m0[1] - 3 + iy, K1);
            const T* line = phi + ((size_t)gx * K1 + gy) * K2;
            int gz = wrapi(m0[2] - 3, K2);
            T s0 = T(0), s1 = T(0);
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const T v = __ldg(line + gz);
                s0 += v * Mz[0][t];
                s1 += v * Mz[1][t];
                gz = (gz + 1 == K2) ? 0 : gz + 1;
            }
            const T mx0 = sel6(Mx[0], ix), mx1 = sel6(Mx[1], ix), my0 = sel6(My[0], iy), my1 = sel6(My[1], iy);
            p1 += mx1 * my0 * s0;
            p2 += mx0 * my1 * s0;
            p3 += mx0 * my0 * s1;
        }
    }
    p1 = warp_sum(p1);
    p2 = warp_sum(p2);
    p3 = warp_sum(p3);
    if (lane == 0) {
        const double* B = g.B;
        const double P1 = scale * (double)p1, P2 = scale * (double)p2, P3 = scale * (double)p3;
#pragma unroll
        for (int c = 0; c < 3; ++c) out[3 * at + c] = -(P1 * B[c] + P2 * B[3 + c] + P3 * B[6 + c]);
    }
}

// ---------------------------------------------------------------------------------------------
// Stencil cache for the CG loop.  Positions are fixed during the dipole solve, so the wrapped
// first stencil point (m0 - 3 per dimension) and the value / first-derivative B-spline weights
// of every atom are computed once per evaluation (k_stencil_prep, with the same arithmetic as
// stencil01) and read by the cached dipole spread and field gather, instead of every lane
// recomputing three spline sets and two integer wraps per pass in every iteration.
// Weights per atom: Mx0[6] Mx1[6] My0[6] My1[6] Mz0[6] Mz1[6].
template <typename T>
struct StencilCache {
    const int4* org;  // wrapped first stencil point per dimension (w unused)
    const T* w;       // [n * 36]
};

// g + d wrapped into [0, K) for g in [0, K), d >= 0
__device__ __forceinline__ int wrap_up(int g, int K) {
    while (g >= K) g -= K;
    return g;
}

template <typename T>
__global__ void __launch_bounds__(256) k_stencil_prep(int n, const double* pos, MeshGeom g, int4* org, T* w) {
    const int at = blockIdx.x * blockDim.x + threadIdx.x;
    if (at >= n) return;
    int m0[3];
    T Mx[2][6], My[2][6], Mz[2][6];
    stencil01<T>(g, pos, at, m0, Mx, My, Mz);
    org[at] = make_int4(wrapi(m0[0] - 3, g.K[0]), wrapi(m0[1] - 3, g.K[1]), wrapi(m0[2] - 3, g.K[2]), 0);
    T* o = w + 36 * (size_t)at;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        o[j] = Mx[0][j];
        o[6 + j] = Mx[1][j];
        o[12 + j] = My[0][j];
        o[18 + j] = My[1][j];
        o[24 + j] = Mz[0][j];
        o[30 + j] = Mz[1][j];
    }
}

// Dipole-only spread of the CG loop from the cached stencil: a warp per atom, lanes 0..29 form
// five groups of six consecutive z points of one (x, y) stencil column; the 36 columns take eight
// passes, so a warp's atomics of one pass touch five runs of six consecutive floats (coalesced in
// L2) instead of 32 scattered addresses.
template <typename T>
__device__ __forceinline__ void spread_dip_atom(const SpreadArgs<T>& a, const StencilCache<T>& st, int warp,
                                                int lane) {
    const int at = (int)(((int64_t)warp * a.perm_mul) % a.n);
    const T mu0 = (T)a.U[3 * at], mu1 = (T)a.U[3 * at + 1], mu2 = (T)a.U[3 * at + 2];
    const int grp = lane / 6, iz = lane - 6 * grp;
    const int4 o = st.org[at];
    const T* w = st.w + 36 * (size_t)at;
    const double* B = a.g.B;
    const T c1 = -(T(B[0]) * mu0 + T(B[1]) * mu1 + T(B[2]) * mu2);
    const T c2 = -(T(B[3]) * mu0 + T(B[4]) * mu1 + T(B[5]) * mu2);
    const T c3 = -(T(B[6]) * mu0 + T(B[7]) * mu1 + T(B[8]) * mu2);
    const int K0 = a.g.K[0], K1 = a.g.K[1], K2 = a.g.K[2];
    // the atom's 36 weights sit in lanes (w[0..31] in wl, w[32..35] in wh of lanes 0..3) and the
    // wrapped mesh bases in lanes 0..5 (x rows times K1) and 6..11 (y columns); the passes read
    // them by shuffles instead of loads and integer wraps
    const T wl = __ldg(w + lane);
    const T wh = lane < 4 ? __ldg(w + 32 + lane) : T(0);
    int base = 0;
    if (lane < 6) base = wrap_up(o.x + lane, K0) * K1;
    else if (lane < 12) base = wrap_up(o.y + lane - 6, K1);
    const int izc = iz < 6 ? iz : 0;
    const T mz0 = __shfl_sync(0xffffffffu, wl, 24 + izc);
    const T mz1a = __shfl_sync(0xffffffffu, wl, (30 + izc) & 31), mz1b = __shfl_sync(0xffffffffu, wh, (izc + 30) & 3);
    const T mz1 = 30 + izc < 32 ? mz1a : mz1b;
    const int gz = wrap_up(o.z + izc, K2);
#pragma unroll
    for (int pass = 0; pass < 8; ++pass) {
        const int col = grp + 5 * pass;
        const int cc = col < 36 ? col : 35;
        const int ix = cc / 6, iy = cc - 6 * ix;
        const T mx0 = __shfl_sync(0xffffffffu, wl, ix), mx1 = __shfl_sync(0xffffffffu, wl, 6 + ix);
        const T my0 = __shfl_sync(0xffffffffu, wl, 12 + iy), my1 = __shfl_sync(0xffffffffu, wl, 18 + iy);
        const int xb = __shfl_sync(0xffffffffu, base, ix), yb = __shfl_sync(0xffffffffu, base, 6 + iy);
        if (grp < 5 && col < 36) {
            const T v = (c1 * mx1 * my0 + c2 * mx0 * my1) * mz0 + c3 * mx0 * my0 * mz1;
            atomicAdd(a.grid + (size_t)(xb + yb) * K2 + gz, v);
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_spread_dip_cached(SpreadArgs<T> a, StencilCache<T> st) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (blockIdx.x == 0 && threadIdx.x < 3 && a.zero_scal[threadIdx.x]) *a.zero_scal[threadIdx.x] = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && a.ctr_inc) *a.ctr_inc += 1ull;
    if (warp >= a.n) return;  // whole warps: every lane takes part in the shuffles
    spread_dip_atom<T>(a, st, warp, lane);
}

// Field terms folded into the gather: out = recip [+ mv] [+ (1/pol + self1) U]; with dot_out,
// sum U . out is reduced into *dot_out; *zero1 is cleared by thread 0 of block 0.
struct FieldCombine {
    const double* mv = nullptr;  // real-space matvec field (may be null)
    const double* U = nullptr;   // dipoles of the diagonal term (null: no diagonal term)
    const double* pol = nullptr;
    double self1 = 0.0;
    double* dot_out = nullptr;
    double* zero1 = nullptr;
    // with ctr: zero_pair[1 - ((*ctr - 1) & 1)] is cleared as well (the r.z slot of the CG step
    // whose counter the spread has just advanced)
    double* zero_pair = nullptr;
    const unsigned long long* ctr = nullptr;
};

// k_gather_field with the cached stencil: lanes own whole (x, y) columns (lanes 0..31, then
// lanes 0..3) and read the column's six z points in sequence (one or two sectors, L1 hits after
// the first), contracting them with the warp-uniform z weights.  One warp per atom; returns
// U_at . out_at in lane 0 when cmb.dot_out is set (0 elsewhere).
template <typename T>
__device__ __forceinline__ double gather_field_atom(const StencilCache<T>& st, const MeshGeom& g, const T* phi,
                                                    double scale, double* out, const FieldCombine& cmb, int at,
                                                    int lane) {
    T p1 = T(0), p2 = T(0), p3 = T(0);
    const int4 o = st.org[at];
    const T* w = st.w + 36 * (size_t)at;
    const int K0 = g.K[0], K1 = g.K[1], K2 = g.K[2];
    T mz0[6], mz1[6];
#pragma unroll
    for (int t = 0; t < 6; ++t) {
        mz0[t] = __ldg(w + 24 + t);
        mz1[t] = __ldg(w + 30 + t);
    }
#pragma unroll
    for (int pass = 0; pass < 2; ++pass) {
        const int L = lane + 32 * pass;
        if (L < 36) {
            const int ix = L / 6, iy = L - 6 * ix;
            const int gx = wrap_up(o.x + ix, K0), gy = wrap_up(o.y + iy, K1);
            const T* line = phi + ((size_t)gx * K1 + gy) * K2;
            int gz = o.z;
            T s0 = T(0), s1 = T(0);
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const T v = line[gz];
                s0 += v * mz0[t];
                s1 += v * mz1[t];
                gz = (gz + 1 == K2) ? 0 : gz + 1;
            }
            const T mx0 = __ldg(w + ix), mx1 = __ldg(w + 6 + ix), my0 = __ldg(w + 12 + iy), my1 = __ldg(w + 18 + iy);
            p1 += mx1 * my0 * s0;
            p2 += mx0 * my1 * s0;
            p3 += mx0 * my0 * s1;
        }
    }
    p1 = warp_sum(p1);
    p2 = warp_sum(p2);
    p3 = warp_sum(p3);
    if (lane != 0) return 0.0;
    const double* B = g.B;
    const double P1 = scale * (double)p1, P2 = scale * (double)p2, P3 = scale * (double)p3;
    double pp = 0.0, d = 0.0;
    if (cmb.U) {
        pp = cmb.pol[at];
        pp = pp < 1e-8 ? 1e-8 : pp;
        pp = DMFFB_DIELECTRIC / pp + cmb.self1;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double v = -(P1 * B[c] + P2 * B[3 + c] + P3 * B[6 + c]);
        if (cmb.mv) v += cmb.mv[3 * at + c];
        if (cmb.U) v += pp * cmb.U[3 * at + c];
        out[3 * at + c] = v;
        if (cmb.dot_out) d += cmb.U[3 * at + c] * v;
    }
    return d;
}

template <typename T>
__global__ void __launch_bounds__(256) k_gather_field_cached(int n, StencilCache<T> st, MeshGeom g, const T* phi,
                                                             double scale, double* out, FieldCombine cmb) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (blockIdx.x == 0 && threadIdx.x == 0 && cmb.zero1) *cmb.zero1 = 0.0;
    if (blockIdx.x == 0 && threadIdx.x == 0 && cmb.zero_pair) cmb.zero_pair[1 - (int)((*cmb.ctr - 1ull) & 1ull)] = 0.0;
    double d[1] = {0.0};
    if (warp < n) d[0] = gather_field_atom<T>(st, g, phi, scale, out, cmb, warp, lane);
    if (cmb.dot_out) block_reduce_add<1>(d, cmb.dot_out);
}

}  // namespace dmffb
