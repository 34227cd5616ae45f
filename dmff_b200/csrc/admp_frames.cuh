// Local frames, multipole rotation, self terms and the frame chain rule (sm_100a, FP64).
//
// Frame construction follows dmff/admp/spatial.py:44-156 (ZThenX, Bisector, ZBisect,
// ThreeFold, ZOnly, NoAxisType) and the rotation multipole.py:129-236.  The reference gets
// the forces on axis atoms from autodiff through the frame; here each atom's accumulated
// multipole torque tau (dE = tau . omega for a rigid rotation omega of its frame) is mapped
// onto its axis atoms: omega = z x dz + (y . dx) z, where dz, dx are the frame axes'
// derivatives along one position coordinate, evaluated by forward-mode (value, tangent)
// arithmetic with one tangent per call so the kernel stays small.
#pragma once
#include "common.cuh"
#include "admp_real.cuh"

namespace dmffb {

struct D1 {
    double v, d;
};
__device__ __forceinline__ D1 operator+(D1 a, D1 b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ D1 operator-(D1 a, D1 b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ D1 operator*(D1 a, D1 b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }

struct V3D {
    D1 x, y, z;
};
__device__ __forceinline__ V3D vadd(V3D a, V3D b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3D vsub(V3D a, V3D b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3D vscale(V3D a, D1 s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D1 vdot(V3D a, V3D b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3D vnorm(V3D a) {
    D1 n2 = vdot(a, a);
    double inv = 1.0 / sqrt(n2.v);
    D1 s = {inv, -0.5 * n2.d * inv * inv * inv};
    return vscale(a, s);
}
__device__ __forceinline__ V3D vcross(V3D a, V3D b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// p_b - p_a shifted to the minimum image (spatial.py:14-32); the image is a constant of motion
__device__ __forceinline__ V3D pbc_vec(const Box& bx, V3D pa, V3D pb, double n[3]) {
    V3D d = vsub(pb, pa);
    double s0 = d.x.v * bx.hinv[0] + d.y.v * bx.hinv[3] + d.z.v * bx.hinv[6];
    double s1 = d.x.v * bx.hinv[1] + d.y.v * bx.hinv[4] + d.z.v * bx.hinv[7];
    double s2 = d.x.v * bx.hinv[2] + d.y.v * bx.hinv[5] + d.z.v * bx.hinv[8];
    n[0] = floor(s0 + 0.5);
    n[1] = floor(s1 + 0.5);
    n[2] = floor(s2 + 0.5);
    d.x.v -= n[0] * bx.h[0] + n[1] * bx.h[3] + n[2] * bx.h[6];
    d.y.v -= n[0] * bx.h[1] + n[1] * bx.h[4] + n[2] * bx.h[7];
    d.z.v -= n[0] * bx.h[2] + n[1] * bx.h[5] + n[2] * bx.h[8];
    return d;
}

struct FrameArgs {
    int n;
    const double* pos;        // [n*3]
    const int32_t* axis_type;  // [n]
    const int32_t* axis_idx;   // [n*3]
    Box box;
};

// frame of atom a with an optional tangent on (slot, coord); slots 0=a 1=z 2=x 3=y.
// Returns false for NoAxisType.  nimg[slot-1][3] receives the image of each axis vector.
__device__ __forceinline__ bool build_frame(const FrameArgs& f, int a, int tslot, int tc, V3D& X, V3D& Y, V3D& Z,
                                            double nimg[3][3]) {
    const int type = f.axis_type[a];
    const int ids[4] = {a, f.axis_idx[3 * a], f.axis_idx[3 * a + 1], f.axis_idx[3 * a + 2]};
    if (type == 5) return false;
    V3D P[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        int id = ids[s] >= 0 ? ids[s] : a;
        P[s].x = {f.pos[3 * id], (tslot == s && tc == 0) ? 1.0 : 0.0};
        P[s].y = {f.pos[3 * id + 1], (tslot == s && tc == 1) ? 1.0 : 0.0};
        P[s].z = {f.pos[3 * id + 2], (tslot == s && tc == 2) ? 1.0 : 0.0};
    }
    V3D vz = vnorm(pbc_vec(f.box, P[0], P[1], nimg[0]));
    V3D vx;
    if (type == 4) {  // ZOnly: lab axis (spatial.py:101-104)
        double r = rint(fabs(vz.x.v));
        vx = {{1.0 - r, 0.0}, {r, 0.0}, {0.0, 0.0}};
        nimg[1][0] = nimg[1][1] = nimg[1][2] = 0.0;
    } else {
        vx = vnorm(pbc_vec(f.box, P[0], P[2], nimg[1]));
    }
    nimg[2][0] = nimg[2][1] = nimg[2][2] = 0.0;
    if (type == 1) vz = vnorm(vadd(vz, vx));
    if (type == 2 || type == 3) {
        V3D vy = vnorm(pbc_vec(f.box, P[0], P[3], nimg[2]));
        if (type == 2) vx = vnorm(vadd(vx, vy));
        else vz = vnorm(vadd(vadd(vz, vx), vy));
    }
    D1 xz = vdot(vx, vz);
    X = vnorm(vsub(vx, vscale(vz, xz)));
    Z = vz;
    Y = vcross(Z, X);
    return true;
}

template <typename T>
struct PrepArgs {
    FrameArgs f;
    const double* Qloc;  // [n*9] local harmonic multipoles
    int lmax;
    T* posT;             // [n*4]
    T* QgT;              // [n*9]
    double* Qg;          // [n*9]
};

// positions in kernel precision, local frames, and Q_global = rot_local2global(Q_local)
template <typename T>
__global__ void k_prepare(PrepArgs<T> a) {
    const int at = blockIdx.x * blockDim.x + threadIdx.x;
    if (at >= a.f.n) return;
    const double* p = a.f.pos + 3 * at;
    a.posT[4 * at] = (T)p[0];
    a.posT[4 * at + 1] = (T)p[1];
    a.posT[4 * at + 2] = (T)p[2];
    a.posT[4 * at + 3] = T(0);
    double Q[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) Q[k] = a.Qloc[9 * at + k];
    double q[9];
    if (a.lmax == 0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) q[k] = (k == 0) ? Q[0] : 0.0;
    } else {
        V3D X, Y, Z;
        double nimg[3][3];
        double F[3][3];
        if (build_frame(a.f, at, -1, 0, X, Y, Z, nimg)) {
            F[0][0] = X.x.v; F[0][1] = X.y.v; F[0][2] = X.z.v;
            F[1][0] = Y.x.v; F[1][1] = Y.y.v; F[1][2] = Y.z.v;
            F[2][0] = Z.x.v; F[2][1] = Z.y.v; F[2][2] = Z.z.v;
        } else {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) F[r][c] = r == c ? 1.0 : 0.0;
        }
        // local -> global = rotate with the transposed frame (multipole.py:218-236)
        const double ex[3] = {F[0][0], F[1][0], F[2][0]};
        const double ey[3] = {F[0][1], F[1][1], F[2][1]};
        const double ez[3] = {F[0][2], F[1][2], F[2][2]};
        double C[5][5];
        quad_rot<double>(ex, ey, ez, C);
        rot9<double>(Q, ex, ey, ez, C, q);
        if (a.lmax < 2) for (int k = 4; k < 9; ++k) q[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        a.Qg[9 * at + k] = q[k];
        a.QgT[9 * at + k] = (T)q[k];
    }
}

template <typename T>
struct SelfArgs {
    FrameArgs f;
    const double* Qg;     // [n*9]
    const double* U;      // [n*3] or null
    const double* pol;    // [n] or null
    const T* torque;      // [n*3] accumulated torques (real + recip)
    double kappa;
    int lmax_eff;
    int lpme;
    int want_box;
    double* grad;         // [n*3] += frame forces
    double* scal;         // [0] E_self, [1] E_pol, [2..10] box grad (frames)
    double* tau_out;      // [n*3] total torque (may be null)
};

// self energy (pme.py:1183-1222), polarization penalty (pme.py:1225-1240), torque -> forces
// One thread per (atom, frame slot s, component c): 12 per atom.  Thread (at, 0, 0) also adds the
// Ewald self energy and the polarization penalty and writes tau_out; every thread forms the
// atom's torque (permanent + self term) and maps it onto the force on the slot's atom along c
// through the derivative of the local frame (build_frame's forward mode), so the twelve frame
// derivatives of an atom run in parallel instead of in one thread.
constexpr int kSelfTasks = 12;

template <typename T>
__global__ void __launch_bounds__(128) k_self_frames(SelfArgs<T> a) {
    const int64_t task = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int at = (int)(task / kSelfTasks), sc = (int)(task - (int64_t)at * kSelfTasks);
    const int s = sc / 3, c = sc - 3 * (sc / 3);
    double red[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) red[k] = 0.0;
    if (at < a.f.n) {
        const double D = DMFFB_DIELECTRIC;
        double Ux = 0, Uy = 0, Uz = 0;
        if (a.U) { Ux = a.U[3 * at]; Uy = a.U[3 * at + 1]; Uz = a.U[3 * at + 2]; }
        double tau[3] = {(double)a.torque[3 * at], (double)a.torque[3 * at + 1], (double)a.torque[3 * at + 2]};
        if (a.lpme) {
            const double k = a.kappa;
            const double f0 = k / 1.7724538509055159;
            const double f1 = f0 * 2.0 * k * k / 3.0;
            const double f2 = f0 * 4.0 * k * k * k * k / 15.0;
            if (sc == 0) {
                double Qt[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) Qt[q] = a.Qg[9 * at + q];
                Qt[1] += Uz; Qt[2] += Ux; Qt[3] += Uy;
                double e = f0 * Qt[0] * Qt[0];
                if (a.lmax_eff >= 1) e += f1 * (Qt[1] * Qt[1] + Qt[2] * Qt[2] + Qt[3] * Qt[3]);
                if (a.lmax_eff >= 2) e += f2 * (Qt[4] * Qt[4] + Qt[5] * Qt[5] + Qt[6] * Qt[6] + Qt[7] * Qt[7] + Qt[8] * Qt[8]);
                red[0] = -D * e;
            }
            // torque of the self term: mu_perm x (-2 D f1 (mu_perm + U))  = -2 D f1 mu_perm x U
            const double mx = a.Qg[9 * at + 2], my = a.Qg[9 * at + 3], mz = a.Qg[9 * at + 1];
            const double sf = -2.0 * D * f1;
            tau[0] += sf * (my * Uz - mz * Uy);
            tau[1] += sf * (mz * Ux - mx * Uz);
            tau[2] += sf * (mx * Uy - my * Ux);
        }
        if (sc == 0) {
            if (a.U && a.pol) {
                double p = a.pol[at];
                p = p < 1e-8 ? 1e-8 : p;
                red[1] = D * 0.5 / p * (Ux * Ux + Uy * Uy + Uz * Uz);
            }
            if (a.tau_out) { a.tau_out[3 * at] = tau[0]; a.tau_out[3 * at + 1] = tau[1]; a.tau_out[3 * at + 2] = tau[2]; }
        }
        if (a.lmax_eff >= 1 && a.f.axis_type[at] != 5 && a.f.axis_idx) {
            const int type = a.f.axis_type[at];
            const int nslot = (type == 2 || type == 3) ? 4 : (type == 4 ? 2 : 3);
            if (s < nslot) {
                const int atom = s == 0 ? at : a.f.axis_idx[3 * at + s - 1];
                double nimg[3][3];
                V3D X, Y, Z;
                build_frame(a.f, at, s, c, X, Y, Z, nimg);
                // omega = z x dz + (y . dx) z
                const double zx = Z.x.v, zy = Z.y.v, zz = Z.z.v;
                const double dzx = Z.x.d, dzy = Z.y.d, dzz = Z.z.d;
                const double ydx = Y.x.v * X.x.d + Y.y.v * X.y.d + Y.z.v * X.z.d;
                const double om0 = zy * dzz - zz * dzy + ydx * zx;
                const double om1 = zz * dzx - zx * dzz + ydx * zy;
                const double om2 = zx * dzy - zy * dzx + ydx * zz;
                const double g = tau[0] * om0 + tau[1] * om1 + tau[2] * om2;
                atomicAdd(a.grad + 3 * atom + c, g);
                if (a.want_box && s > 0)
                    for (int k = 0; k < 3; ++k) red[2 + 3 * k + c] += -nimg[s - 1][k] * g;
            }
        }
    }
    block_reduce_add<11>(red, a.scal);
}

// Per-atom end of the parameter adjoints (after the pair pass and the reciprocal gather have
// accumulated dE/dQ_global into dQ): the Ewald self term's -2 D f_l (Q + U) (pme.py:1183-1222),
// dE/dpol from the penalty D |U|^2 / (2 pol) (pme.py:1225-1240, zero where pol is clamped at 1e-8)
// plus the pair damping sum dpa (-dpa / (6 pol)), and dE/dQ_local as the transpose of the
// local -> global rotation k_prepare applies (rot_local2global, multipole.py:218-236).
struct LocalGradArgs {
    FrameArgs f;
    const double* Qg;     // [n*9]
    const double* U;      // [n*3] or null
    const double* pol;    // [n] or null
    const double* dpa;    // [n] or null
    double kappa;
    int lmax, lmax_eff, lpme;
    double* dQ;           // [n*9] in: dE/dQ_global (pair + reciprocal), out: + self
    double* dQloc;        // [n*9] out: dE/dQ_local
    double* dpol;         // [n] out (may be null)
};

__global__ void __launch_bounds__(128) k_local_grad(LocalGradArgs a) {
    const int at = blockIdx.x * blockDim.x + threadIdx.x;
    if (at >= a.f.n) return;
    const double D = DMFFB_DIELECTRIC;
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = a.dQ[9 * at + k];
    double Ux = 0, Uy = 0, Uz = 0;
    if (a.U) { Ux = a.U[3 * at]; Uy = a.U[3 * at + 1]; Uz = a.U[3 * at + 2]; }
    if (a.lpme) {
        const double k = a.kappa;
        const double f0 = k / 1.7724538509055159;
        const double f1 = f0 * 2.0 * k * k / 3.0;
        const double f2 = f0 * 4.0 * k * k * k * k / 15.0;
        double Qt[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) Qt[q] = a.Qg[9 * at + q];
        Qt[1] += Uz; Qt[2] += Ux; Qt[3] += Uy;
        g[0] += -2.0 * D * f0 * Qt[0];
        if (a.lmax_eff >= 1)
            for (int q = 1; q < 4; ++q) g[q] += -2.0 * D * f1 * Qt[q];
        if (a.lmax_eff >= 2)
            for (int q = 4; q < 9; ++q) g[q] += -2.0 * D * f2 * Qt[q];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) a.dQ[9 * at + k] = g[k];
    if (a.dpol) {
        const double p = a.pol ? a.pol[at] : 0.0;
        double d = 0.0;
        if (a.U && p >= 1e-8) d += -0.5 * D * (Ux * Ux + Uy * Uy + Uz * Uz) / (p * p);
        if (a.dpa && p > 0.0) d += -a.dpa[at] / (6.0 * p);
        a.dpol[at] = d;
    }
    double gl[9];
    if (a.lmax == 0) {
        for (int k = 0; k < 9; ++k) gl[k] = k == 0 ? g[0] : 0.0;
    } else {
        V3D X, Y, Z;
        double nimg[3][3];
        double F[3][3];
        if (build_frame(a.f, at, -1, 0, X, Y, Z, nimg)) {
            F[0][0] = X.x.v; F[0][1] = X.y.v; F[0][2] = X.z.v;
            F[1][0] = Y.x.v; F[1][1] = Y.y.v; F[1][2] = Y.z.v;
            F[2][0] = Z.x.v; F[2][1] = Z.y.v; F[2][2] = Z.z.v;
        } else {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) F[r][c] = r == c ? 1.0 : 0.0;
        }
        const double ex[3] = {F[0][0], F[1][0], F[2][0]};
        const double ey[3] = {F[0][1], F[1][1], F[2][1]};
        const double ez[3] = {F[0][2], F[1][2], F[2][2]};
        double C[5][5];
        quad_rot<double>(ex, ey, ez, C);
        rot9T<double>(g, ex, ey, ez, C, gl);
        if (a.lmax < 2) for (int k = 4; k < 9; ++k) gl[k] = 0.0;
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) a.dQloc[9 * at + k] = gl[k];
}

// forces = -(pair gradient + everything accumulated in FP64)
template <typename T>
__global__ void k_finalize_forces(int n, const T* gpair, const double* gd, double* forces) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    forces[k] = -((double)gpair[k] + gd[k]);
}

}  // namespace dmffb
