// Dispersion PME real space and Tang-Toennies short range (sm_100a).
//
// Real-space dispersion PME, dmff/admp/disp_pme.py:133-261: for p = 6, 8, 10
//   E_lr += (m + g_p(kappa^2 r^2) - 1) c_i c_j / r^p,  g_6 = (1 + x2 + x2^2/2) e^-x2, g_8 adds
//   x2^3/6 e^-x2, g_10 adds x2^4/24 e^-x2;
// ADMPDispForce short range, dmff/admp/pairwise.py:100-118 (r_b = r in bohr, b = sqrt(b_i b_j)):
//   E_sr += m [2625.5 a e^-b r_b - 2625.5 e^-b r_b (1 + b r_b) q / r_b + f_6(b r_b) c / r^6],
//   f_6 the incomplete exponential sum to (b r_b)^6 / 720.
// One thread per pair row with the ADMP kernel's layout: value+slope arithmetic for dE/dr,
// i-side warp segmented sums, j-side atomics, FP64 energies and box gradient; rows with a
// topological scale run in FP64 (m - 1 + g cancels for excluded pairs).
#pragma once
#include "common.cuh"
#include "admp_real.cuh"

namespace dmffb {

template <typename T>
struct DispArgs {
    int n;
    int64_t npairs;
    const int32_t* pairs;
    const double* pos;   // [n*3] FP64
    const T* c;          // [3][n] channel-major sqrt(C6), sqrt(C8), sqrt(C10) in A units
    const T* a;          // [n] TT (Hartree), may be null
    const T* b;          // [n] TT (1/bohr)
    const T* q;          // [n]
    T ms[6];
    T kappa;
    int pmax;
    Box boxd;
    T* grad_lr;          // [n*3] dE_lr/dpos
    T* grad_sr;          // [n*3] dE_sr/dpos (TT)
    double* scal;        // [0] E_lr real, [1] E_sr, [2..10] box grad lr, [11..19] box grad sr
    double* dlr;         // [3][n] += dE_lr/dc (channel-major), parameter adjoints, or null
    double* dsr;         // [4][n] += dE_sr/d(a, b, q, c6), or null
    const int32_t* rowmap = nullptr;  // ROWS == 2 launches: indices of the rows with nbond != 0
    int64_t nrowmap = 0;
};

// Parameter partials of one pair: dE_lr/dc_i^p and dE_lr/dc_j^p (p = 6, 8, 10; the real-space
// factor (m + g_p - 1) / r^p times the partner's c), and for the TT term dE_sr/d(a, b, q, c6) of
// both sites through a = sqrt(a_i a_j), b = sqrt(b_i b_j), q = q_i q_j, c = c6_i c6_j.  With
// x = b r_b, the truncated exponential sum obeys d/dx [e^-x P6(x)] = -e^-x x^6 / 720.
template <typename TC>
__device__ __forceinline__ void disp_pgrad(TC r, TC m, const TC ci[3], const TC cj[3], TC kap, int pmax, bool tt, TC ai,
                                           TC aj, TC bi, TC bj, TC qi, TC qj, TC li[3], TC lj[3], TC si[4], TC sj[4]) {
    const TC x2 = kap * kap * r * r;
    const TC e = d_exp(-x2);
    const TC rinv2 = TC(1) / (r * r);
    const TC rinv6 = rinv2 * rinv2 * rinv2;
    const TC x4 = x2 * x2;
    const TC P6 = TC(1) + x2 + TC(0.5) * x4;
    const TC P8 = P6 + TC(1.0 / 6.0) * x4 * x2;
    const TC P10 = P8 + TC(1.0 / 24.0) * x4 * x4;
    const TC f6 = ((m - TC(1)) + e * P6) * rinv6;
    const TC f8 = ((m - TC(1)) + e * P8) * rinv6 * rinv2;
    const TC f10 = ((m - TC(1)) + e * P10) * rinv6 * rinv2 * rinv2;
    li[0] = f6 * cj[0];
    lj[0] = f6 * ci[0];
    li[1] = pmax >= 8 ? f8 * cj[1] : TC(0);
    lj[1] = pmax >= 8 ? f8 * ci[1] : TC(0);
    li[2] = pmax >= 10 ? f10 * cj[2] : TC(0);
    lj[2] = pmax >= 10 ? f10 * ci[2] : TC(0);
    for (int k = 0; k < 4; ++k) si[k] = sj[k] = TC(0);
    if (tt) {
        const TC BOHR = TC(1.889726878);
        const TC a = d_sqrt(ai * aj), b = d_sqrt(bi * bj), c = ci[0] * cj[0], q = qi * qj;
        const TC rb = r * BOHR;
        const TC br = b * rb;
        const TC eb = d_exp(-br);
        const TC br2 = br * br, br3 = br2 * br, br6 = br3 * br3;
        const TC poly = TC(1) + br + TC(0.5) * br2 + TC(1.0 / 6.0) * br3 + TC(1.0 / 24.0) * (br2 * br2) +
                        TC(1.0 / 120.0) * (br3 * br2) + TC(1.0 / 720.0) * br6;
        const TC dfa = m * TC(2625.5) * eb;                          // dE/da
        const TC dfq = -m * TC(2625.5) * eb * (TC(1) + br) / rb;     // dE/dq
        const TC dfc = m * eb * poly * rinv6;                        // dE/dc
        const TC dfb = m * rb * (-TC(2625.5) * a * eb + TC(2625.5) * q * eb * br / rb - c * eb * br6 / TC(720) * rinv6);
        si[0] = a > TC(0) ? dfa * aj / (TC(2) * a) : TC(0);
        sj[0] = a > TC(0) ? dfa * ai / (TC(2) * a) : TC(0);
        si[1] = b > TC(0) ? dfb * bj / (TC(2) * b) : TC(0);
        sj[1] = b > TC(0) ? dfb * bi / (TC(2) * b) : TC(0);
        si[2] = dfq * qj;
        sj[2] = dfq * qi;
        si[3] = dfc * cj[0];
        sj[3] = dfc * ci[0];
    }
}

template <typename TC>
__device__ __forceinline__ void disp_eval(TC r, TC m, const TC ci[3], const TC cj[3], TC kap, int pmax, bool tt,
                                          TC ai, TC aj, TC bi, TC bj, TC qi, TC qj, TC& e_lr, TC& de_lr, TC& e_sr,
                                          TC& de_sr) {
    const Dl<TC> R(r, TC(1));
    const Dl<TC> R2 = R * R;
    const Dl<TC> Rinv2(TC(1) / (r * r), TC(-2) / (r * r * r));
    const Dl<TC> Rinv6 = Rinv2 * Rinv2 * Rinv2;
    const Dl<TC> x2 = (kap * kap) * R2;
    const TC ev = d_exp(-x2.v);
    const Dl<TC> e(ev, -x2.d * ev);
    const Dl<TC> x4 = x2 * x2;
    const Dl<TC> P6 = TC(1) + (x2 + TC(0.5) * x4);
    Dl<TC> E = ((m - TC(1)) + (e * P6)) * Dl<TC>(ci[0] * cj[0], 0) * Rinv6;
    if (pmax >= 8) {
        const Dl<TC> P8 = P6 + TC(1.0 / 6.0) * (x4 * x2);
        const Dl<TC> Rinv8 = Rinv6 * Rinv2;
        E = E + ((m - TC(1)) + (e * P8)) * Dl<TC>(ci[1] * cj[1], 0) * Rinv8;
        if (pmax >= 10) {
            const Dl<TC> P10 = P8 + TC(1.0 / 24.0) * (x4 * x4);
            E = E + ((m - TC(1)) + (e * P10)) * Dl<TC>(ci[2] * cj[2], 0) * (Rinv8 * Rinv2);
        }
    }
    e_lr = E.v;
    de_lr = E.d;
    e_sr = de_sr = TC(0);
    if (tt) {
        const TC BOHR = TC(1.889726878);
        const TC a = d_sqrt(ai * aj), b = d_sqrt(bi * bj), c = ci[0] * cj[0], q = qi * qj;
        const Dl<TC> rb(r * BOHR, BOHR);
        const Dl<TC> br = b * rb;
        const TC ebv = d_exp(-br.v);
        const Dl<TC> eb(ebv, -br.d * ebv);
        const Dl<TC> br2 = br * br, br3 = br2 * br;
        const Dl<TC> br6 = br3 * br3;
        const Dl<TC> poly = TC(1) + (br + TC(0.5) * br2 + TC(1.0 / 6.0) * br3 + TC(1.0 / 24.0) * (br2 * br2) +
                                     TC(1.0 / 120.0) * (br3 * br2) + TC(1.0 / 720.0) * br6);
        const Dl<TC> rbinv(TC(1) / rb.v, -rb.d / (rb.v * rb.v));
        const Dl<TC> f = TC(2625.5) * a * eb - TC(2625.5) * q * (eb * (TC(1) + br) * rbinv) + c * (eb * poly * Rinv6);
        e_sr = m * f.v;
        de_sr = m * f.d;
    }
}

template <typename T, int ROWS, bool TT>
__global__ void __launch_bounds__(128) k_disp_pair(DispArgs<T> a) {
    const int64_t row = launch_row<ROWS>(a);
    int i = -1, j = -1, nb = 0;
    if (row < a.npairs) {
        i = a.pairs[3 * row];
        j = a.pairs[3 * row + 1];
        nb = a.pairs[3 * row + 2];
    }
    const bool valid = (row < a.npairs) && i >= 0 && i < j && j < a.n &&
                       (ROWS == 0 || (ROWS == 1) == (nb == 0));
    const int key = valid ? i : -1;
    T gl[3] = {T(0), T(0), T(0)}, gs[3] = {T(0), T(0), T(0)};
    double red[20];
#pragma unroll
    for (int k = 0; k < 20; ++k) red[k] = 0.0;
    if (valid) {
        double dr[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
        BoxT<double> bx;
#pragma unroll
        for (int k = 0; k < 9; ++k) { bx.h[k] = a.boxd.h[k]; bx.hinv[k] = a.boxd.hinv[k]; }
        double nimg[3];
        pbc_shift(bx, dr[0], dr[1], dr[2], nimg);
        int sidx = nb - 1;
        if (sidx < 0) sidx += 6;
        sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
        const double r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        double elr, delr, esr, desr;
        if (sizeof(T) < sizeof(double) && nb != 0) {
            const double ci[3] = {a.c[i], a.c[a.n + i], a.c[2 * a.n + i]};
            const double cj[3] = {a.c[j], a.c[a.n + j], a.c[2 * a.n + j]};
            disp_eval<double>(r, (double)a.ms[sidx], ci, cj, (double)a.kappa, a.pmax, TT,
                              TT ? (double)a.a[i] : 0.0, TT ? (double)a.a[j] : 0.0, TT ? (double)a.b[i] : 0.0,
                              TT ? (double)a.b[j] : 0.0, TT ? (double)a.q[i] : 0.0, TT ? (double)a.q[j] : 0.0,
                              elr, delr, esr, desr);
        } else {
            const T ci[3] = {a.c[i], a.c[a.n + i], a.c[2 * a.n + i]};
            const T cj[3] = {a.c[j], a.c[a.n + j], a.c[2 * a.n + j]};
            T e1, d1, e2, d2;
            disp_eval<T>((T)r, a.ms[sidx], ci, cj, a.kappa, a.pmax, TT, TT ? a.a[i] : T(0), TT ? a.a[j] : T(0),
                         TT ? a.b[i] : T(0), TT ? a.b[j] : T(0), TT ? a.q[i] : T(0), TT ? a.q[j] : T(0), e1, d1,
                         e2, d2);
            elr = e1; delr = d1; esr = e2; desr = d2;
        }
        red[0] = elr;
        red[1] = esr;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double u = dr[c] / r;
            gl[c] = (T)(delr * u);
            gs[c] = (T)(desr * u);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                red[2 + 3 * k + c] = -nimg[k] * delr * u;
                red[11 + 3 * k + c] = -nimg[k] * desr * u;
            }
        }
    }
    const bool head = seg_head(key);
    const int run = seg_run_id(key);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T s1 = seg_sum(gl[c], run);
        const T s2 = TT ? seg_sum(gs[c], run) : T(0);
        if (head && key >= 0) {
            atomicAdd(a.grad_lr + 3 * key + c, s1);
            if (TT) atomicAdd(a.grad_sr + 3 * key + c, s2);
        }
        if (valid) {
            atomicAdd(a.grad_lr + 3 * j + c, -gl[c]);
            if (TT) atomicAdd(a.grad_sr + 3 * j + c, -gs[c]);
        }
    }
    if (a.dlr) {  // parameter adjoints (FP64, i-side segmented sums, j-side atomics)
        double pi_[7], pj_[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) pi_[k] = pj_[k] = 0.0;
        if (valid) {
            double dv[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
            BoxT<double> bx;
#pragma unroll
            for (int k = 0; k < 9; ++k) { bx.h[k] = a.boxd.h[k]; bx.hinv[k] = a.boxd.hinv[k]; }
            double nim[3];
            pbc_shift(bx, dv[0], dv[1], dv[2], nim);
            const double r = sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            int sidx = nb - 1;
            if (sidx < 0) sidx += 6;
            sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
            const double ci[3] = {(double)a.c[i], (double)a.c[a.n + i], (double)a.c[2 * a.n + i]};
            const double cj[3] = {(double)a.c[j], (double)a.c[a.n + j], (double)a.c[2 * a.n + j]};
            double li[3], lj[3], si[4], sj[4];
            disp_pgrad<double>(r, (double)a.ms[sidx], ci, cj, (double)a.kappa, a.pmax, TT, TT ? (double)a.a[i] : 0.0,
                               TT ? (double)a.a[j] : 0.0, TT ? (double)a.b[i] : 0.0, TT ? (double)a.b[j] : 0.0,
                               TT ? (double)a.q[i] : 0.0, TT ? (double)a.q[j] : 0.0, li, lj, si, sj);
            for (int k = 0; k < 3; ++k) { pi_[k] = li[k]; pj_[k] = lj[k]; }
            for (int k = 0; k < 4; ++k) { pi_[3 + k] = si[k]; pj_[3 + k] = sj[k]; }
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) {
            if (!TT && k >= 3) break;
            const double sum = seg_sum(pi_[k], run);
            double* base = k < 3 ? a.dlr + (size_t)k * a.n : a.dsr + (size_t)(k - 3) * a.n;
            if (head && key >= 0) atomicAdd(base + key, sum);
            if (valid) atomicAdd(base + j, pj_[k]);
        }
    }
    block_reduce_add<20>(red, a.scal);
}

}  // namespace dmffb

namespace dmffb {
// Ewald self term of the dispersion parameter adjoints (disp_pme.py:264-289):
// dE/dc6_i -= kappa^6 / 6 c6_i, dE/dc8_i -= kappa^8 / 24 c8_i, dE/dc10_i -= kappa^10 / 120 c10_i
template <typename T>
__global__ void k_disp_self_dc(int n, int pmax, double kappa, const T* c, double* dc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double k2 = kappa * kappa, k6 = k2 * k2 * k2;
    dc[i] -= k6 / 6.0 * (double)c[i];
    if (pmax >= 8) dc[n + i] -= k6 * k2 / 24.0 * (double)c[n + i];
    if (pmax >= 10) dc[2 * n + i] -= k6 * k2 * k2 / 120.0 * (double)c[2 * n + i];
}
}  // namespace dmffb
