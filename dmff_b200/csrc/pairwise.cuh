// Short-range pairwise terms with per-atom parameters and closed-form kernels on sm_100a: the
// built-in kernels of dmff/admp/pairwise.py, used by the ADMP short-range generators
// (dmff/generators/admp.py:22-863).  r in Angstrom, m = mScales[nbond - 1].
//   SR_TT_QQ     (pairwise.py:121-128, QqTtDampingForce):
//                E = -D e^-x (1 + x) q / r,  x = b r,  b = sqrt(b_i b_j),  q = q_i q_j
//   SR_SLATER_DISP (pairwise.py:131-156, SlaterDampingForce):
//                E = sum_{n=6,8,10} e^-x s_n(x) c_n / r^n,  c_n = c_n,i c_n,j,
//                x = y - (2 y^2 + 3 y) / (y^2 + 3 y + 3),  y = b r,
//                s_n the exponential series to x^n / n!
//   SR_SLATER    (pairwise.py:159-171, SlaterExForce and the SlaterSr*/SlaterDhf terms with a sign):
//                E = a (y^2 / 3 + y + 1) e^-y,  a = a_i a_j,  y = b r
//   SR_TT_QQ_C6  (pairwise.py:100-118, generate_pairwise_interaction(TT_damping_qq_c6_kernel)):
//                E = 2625.5 a e^-x - 2625.5 e^-x (1 + x) q / r_b + e^-x P6(x) c / r^6,
//                r_b = 1.889726878 r,  x = b r_b,  a = sqrt(a_i a_j), q = q_i q_j, c = c_i c_j
//   SR_QEQ_GAUSS3 (qeq.py:98-112, the Gaussian-charge short range of ADMPQeqForce, DampMod 3):
//                E = -D erfc(r / s) q / r,  s = sqrt(eta_i^2 + eta_j^2),  q = q_i q_j (0 when s <= 1e-4)
//   SR_QEQ_GAUSS2 (qeq.py:85-95, DampMod 2): the same with s = sqrt(2 (eta_i^2 + eta_j^2))
// each times m.  One thread per pair row (the layout of the classical pair kernel: minimum image
// in FP64, i-side warp segmented sums, j-side atomics, FP64 block reduction of the energy and box
// gradient); dE/dr and every per-atom parameter partial come from the closed forms, using
// d/dx [e^-x S_k(x)] = -e^-x x^k / k! for a truncated exponential series S_k.
#pragma once
#include "common.cuh"
#include "admp_real.cuh"

namespace dmffb {

enum { SR_TT_QQ = 0, SR_SLATER_DISP = 1, SR_SLATER = 2, SR_TT_QQ_C6 = 3, SR_QEQ_GAUSS3 = 4, SR_QEQ_GAUSS2 = 5 };

// parameters per atom of each kind
__host__ __device__ constexpr int sr_nparam(int kind) {
    return kind == SR_SLATER_DISP || kind == SR_TT_QQ_C6 ? 4 : 2;
}

template <typename T>
struct SrArgs {
    int n;
    int64_t npairs;
    const int32_t* pairs;
    const double* pos;     // [3n]
    const T* p;            // [nparam][n] per-atom parameters, channel-major
    T ms[6];
    T sign;                // overall factor (-1 for the SlaterSr*/SlaterDhf terms)
    Box boxd;
    T* grad;               // [3n] dE/dpos
    double* dp;            // [nparam][n] += dE/dparameter (null: no adjoints)
    double* scal;          // [0] energy, [1..9] box gradient
};

// exponential series sum_{k=0}^{K} x^k / k! and its last term x^K / K!
template <typename TC>
__device__ __forceinline__ void exp_series(TC x, int K, TC& s, TC& last) {
    TC t = TC(1);
    s = TC(1);
    for (int k = 1; k <= K; ++k) {
        t = t * x / TC(k);
        s += t;
    }
    last = t;
}

// E(r) and dE/dr of one pair, with dE/d(pair parameter) in gp[0..3]: the pair parameters are
// (b, q) for TT_QQ, (b, c6, c8, c10) for SLATER_DISP, (a, b) for SLATER, (a, b, q, c) for TT_QQ_C6,
// (q, s) for the QEQ_GAUSS kinds, where a, b, s (and the Slater a) are the combined values above
template <int KIND, typename TC>
__device__ __forceinline__ void sr_eval(TC r, const TC pp[4], TC& e, TC& de, TC gp[4]) {
    const TC D = TC(DMFFB_DIELECTRIC);
    if (KIND == SR_TT_QQ) {
        const TC b = pp[0], q = pp[1];
        const TC x = b * r, ex = d_exp(-x);
        const TC f = ex * (TC(1) + x);            // f'(x) = -x e^-x
        const TC rinv = TC(1) / r;
        e = -D * q * f * rinv;
        de = -D * q * (-b * x * ex * rinv - f * rinv * rinv);
        gp[0] = -D * q * (-x * ex) * rinv * r;    // dE/db = dE/dx * r
        gp[1] = -D * f * rinv;
        gp[2] = gp[3] = TC(0);
    } else if (KIND == SR_SLATER_DISP) {
        const TC b = pp[0];
        const TC y = b * r, y2 = y * y;
        const TC den = y2 + TC(3) * y + TC(3);
        const TC num = TC(2) * y2 + TC(3) * y;
        const TC x = y - num / den;
        const TC dxdy = TC(1) - ((TC(4) * y + TC(3)) * den - num * (TC(2) * y + TC(3))) / (den * den);
        const TC ex = d_exp(-x);
        const TC rinv = TC(1) / r;
        const TC r2i = rinv * rinv;
        const TC r6i = r2i * r2i * r2i;
        TC s, last;
        e = de = TC(0);
        TC dEdx = TC(0);
        const TC rp[3] = {r6i, r6i * r2i, r6i * r2i * r2i};
        for (int q = 0; q < 3; ++q) {
            const int nn = 6 + 2 * q;
            exp_series(x, nn, s, last);
            const TC fq = ex * s;               // d/dx = -e^-x x^n / n!
            const TC c = pp[1 + q];
            e += fq * c * rp[q];
            dEdx += -ex * last * c * rp[q];
            de += -TC(nn) * fq * c * rp[q] * rinv;
            gp[1 + q] = fq * rp[q];
        }
        de += dEdx * dxdy * b;
        gp[0] = dEdx * dxdy * r;
    } else if (KIND == SR_SLATER) {
        const TC a = pp[0], b = pp[1];
        const TC y = b * r, ey = d_exp(-y);
        const TC P = y * y / TC(3) + y + TC(1);
        const TC dEdy = -a * ey * y * (TC(1) + y) / TC(3);
        e = a * P * ey;
        de = dEdy * b;
        gp[0] = P * ey;
        gp[1] = dEdy * r;
        gp[2] = gp[3] = TC(0);
    } else if (KIND == SR_QEQ_GAUSS3 || KIND == SR_QEQ_GAUSS2) {
        const TC q = pp[0], sw = pp[1];
        gp[2] = gp[3] = TC(0);
        if (!(sw > TC(1e-4))) {
            e = de = gp[0] = gp[1] = TC(0);
        } else {
            const TC rinv = TC(1) / r;
            const TC x = r / sw;
            const TC ec = d_erfc(x);
            const TC g = TC(DMFFB_TWO_OVER_SQRTPI) * d_exp(-x * x);  // -d erfc / dx
            e = -D * q * ec * rinv;
            de = -D * q * (-g / sw * rinv - ec * rinv * rinv);
            gp[0] = -D * ec * rinv;
            gp[1] = -D * q * g / (sw * sw);  // d erfc(r / s) / ds = g r / s^2
        }
    } else {  // SR_TT_QQ_C6
        const TC a = pp[0], b = pp[1], q = pp[2], c = pp[3];
        const TC kb = TC(1.889726878);
        const TC rb = kb * r;
        const TC x = b * rb, ex = d_exp(-x);
        const TC rbinv = TC(1) / rb;
        const TC rinv = TC(1) / r;
        const TC r2i = rinv * rinv;
        const TC r6i = r2i * r2i * r2i;
        TC s6, last6;
        exp_series(x, 6, s6, last6);
        const TC t1 = TC(2625.5) * a * ex;
        const TC t2 = -TC(2625.5) * ex * (TC(1) + x) * q * rbinv;
        const TC t3 = ex * s6 * c * r6i;
        e = t1 + t2 + t3;
        // dE/dx at fixed r_b, then d/dr through x = b k r and the explicit 1/r_b, 1/r^6
        const TC dEdx = -t1 + TC(2625.5) * x * ex * q * rbinv - ex * last6 * c * r6i;
        de = dEdx * b * kb - t2 * rinv - TC(6) * t3 * rinv;
        gp[0] = TC(2625.5) * ex;
        gp[1] = dEdx * rb;
        gp[2] = -TC(2625.5) * ex * (TC(1) + x) * rbinv;
        gp[3] = ex * s6 * r6i;
    }
}

template <typename T, int KIND>
__global__ void __launch_bounds__(128) k_sr_pair(SrArgs<T> a) {
    constexpr int NP = sr_nparam(KIND);
    const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int i = -1, j = -1, nb = 0;
    if (row < a.npairs) {
        i = a.pairs[3 * row];
        j = a.pairs[3 * row + 1];
        nb = a.pairs[3 * row + 2];
    }
    const bool valid = (row < a.npairs) && i >= 0 && i < j && j < a.n;
    const int key = valid ? i : -1;
    T g[3] = {T(0), T(0), T(0)};
    double red[10];
#pragma unroll
    for (int k = 0; k < 10; ++k) red[k] = 0.0;
    T pi_grad[4] = {T(0), T(0), T(0), T(0)};
    if (valid) {
        double dr[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
        double nimg[3];
        BoxT<double> bx;
#pragma unroll
        for (int k = 0; k < 9; ++k) { bx.h[k] = a.boxd.h[k]; bx.hinv[k] = a.boxd.hinv[k]; }
        pbc_shift(bx, dr[0], dr[1], dr[2], nimg);
        const double r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        int sidx = nb - 1;
        if (sidx < 0) sidx += 6;
        sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
        const T m = a.ms[sidx] * a.sign;
        T vi[4], vj[4], pp[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            vi[k] = k < NP ? a.p[(size_t)k * a.n + i] : T(0);
            vj[k] = k < NP ? a.p[(size_t)k * a.n + j] : T(0);
        }
        // combination rules of the pair parameters
        if (KIND == SR_TT_QQ) {
            pp[0] = sqrt(vi[0] * vj[0]);
            pp[1] = vi[1] * vj[1];
        } else if (KIND == SR_SLATER_DISP) {
            pp[0] = sqrt(vi[0] * vj[0]);
            pp[1] = vi[1] * vj[1];
            pp[2] = vi[2] * vj[2];
            pp[3] = vi[3] * vj[3];
        } else if (KIND == SR_SLATER) {
            pp[0] = vi[0] * vj[0];
            pp[1] = sqrt(vi[1] * vj[1]);
        } else if (KIND == SR_QEQ_GAUSS3 || KIND == SR_QEQ_GAUSS2) {
            pp[0] = vi[0] * vj[0];
            const T c2 = KIND == SR_QEQ_GAUSS2 ? T(2) : T(1);
            pp[1] = sqrt(c2 * (vi[1] * vi[1] + vj[1] * vj[1]));
        } else {
            pp[0] = sqrt(vi[0] * vj[0]);
            pp[1] = sqrt(vi[1] * vj[1]);
            pp[2] = vi[2] * vj[2];
            pp[3] = vi[3] * vj[3];
        }
        T e, de, gp[4];
        sr_eval<KIND, T>((T)r, pp, e, de, gp);
        e *= m;
        de *= m;
        red[0] = (double)e;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double u = dr[c] / r;
            g[c] = (T)((double)de * u);
#pragma unroll
            for (int k = 0; k < 3; ++k) red[1 + 3 * k + c] = -nimg[k] * (double)de * u;
        }
        if (a.dp) {
            // chain rule of the combination rules to the per-atom parameters of i and j
            T gi[4] = {T(0), T(0), T(0), T(0)}, gj[4] = {T(0), T(0), T(0), T(0)};
            auto sq = [](T p, T other, T comb) { return comb > T(0) ? T(0.5) * other / comb : T(0); };
            if (KIND == SR_TT_QQ) {
                gi[0] = gp[0] * sq(vi[0], vj[0], pp[0]); gj[0] = gp[0] * sq(vj[0], vi[0], pp[0]);
                gi[1] = gp[1] * vj[1]; gj[1] = gp[1] * vi[1];
            } else if (KIND == SR_SLATER_DISP) {
                gi[0] = gp[0] * sq(vi[0], vj[0], pp[0]); gj[0] = gp[0] * sq(vj[0], vi[0], pp[0]);
#pragma unroll
                for (int k = 1; k < 4; ++k) { gi[k] = gp[k] * vj[k]; gj[k] = gp[k] * vi[k]; }
            } else if (KIND == SR_SLATER) {
                gi[0] = gp[0] * vj[0]; gj[0] = gp[0] * vi[0];
                gi[1] = gp[1] * sq(vi[1], vj[1], pp[1]); gj[1] = gp[1] * sq(vj[1], vi[1], pp[1]);
            } else if (KIND == SR_QEQ_GAUSS3 || KIND == SR_QEQ_GAUSS2) {
                // s^2 = c2 (eta_i^2 + eta_j^2): ds / deta_i = c2 eta_i / s
                const T c2 = KIND == SR_QEQ_GAUSS2 ? T(2) : T(1);
                gi[0] = gp[0] * vj[0]; gj[0] = gp[0] * vi[0];
                const T sinv = pp[1] > T(0) ? T(1) / pp[1] : T(0);
                gi[1] = gp[1] * c2 * vi[1] * sinv; gj[1] = gp[1] * c2 * vj[1] * sinv;
            } else {
                gi[0] = gp[0] * sq(vi[0], vj[0], pp[0]); gj[0] = gp[0] * sq(vj[0], vi[0], pp[0]);
                gi[1] = gp[1] * sq(vi[1], vj[1], pp[1]); gj[1] = gp[1] * sq(vj[1], vi[1], pp[1]);
                gi[2] = gp[2] * vj[2]; gj[2] = gp[2] * vi[2];
                gi[3] = gp[3] * vj[3]; gj[3] = gp[3] * vi[3];
            }
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                pi_grad[k] = gi[k] * m;
                atomicAdd(a.dp + (size_t)k * a.n + j, (double)(gj[k] * m));
            }
        }
    }
    const bool head = seg_head(key);
    const int run = seg_run_id(key);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T s1 = seg_sum(g[c], run);
        if (head && key >= 0) atomicAdd(a.grad + 3 * key + c, s1);
        if (valid) atomicAdd(a.grad + 3 * j + c, -g[c]);
    }
    if (a.dp) {
#pragma unroll
        for (int k = 0; k < NP; ++k) {
            const double s1 = seg_sum((double)pi_grad[k], run);
            if (head && key >= 0) atomicAdd(a.dp + (size_t)k * a.n + key, s1);
        }
    }
    block_reduce_add<10>(red, a.scal);
}

template <typename T>
__global__ void k_sr_finalize(int n, const T* grad, double* forces) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < 3 * n) forces[k] = -(double)grad[k];
}

}  // namespace dmffb
