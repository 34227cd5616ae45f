// Classical force-field terms on sm_100a: Lennard-Jones + point-charge Coulomb pair kernel
// and the harmonic bond / harmonic angle / periodic torsion term kernels.
//
// Pair kernel, one thread per pair row (i, j, nbond), the ADMP kernel's layout (i-side warp
// segmented sums, j-side atomics, FP64 block reduction of energies and box gradient):
//   LJ   dmff/classical/inter.py:37-93:  E = 4 eps_ij m_lj (s^12 - s^6), s = sigma_ij / r, with
//        sigma_ij / eps_ij read from type-pair tables (Lorentz-Berthelot mixing and NBFix
//        overrides are applied on the host when the tables are built);
//   Coulomb, one of
//        PME real space (inter.py:269-335 -> energy_pme lmax 0, pme.py:633-710 cc term):
//            E = D q_i q_j (m_c - erf(kappa r)) / r;
//        reaction field (inter.py:210-260): E = D q_i q_j m_c (1/r + k_rf r^2 - c_rf);
//        no cutoff (inter.py:134-170): E = D q_i q_j m_c / r  (no periodic image);
//   D = 1389.35455846 kJ/mol A / e^2.  Units: Angstrom, e, kJ/mol.
// Rows with a topological scale (nbond != 0) run in FP64 in their own launch when the kernel
// precision is FP32: for excluded pairs m_c - erf is a large term that the reciprocal sum
// cancels.  Optional parameter adjoints: dE/dq per atom and dE/dsigma_ij, dE/deps_ij per type
// pair (FP64 atomics).
//
// Bonded terms (dmff/classical/intra.py:5-138), FP64, one thread per term, no periodic image
// (the reference evaluates them on raw coordinates):
//   bond    E = k/2 (|r_j - r_i| - r0)^2
//   angle   E = k/2 (theta - theta0)^2, theta = arccos(u.v), u = (p2-p1)/|.|, v = (p2-p3)/|.|
//   torsion E = k (1 + cos(n phi - psi)), phi = atan2(|b2| b1.(b2 x b3), (b2 x b3).(b1 x b2)),
//           b1 = p2-p1, b2 = p3-p2, b3 = p4-p3; the phi gradient is the chain rule of that
//           atan2 through b1, b2, b3.
// Each term optionally writes its parameter derivatives (dE/dk, dE/dr0 | dtheta0 | dpsi).
#pragma once
#include "common.cuh"
#include "admp_real.cuh"
#include "nblist.cuh"

namespace dmffb {

enum { COUL_NONE = 0, COUL_PME = 1, COUL_RF = 2, COUL_NOCUT = 3 };

template <typename T>
struct NbPairArgs {
    int n;
    int64_t npairs;
    const int32_t* pairs;
    const double* pos;     // [3n] FP64
    const double* q;       // [n] FP64 charges
    const T* qT;           // [n] charges in kernel precision
    const int32_t* type;   // [n] LJ type index, null when there is no LJ
    int ntypes;
    const T* sig_tt;       // [ntypes^2]
    const T* eps_tt;       // [ntypes^2]
    T mc[6], ml[6];
    T kappa, krf, crf;
    int coul;
    int pbc;               // minimum image on the pair vector
    Box boxd;
    T* grad;               // [3n] dE/dpos
    double* dq;            // [n] dE/dq or null
    double* dsig;          // [ntypes^2] dE/dsigma_ij or null
    double* deps;          // [ntypes^2] dE/deps_ij or null
    double* scal;          // [0] E_coul real space, [1] E_lj, [2..10] box gradient
    const int32_t* rowmap = nullptr;  // ROWS == 2 launches: indices of the rows with nbond != 0
    int64_t nrowmap = 0;
    double cut = 0.0;  // > 0: only rows whose minimum-image distance is < cut (the list build's test)
};

// energies and d/dr of one pair; phi = dE_coul / d(q_i q_j)
template <typename TC>
__device__ __forceinline__ void nb_eval(TC r, TC qq, TC mc, TC ml, TC sig, TC eps, bool lj, int coul, TC kappa,
                                        TC krf, TC crf, TC& ec, TC& dec, TC& phi, TC& el, TC& del, TC& dsig,
                                        TC& deps) {
    const TC D = TC(DMFFB_DIELECTRIC);
    const TC rinv = TC(1) / r;
    TC f = TC(0), fp = TC(0);
    if (coul == COUL_PME) {
        const TC kr = kappa * r;
        f = (mc - d_erf(kr)) * rinv;
        fp = -TC(1.1283791670955126) * kappa * d_exp(-kr * kr) * rinv - f * rinv;
    } else if (coul == COUL_RF) {
        f = mc * (rinv + krf * r * r - crf);
        fp = mc * (-rinv * rinv + TC(2) * krf * r);
    } else if (coul == COUL_NOCUT) {
        f = mc * rinv;
        fp = -mc * rinv * rinv;
    }
    phi = D * f;
    ec = D * qq * f;
    dec = D * qq * fp;
    el = del = dsig = deps = TC(0);
    if (lj) {
        const TC s2 = sig * sig * rinv * rinv;
        const TC s6 = s2 * s2 * s2;
        const TC s12 = s6 * s6;
        const TC w = TC(4) * ml;
        el = w * eps * (s12 - s6);
        del = w * eps * (TC(6) * s6 - TC(12) * s12) * rinv;
        deps = w * (s12 - s6);
        // d/dsigma without dividing by sigma (sigma may be 0): s^6/sigma = sigma^5 / r^6
        const TC r2i = rinv * rinv;
        const TC r6i = r2i * r2i * r2i;
        const TC sg2 = sig * sig;
        const TC sg5 = sg2 * sg2 * sig;
        const TC s6_over_sig = sg5 * r6i;
        dsig = w * eps * (TC(12) * s6 * s6_over_sig - TC(6) * s6_over_sig);
    }
}

template <typename T, int ROWS>
__global__ void __launch_bounds__(128) k_nb_pair(NbPairArgs<T> a) {
    const int64_t row = launch_row<ROWS>(a);
    int i = -1, j = -1, nb = 0;
    if (row < a.npairs) {
        i = a.pairs[3 * row];
        j = a.pairs[3 * row + 1];
        nb = a.pairs[3 * row + 2];
    }
    bool valid = (row < a.npairs) && i >= 0 && i < j && j < a.n && (ROWS == 0 || (ROWS == 1) == (nb == 0));
    if (valid && a.cut > 0.0) valid = within_rc(a.boxd, a.pos + 3 * i, a.pos + 3 * j, a.cut);
    const int key = valid ? i : -1;
    T g[3] = {T(0), T(0), T(0)};
    double red[11];
#pragma unroll
    for (int k = 0; k < 11; ++k) red[k] = 0.0;
    double phi_ij = 0.0;
    if (valid) {
        double dr[3] = {a.pos[3 * i] - a.pos[3 * j], a.pos[3 * i + 1] - a.pos[3 * j + 1], a.pos[3 * i + 2] - a.pos[3 * j + 2]};
        double nimg[3] = {0.0, 0.0, 0.0};
        if (a.pbc) {
            BoxT<double> bx;
#pragma unroll
            for (int k = 0; k < 9; ++k) { bx.h[k] = a.boxd.h[k]; bx.hinv[k] = a.boxd.hinv[k]; }
            pbc_shift(bx, dr[0], dr[1], dr[2], nimg);
        }
        int sidx = nb - 1;
        if (sidx < 0) sidx += 6;
        sidx = sidx < 0 ? 0 : (sidx > 5 ? 5 : sidx);
        const double r = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        const bool lj = a.type != nullptr;
        int tp = 0;
        if (lj) tp = a.type[i] * a.ntypes + a.type[j];
        double ec, dec, phi, el, del, dsg, dep;
        if (sizeof(T) < sizeof(double) && nb != 0) {
            double e1, d1, p1, e2, d2, s1, s2;
            nb_eval<double>(r, a.q[i] * a.q[j], (double)a.mc[sidx], (double)a.ml[sidx],
                            lj ? (double)a.sig_tt[tp] : 0.0, lj ? (double)a.eps_tt[tp] : 0.0, lj, a.coul,
                            (double)a.kappa, (double)a.krf, (double)a.crf, e1, d1, p1, e2, d2, s1, s2);
            ec = e1; dec = d1; phi = p1; el = e2; del = d2; dsg = s1; dep = s2;
        } else {
            T e1, d1, p1, e2, d2, s1, s2;
            nb_eval<T>((T)r, a.qT[i] * a.qT[j], a.mc[sidx], a.ml[sidx], lj ? a.sig_tt[tp] : T(0),
                       lj ? a.eps_tt[tp] : T(0), lj, a.coul, a.kappa, a.krf, a.crf, e1, d1, p1, e2, d2, s1, s2);
            ec = e1; dec = d1; phi = p1; el = e2; del = d2; dsg = s1; dep = s2;
        }
        red[0] = ec;
        red[1] = el;
        const double de = dec + del;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double u = dr[c] / r;
            g[c] = (T)(de * u);
#pragma unroll
            for (int k = 0; k < 3; ++k) red[2 + 3 * k + c] = -nimg[k] * de * u;
        }
        phi_ij = phi;
        if (a.dq) atomicAdd(a.dq + j, phi * a.q[i]);
        if (lj && a.dsig) {
            atomicAdd(a.dsig + tp, dsg);
            atomicAdd(a.deps + tp, dep);
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
    if (a.dq) {
        const double dqi = seg_sum(valid ? phi_ij * a.q[j] : 0.0, run);
        if (head && key >= 0) atomicAdd(a.dq + key, dqi);
    }
    block_reduce_add<11>(red, a.scal);
}

// ------------------------------------------------------------------ bonded terms (FP64)
struct BondedArgs {
    int nterm;
    const int32_t* idx;   // [nterm * arity]
    const double* prm;    // bond (k, r0) | angle (k, theta0) | torsion (k, psi, periodicity)
    const double* pos;    // [3n]
    double* grad;         // [3n] dE/dpos
    double* dprm;         // [nterm * 2] (dE/dk, dE/d(r0 | theta0 | psi)) or null
    double* scal;         // energy slot
};

__device__ __forceinline__ void ld3(const double* p, int i, double v[3]) {
    v[0] = p[3 * i];
    v[1] = p[3 * i + 1];
    v[2] = p[3 * i + 2];
}
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
__device__ __forceinline__ void add_grad(double* g, int i, const double v[3], double s) {
    atomicAdd(g + 3 * i, s * v[0]);
    atomicAdd(g + 3 * i + 1, s * v[1]);
    atomicAdd(g + 3 * i + 2, s * v[2]);
}

__global__ void __launch_bounds__(128) k_bonds(BondedArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double red[1] = {0.0};
    if (t < a.nterm) {
        const int i = a.idx[2 * t], j = a.idx[2 * t + 1];
        const double k = a.prm[2 * t], r0 = a.prm[2 * t + 1];
        double pi[3], pj[3], d[3];
        ld3(a.pos, i, pi);
        ld3(a.pos, j, pj);
        for (int c = 0; c < 3; ++c) d[c] = pi[c] - pj[c];
        const double r = sqrt(dot3(d, d));
        const double x = r - r0;
        red[0] = 0.5 * k * x * x;
        const double s = k * x / r;  // dE/dr / r
        add_grad(a.grad, i, d, s);
        add_grad(a.grad, j, d, -s);
        if (a.dprm) {
            a.dprm[2 * t] = 0.5 * x * x;
            a.dprm[2 * t + 1] = -k * x;
        }
    }
    block_reduce_add<1>(red, a.scal);
}

__global__ void __launch_bounds__(128) k_angles(BondedArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double red[1] = {0.0};
    if (t < a.nterm) {
        const int i1 = a.idx[3 * t], i2 = a.idx[3 * t + 1], i3 = a.idx[3 * t + 2];
        const double k = a.prm[2 * t], th0 = a.prm[2 * t + 1];
        double p1[3], p2[3], p3[3], u[3], w[3];
        ld3(a.pos, i1, p1);
        ld3(a.pos, i2, p2);
        ld3(a.pos, i3, p3);
        for (int c = 0; c < 3; ++c) {
            u[c] = p2[c] - p1[c];
            w[c] = p2[c] - p3[c];
        }
        const double lu = sqrt(dot3(u, u)), lw = sqrt(dot3(w, w));
        double e1[3], e2[3];
        for (int c = 0; c < 3; ++c) {
            e1[c] = u[c] / lu;
            e2[c] = w[c] / lw;
        }
        const double cs = dot3(e1, e2);
        const double th = acos(fmin(1.0, fmax(-1.0, cs)));
        const double x = th - th0;
        red[0] = 0.5 * k * x * x;
        double sn = sqrt(fmax(1.0 - cs * cs, 1e-30));
        const double dEdc = -k * x / sn;  // dE/dcos(theta)
        double ga[3], gc[3];
        for (int c = 0; c < 3; ++c) {
            // d cos / d u = (e2 - cs e1)/|u|, u = p2 - p1;  d cos / d w = (e1 - cs e2)/|w|, w = p2 - p3
            ga[c] = -dEdc * (e2[c] - cs * e1[c]) / lu;
            gc[c] = -dEdc * (e1[c] - cs * e2[c]) / lw;
        }
        add_grad(a.grad, i1, ga, 1.0);
        add_grad(a.grad, i3, gc, 1.0);
        double gb[3] = {-(ga[0] + gc[0]), -(ga[1] + gc[1]), -(ga[2] + gc[2])};
        add_grad(a.grad, i2, gb, 1.0);
        if (a.dprm) {
            a.dprm[2 * t] = 0.5 * x * x;
            a.dprm[2 * t + 1] = -k * x;
        }
    }
    block_reduce_add<1>(red, a.scal);
}

__global__ void __launch_bounds__(128) k_torsions(BondedArgs a) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    double red[1] = {0.0};
    if (t < a.nterm) {
        const int i1 = a.idx[4 * t], i2 = a.idx[4 * t + 1], i3 = a.idx[4 * t + 2], i4 = a.idx[4 * t + 3];
        const double k = a.prm[3 * t], psi = a.prm[3 * t + 1], per = a.prm[3 * t + 2];
        double p1[3], p2[3], p3[3], p4[3], b1[3], b2[3], b3[3];
        ld3(a.pos, i1, p1);
        ld3(a.pos, i2, p2);
        ld3(a.pos, i3, p3);
        ld3(a.pos, i4, p4);
        for (int c = 0; c < 3; ++c) {
            b1[c] = p2[c] - p1[c];
            b2[c] = p3[c] - p2[c];
            b3[c] = p4[c] - p3[c];
        }
        double m[3], nn[3];
        cross3(b1, b2, m);
        cross3(b2, b3, nn);
        const double gl = sqrt(dot3(b2, b2));
        const double y = gl * dot3(b1, nn), x = dot3(nn, m);
        const double phi = atan2(y, x);
        const double arg = per * phi - psi;
        red[0] = k * (1.0 + cos(arg));
        const double dEdphi = -k * per * sin(arg);
        // d phi = (x dy - y dx) / (x^2 + y^2) with y, x differentiated through b1, b2, b3
        const double den = x * x + y * y;
        double dy1[3], dy2[3], dy3[3], dx1[3], dx2[3], dx3[3], t1[3], t2[3];
        const double b1n = dot3(b1, nn);
        for (int c = 0; c < 3; ++c) {
            dy1[c] = gl * nn[c];
            dy3[c] = gl * m[c];
        }
        cross3(b3, b1, t1);
        for (int c = 0; c < 3; ++c) dy2[c] = b2[c] / gl * b1n + gl * t1[c];
        cross3(b2, nn, dx1);
        cross3(m, b2, dx3);
        cross3(b3, m, t1);
        cross3(nn, b1, t2);
        for (int c = 0; c < 3; ++c) dx2[c] = t1[c] + t2[c];
        double d1[3], d2[3], d3[3];
        const double sc = dEdphi / den;
        for (int c = 0; c < 3; ++c) {
            d1[c] = sc * (x * dy1[c] - y * dx1[c]);
            d2[c] = sc * (x * dy2[c] - y * dx2[c]);
            d3[c] = sc * (x * dy3[c] - y * dx3[c]);
        }
        // b1 = p2 - p1, b2 = p3 - p2, b3 = p4 - p3
        double g2[3], g3[3];
        for (int c = 0; c < 3; ++c) {
            g2[c] = d1[c] - d2[c];
            g3[c] = d2[c] - d3[c];
        }
        add_grad(a.grad, i1, d1, -1.0);
        add_grad(a.grad, i2, g2, 1.0);
        add_grad(a.grad, i3, g3, 1.0);
        add_grad(a.grad, i4, d3, 1.0);
        if (a.dprm) {
            a.dprm[2 * t] = 1.0 + cos(arg);
            a.dprm[2 * t + 1] = k * sin(arg);
        }
    }
    block_reduce_add<1>(red, a.scal);
}

}  // namespace dmffb
