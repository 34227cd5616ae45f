// Lennard-Jones + point-charge Coulomb over the cell grid, without a pair list.
//
// The engine's own neighbour list (dmff/common/nblist.py:27-55 semantics: every i < j whose
// minimum-image distance is < rc, nbond from the covalent map) is, for the classical terms,
// written once per step and read once by the pair kernel: at 100 000 atoms and rc 10 A that is
// 61 M rows, 0.74 GB out and back, plus j-side force atomics.  This pass evaluates the same pair
// set straight from the cell binning of the step's positions:
//   * one warp per atom i walks the forward half of the 5^3 stencil of half-width cells (the 62
//     offsets after (0, 0, 0) in lexicographic order, and in its own cell the atoms after it in
//     cell order), so every unordered pair is met once, as one concatenated candidate list, 32
//     candidates per batch, reading a cell-ordered float4 copy of the positions (contiguous runs
//     per cell, the atom index in the w slot); atoms are taken in cell order, so the warps of a
//     block share their candidates through L1 (with at least 5 cells per axis the 5 offsets of an
//     axis are distinct cells, and a box of at least 2.5 rc has one image of a pair within rc);
//   * stencil cells with no point within rc of the atom are skipped (per atom, from its position
//     in its cell);
//   * FP32 prefilter on float positions, the exact FP64 test of the list build (within_rc on the
//     lower/higher orientation) inside a 2e-3 A band around rc, so the kept set is the list's
//     set bit for bit;
//   * pairs with a topological scale (nbond != 0, a covalent partner whose index lies in the
//     atom's [cov_lo, cov_hi] range) are skipped here: an FP64 pass over the covalent rows
//     within rc evaluates them (k_nb_pair with a cut-off test);
//   * every other kept pair is queued in shared memory and evaluated 32 at a time (every lane
//     busy): nb_eval in kernel precision on the FP64 minimum-image vector and distance of
//     k_nb_pair; the force on i accumulates in lane registers (one warp sum and one atomic per
//     atom), the force on j goes out as an atomic;
//   * the count of kept pairs (scaled ones included) is the list's row count.
// Energies and the box gradient accumulate per lane (about 20 pairs each) and meet in an FP64 block
// reduction.
#pragma once
#include "classical.cuh"
#include "nblist.cuh"

namespace dmffb {

template <typename T>
struct NbCellArgs {
    int n;
    const double* pos;        // [3n] FP64
    const float4* posc;       // [n] FP32 x, y, z and the atom index (as int bits), in cell order
    Box boxd;
    double rc;
    int nc[3];                // half-width cells per axis (>= 5)
    double width[3];          // perpendicular widths of the box (the distance between the faces
                              // of constant fractional coordinate k)
    const int32_t* cell_start;
    NbArgs cov;               // covalent-map lookup (cov_ptr / cov_j / cov_nb over i < j)
    const int32_t* cov_lo;    // [n] smallest / largest covalent partner index (lo > hi: none)
    const int32_t* cov_hi;
    const T* qT;              // [n] charges in kernel precision
    const int32_t* type;      // [n] LJ type or null
    int ntypes;
    const T* sig_tt;
    const T* eps_tt;
    T mc, ml;                 // scales of nbond 0 (the trailing 1.0 entries)
    T kappa, krf, crf;
    int coul;
    T* grad;                  // [3n] dE/dpos, written once per atom
    double* scal;             // [0] E_coul, [1] E_lj, [2..10] box gradient, [11] pairs i < j within rc
};

// One kept pair (i, j), met once: energy, box gradient, the force on i (registers) and on j (atomics).
template <typename T>
__device__ __forceinline__ void nb_cell_pair(const NbCellArgs<T>& a, int i, int j, const double* pi,
                                             const BoxT<double>& bxd, bool lj, int ti, T qi, T& g0, T& g1, T& g2,
                                             T (&acc)[11]) {
    // the pair geometry of k_nb_pair: FP64 minimum image, then kernel precision
    T e[3], r;
    T nn[3];
    {
        double dr[3] = {a.pos[3 * j] - pi[0], a.pos[3 * j + 1] - pi[1], a.pos[3 * j + 2] - pi[2]};
        double nd[3];
        pbc_shift(bxd, dr[0], dr[1], dr[2], nd);
#pragma unroll
        for (int c = 0; c < 3; ++c) { e[c] = (T)dr[c]; nn[c] = (T)nd[c]; }
        r = (T)sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    }
    int tp = 0;
    if (lj) tp = ti * a.ntypes + a.type[j];
    T ec, dec, phi, el, del, ds, dp;
    nb_eval<T>(r, qi * a.qT[j], a.mc, a.ml, lj ? a.sig_tt[tp] : T(0), lj ? a.eps_tt[tp] : T(0), lj, a.coul, a.kappa,
               a.krf, a.crf, ec, dec, phi, el, del, ds, dp);
    // e = r_j - r_i (minimum image); dE/dr_i = -(dE/dr / r) e; image counts of r_i - r_j are -nn
    const T s = (dec + del) / r;
    g0 -= s * e[0];
    g1 -= s * e[1];
    g2 -= s * e[2];
    atomicAdd(a.grad + 3 * j, s * e[0]);
    atomicAdd(a.grad + 3 * j + 1, s * e[1]);
    atomicAdd(a.grad + 3 * j + 2, s * e[2]);
    acc[0] += ec;
    acc[1] += el;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[2 + 3 * k + c] -= nn[k] * s * e[c];
}

template <typename T>
__global__ void __launch_bounds__(32 * kNbWarps, sizeof(T) == 4 ? 4 : 0) k_nb_cells(NbCellArgs<T> a) {
    constexpr int S = 2, W = 2 * S + 1, NQ = (W * W * W + 1) / 2;  // offsets q0 = 62 .. 124 of the 5^3 stencil
    __shared__ int s_beg[kNbWarps][NQ];
    __shared__ int s_off[kNbWarps][NQ + 1];
    __shared__ int s_q[kNbWarps][64];  // kept candidates waiting for a full 32-lane batch
    const int wl = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    // warps take the atoms in cell order: the warps of a block share one stencil, so their
    // candidate reads (contiguous runs of the cell-ordered copy) hit L1 after the first
    const int ks = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const bool live = ks < a.n;  // warps past the end still take part in the block reduction
    double red[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) red[k] = 0.0;
    if (live) {
        const float4 p4 = a.posc[ks];
        const int i = __float_as_int(p4.w);
        const double* pi = a.pos + 3 * i;
        const float pix = p4.x, piy = p4.y, piz = p4.z;
        float hf[9], hif[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) { hf[k] = (float)a.boxd.h[k]; hif[k] = (float)a.boxd.hinv[k]; }
        BoxT<double> bxd;
#pragma unroll
        for (int k = 0; k < 9; ++k) { bxd.h[k] = a.boxd.h[k]; bxd.hinv[k] = a.boxd.hinv[k]; }
        const float rlo = (float)(a.rc - 2e-3), rhi = (float)(a.rc + 2e-3);
        const float rlo2 = rlo * rlo, rhi2 = rhi * rhi;
        int c3[3];
        cell_of(a.boxd, a.nc, pi, c3);
        // the atom's fractional coordinates (as cell_of takes them): a stencil cell none of whose
        // points lies within rc + 0.01 A of the atom is skipped (about a third of the forward half
        // for half-width cells).  Orthorhombic boxes: the exact distance to the cell's box; others
        // the lower bound max_k gap_k width_k (gap_k the fractional gap along k).  The margin
        // covers the FP32 prefilter band (rc +- 2e-3 A) and the rounding of the binning, so the
        // kept pairs are unchanged.
        double sfr[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double v = pi[0] * a.boxd.hinv[k] + pi[1] * a.boxd.hinv[3 + k] + pi[2] * a.boxd.hinv[6 + k];
            sfr[k] = v - floor(v);
        }
        const bool ortho = a.boxd.h[1] == 0.0 && a.boxd.h[2] == 0.0 && a.boxd.h[3] == 0.0 && a.boxd.h[5] == 0.0 &&
                           a.boxd.h[6] == 0.0 && a.boxd.h[7] == 0.0;
        const double rprune = a.rc + 0.01;
        int carry = 0;
        if (lane == 0) s_off[wl][0] = 0;
        for (int q0 = 0; q0 < NQ; q0 += 32) {
            const int q = q0 + lane;
            int cnt = 0;
            if (q < NQ) {
                const int qq = q + NQ - 1;  // (0, 0, 0) and the offsets after it
                const int dx = qq / (W * W) - S, dy = (qq / W) % W - S, dz = qq % W - S;
                const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
                const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
                const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
                const int cc = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                int cs = a.cell_start[cc];
                const int ce = a.cell_start[cc + 1];
                if (q == 0) cs = max(cs, ks + 1);  // own cell: the atoms after i in cell order
                cnt = max(ce - cs, 0);
                if (q > 0) {
                    const int dd[3] = {dx, dy, dz};
                    double d2 = 0.0, dmax = 0.0;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double lo = (double)(c3[k] + dd[k]) / a.nc[k], hi = (double)(c3[k] + dd[k] + 1) / a.nc[k];
                        const double gap = fmax(0.0, fmax(lo - sfr[k], sfr[k] - hi)) * a.width[k];
                        d2 += gap * gap;
                        dmax = fmax(dmax, gap);
                    }
                    if (ortho ? d2 > rprune * rprune : dmax > rprune) cnt = 0;
                }
                s_beg[wl][q] = cs;
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (q < NQ) s_off[wl][q + 1] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        __syncwarp();
        const int total = carry;
        const int lo = a.cov_lo[i], hi = a.cov_hi[i];
        const bool lj = a.type != nullptr;
        const int ti = lj ? a.type[i] : 0;
        const T qi = a.qT[i];
        T g0 = T(0), g1 = T(0), g2 = T(0);
        T acc[11];  // per-lane sums of about 40 pairs, in kernel precision
#pragma unroll
        for (int k = 0; k < 11; ++k) acc[k] = T(0);
        const unsigned lt = (1u << lane) - 1u;
        int qn = 0;  // queued kept candidates (warp-uniform)
        int qc = 0;
        for (int base = 0; base < total; base += 32) {
            const int t = base + lane;
            bool keep = false;
            int j = -1;
            if (t < total) {
                while (t >= s_off[wl][qc + 1]) ++qc;
                const float4 pj = a.posc[s_beg[wl][qc] + (t - s_off[wl][qc])];
                j = __float_as_int(pj.w);
                if (j != i) {
                    const float d0 = pj.x - pix, d1 = pj.y - piy, d2 = pj.z - piz;
                    bool amb = false;
                    float sf[3];
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        const float tt = d0 * hif[q] + d1 * hif[3 + q] + d2 * hif[6 + q];
                        sf[q] = tt - floorf(tt + 0.5f);
                        amb |= fabsf(sf[q]) > 0.4999f;
                    }
                    const float e0 = sf[0] * hf[0] + sf[1] * hf[3] + sf[2] * hf[6];
                    const float e1 = sf[0] * hf[1] + sf[1] * hf[4] + sf[2] * hf[7];
                    const float e2 = sf[0] * hf[2] + sf[1] * hf[5] + sf[2] * hf[8];
                    const float r2 = e0 * e0 + e1 * e1 + e2 * e2;
                    if (!amb && r2 < rlo2) keep = true;
                    else if (!amb && r2 > rhi2) keep = false;
                    else keep = j > i ? within_rc(a.boxd, pi, a.pos + 3 * j, a.rc)
                                      : within_rc(a.boxd, a.pos + 3 * j, pi, a.rc);
                }
            }
            if (keep) red[11] += 1.0;
            // topologically scaled pairs belong to the FP64 covalent pass
            if (keep && j >= lo && j <= hi) {
                const int nbd = j > i ? lookup_nbond(a.cov, i, j) : lookup_nbond(a.cov, j, i);
                if (nbd != 0) keep = false;
            }
            // queue the kept candidates; evaluate them 32 at a time with every lane busy
            const unsigned mk = __ballot_sync(0xffffffffu, keep);
            if (keep) s_q[wl][qn + __popc(mk & lt)] = j;
            qn += __popc(mk);
            __syncwarp();
            if (qn >= 32) {
                nb_cell_pair<T>(a, i, s_q[wl][lane], pi, bxd, lj, ti, qi, g0, g1, g2, acc);
                __syncwarp();
                if (lane < qn - 32) s_q[wl][lane] = s_q[wl][32 + lane];
                qn -= 32;
                __syncwarp();
            }
        }
        if (lane < qn)
            nb_cell_pair<T>(a, i, s_q[wl][lane], pi, bxd, lj, ti, qi, g0, g1, g2, acc);
#pragma unroll
        for (int k = 0; k < 11; ++k) red[k] = (double)acc[k];
        g0 = warp_sum(g0);
        g1 = warp_sum(g1);
        g2 = warp_sum(g2);
        if (lane == 0) {
            atomicAdd(a.grad + 3 * i, g0);
            atomicAdd(a.grad + 3 * i + 1, g1);
            atomicAdd(a.grad + 3 * i + 2, g2);
        }
    }
    block_reduce_add<12>(red, a.scal);
}

}  // namespace dmffb
