// Cell-list neighbour build (sm_100a), replacing the freud AABB query behind
// NeighborList.allocate (dmff/common/nblist.py:27-55).
//
// Output rows (i, j, nbond), i < j, sorted by i: exactly the pairs whose minimum-image distance
// (the reference's pbc_shift, spatial.py:14-32) is < rc, with nbond read from a sparse
// covalent map (the reference reads a dense N x N map, nblist.py:22-25).  The distance test
// runs in FP64 with every product and sum rounded separately in a fixed order, so the pair set
// is reproducible bit for bit by an elementwise float64 computation on the host.
//
// Atoms are binned by fractional coordinates into nc_k >= 3 cells per axis (cell width >=
// rc measured perpendicular to the other two lattice vectors), counting-sorted by cell,
// and each atom scans the 27 surrounding cells twice (count, then write).
#pragma once
#include "common.cuh"

namespace dmffb {

struct NbArgs {
    int n;
    const double* pos;
    Box box;
    double rc;
    int nc[3];
    const int32_t* cell_start;  // [ncell+1]
    const int32_t* cell_atoms;  // [n]
    const int32_t* cov_ptr;     // [n+1] rows of j > i
    const int32_t* cov_j;
    const int32_t* cov_nb;
    const int32_t* cov_lo = nullptr;  // [n] smallest / largest covalent partner (either direction) or null
    const int32_t* cov_hi = nullptr;
    int32_t* count;             // [n] (pass 0) per-atom pair counts
    const int64_t* offset;      // [n+1] (pass 1)
    int32_t* pairs;             // [cap*3]
    int64_t cap;
};

// exact, non-contracted FP64 minimum-image distance test (order: x, y, z; left to right)
__device__ __forceinline__ bool within_rc(const Box& b, const double* pi, const double* pj, double rc) {
    const double d0 = __dsub_rn(pj[0], pi[0]);
    const double d1 = __dsub_rn(pj[1], pi[1]);
    const double d2 = __dsub_rn(pj[2], pi[2]);
    double s[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double t = __dadd_rn(__dadd_rn(__dmul_rn(d0, b.hinv[k]), __dmul_rn(d1, b.hinv[3 + k])), __dmul_rn(d2, b.hinv[6 + k]));
        s[k] = __dsub_rn(t, floor(__dadd_rn(t, 0.5)));
    }
    double e[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        e[c] = __dadd_rn(__dadd_rn(__dmul_rn(s[0], b.h[c]), __dmul_rn(s[1], b.h[3 + c])), __dmul_rn(s[2], b.h[6 + c]));
    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(e[0], e[0]), __dmul_rn(e[1], e[1])), __dmul_rn(e[2], e[2]));
    return __dsqrt_rn(r2) < rc;
}

__device__ __forceinline__ int cell_of(const Box& b, const int nc[3], const double* p, int c3[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double s = p[0] * b.hinv[k] + p[1] * b.hinv[3 + k] + p[2] * b.hinv[6 + k];
        s -= floor(s);
        int c = (int)(s * nc[k]);
        c = c < 0 ? 0 : (c >= nc[k] ? nc[k] - 1 : c);
        c3[k] = c;
    }
    return (c3[0] * nc[1] + c3[1]) * nc[2] + c3[2];
}

static __global__ void k_cell_count(int n, const double* pos, Box b, int nc0, int nc1, int nc2, int32_t* atom_cell,
                             int32_t* cell_count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nc[3] = {nc0, nc1, nc2};
    int c3[3];
    const int c = cell_of(b, nc, pos + 3 * i, c3);
    atom_cell[i] = c;
    atomicAdd(cell_count + c, 1);
}

static __global__ void k_cell_fill(int n, const int32_t* atom_cell, const int32_t* cell_start, int32_t* cursor,
                            int32_t* cell_atoms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int c = atom_cell[i];
    const int k = atomicAdd(cursor + c, 1);
    cell_atoms[cell_start[c] + k] = i;
}

__device__ __forceinline__ int lookup_nbond(const NbArgs& a, int i, int j) {
    for (int k = a.cov_ptr[i]; k < a.cov_ptr[i + 1]; ++k)
        if (a.cov_j[k] == j) return a.cov_nb[k];
    return 0;
}

// pass 0: count pairs per atom; pass 1: write rows at offset[i]
template <int PASS>
__global__ void __launch_bounds__(128) k_pairs(NbArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double* pi = a.pos + 3 * i;
    int c3[3];
    cell_of(a.box, a.nc, pi, c3);
    int cnt = 0;
    int64_t out = (PASS == 1) ? a.offset[i] : 0;
    for (int dx = -1; dx <= 1; ++dx) {
        const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
        for (int dy = -1; dy <= 1; ++dy) {
            const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
            for (int dz = -1; dz <= 1; ++dz) {
                const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
                const int c = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                for (int k = a.cell_start[c]; k < a.cell_start[c + 1]; ++k) {
                    const int j = a.cell_atoms[k];
                    if (j <= i) continue;
                    if (!within_rc(a.box, pi, a.pos + 3 * j, a.rc)) continue;
                    if (PASS == 1) {
                        if (out < a.cap) {
                            a.pairs[3 * out] = i;
                            a.pairs[3 * out + 1] = j;
                            a.pairs[3 * out + 2] = lookup_nbond(a, i, j);
                        }
                        ++out;
                    } else {
                        ++cnt;
                    }
                }
            }
        }
    }
    if (PASS == 0) a.count[i] = cnt;
}

// small boxes (fewer than 3 cells on an axis): every j > i is a candidate
template <int PASS>
__global__ void __launch_bounds__(128) k_pairs_all(NbArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double* pi = a.pos + 3 * i;
    int cnt = 0;
    int64_t out = (PASS == 1) ? a.offset[i] : 0;
    for (int j = i + 1; j < a.n; ++j) {
        if (!within_rc(a.box, pi, a.pos + 3 * j, a.rc)) continue;
        if (PASS == 1) {
            if (out < a.cap) {
                a.pairs[3 * out] = i;
                a.pairs[3 * out + 1] = j;
                a.pairs[3 * out + 2] = lookup_nbond(a, i, j);
            }
            ++out;
        } else {
            ++cnt;
        }
    }
    if (PASS == 0) a.count[i] = cnt;
}


// Warp-per-atom variant: lanes stride over the candidates of each of the 27 cells; a FP32
// distance decides every candidate farther than 1e-3 A from the cutoff (and away from a
// half-box image ambiguity), the exact FP64 test decides the rest, so the pair set is the one
// of within_rc.  Output order: ballot prefix within each chunk keeps rows sorted by i.
template <int PASS>
__global__ void __launch_bounds__(256) k_pairs_warp(NbArgs a) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const double* pi = a.pos + 3 * i;
    const double pix = pi[0], piy = pi[1], piz = pi[2];
    float hf[9], hif[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { hf[k] = (float)a.box.h[k]; hif[k] = (float)a.box.hinv[k]; }
    const float rlo = (float)(a.rc - 1e-3), rhi = (float)(a.rc + 1e-3);
    const float rlo2 = rlo * rlo, rhi2 = rhi * rhi;
    int c3[3];
    cell_of(a.box, a.nc, pi, c3);
    int64_t out = (PASS == 1) ? a.offset[i] : 0;
    int cnt = 0;
    const unsigned lt = (1u << lane) - 1u;
    for (int dx = -1; dx <= 1; ++dx) {
        const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
        for (int dy = -1; dy <= 1; ++dy) {
            const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
            for (int dz = -1; dz <= 1; ++dz) {
                const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
                const int c = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                const int cs = a.cell_start[c], ce = a.cell_start[c + 1];
                for (int base = cs; base < ce; base += 32) {
                    const int k = base + lane;
                    bool keep = false;
                    int j = -1;
                    if (k < ce) {
                        j = a.cell_atoms[k];
                        if (j > i) {
                            const double* pj = a.pos + 3 * j;
                            const float d0 = (float)(pj[0] - pix), d1 = (float)(pj[1] - piy), d2 = (float)(pj[2] - piz);
                            bool amb = false;
                            float sf[3];
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                float t = d0 * hif[q] + d1 * hif[3 + q] + d2 * hif[6 + q];
                                float nn = floorf(t + 0.5f);
                                sf[q] = t - nn;
                                amb |= fabsf(sf[q]) > 0.4999f;
                            }
                            const float e0 = sf[0] * hf[0] + sf[1] * hf[3] + sf[2] * hf[6];
                            const float e1 = sf[0] * hf[1] + sf[1] * hf[4] + sf[2] * hf[7];
                            const float e2 = sf[0] * hf[2] + sf[1] * hf[5] + sf[2] * hf[8];
                            const float r2 = e0 * e0 + e1 * e1 + e2 * e2;
                            if (!amb && r2 < rlo2) keep = true;
                            else if (!amb && r2 > rhi2) keep = false;
                            else keep = within_rc(a.box, pi, pj, a.rc);
                        }
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, keep);
                    if (PASS == 1) {
                        if (keep) {
                            const int64_t slot = out + __popc(m & lt);
                            if (slot < a.cap) {
                                a.pairs[3 * slot] = i;
                                a.pairs[3 * slot + 1] = j;
                                a.pairs[3 * slot + 2] = lookup_nbond(a, i, j);
                            }
                        }
                        out += __popc(m);
                    } else {
                        cnt += __popc(m);
                    }
                }
            }
        }
    }
    if (PASS == 0 && lane == 0) a.count[i] = cnt;
}


// Same cell scan emitting both layouts the engine uses: half rows (i, j, nbond), j > i, sorted
// by i (pair kernels), and the full neighbour CSR (j != i, packed j | scale index << 28) for the
// atomics-free CG matvec.  Positions for the FP32 prefilter come from the FP32 copy (posf);
// borderline candidates fall back to the exact FP64 test on pos.
struct Nb2Args {
    NbArgs a;
    const float* posf;      // [n*4]
    int32_t* count_f;       // [n] pass 0: full-list counts (null: half rows only, no CSR)
    const int64_t* off_f;   // [n+1] pass 1
    int32_t* ent;           // [cap_f]
    int64_t cap_f;
    // keep masks of the candidate batches (k_pairs_warp3): pass 0 stores one word per batch of 32
    // candidates at mask[i * mask_stride + batch] when the atom's batches fit the stride; pass 1
    // reads them instead of repeating the distance tests (null: no masks)
    uint32_t* mask = nullptr;
    int mask_stride = 0;
    // single-pass build (k_pairs_cell pass 2): the distance tests run once and each atom's full-
    // list entries and half rows go to fixed slots, ell_ent[i * ell_cap_f + k] and
    // ell_rows[3 (i * ell_cap_h + k)], which k_ell_compact then copies to the offsets the scans
    // of the true counts give; slots past a capacity are dropped (the counts and maxdeg tell)
    int32_t* ell_ent = nullptr;
    int32_t* ell_rows = nullptr;
    int ell_cap_f = 0, ell_cap_h = 0;
    int* maxdeg = nullptr;  // [2] largest half-row and full-list count over the atoms (passes 0 and 2)
};

template <int PASS>
__global__ void __launch_bounds__(256) k_pairs_warp2(Nb2Args b) {
    const NbArgs& a = b.a;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= a.n) return;
    const double* pi = a.pos + 3 * i;
    const float pix = b.posf[4 * i], piy = b.posf[4 * i + 1], piz = b.posf[4 * i + 2];
    float hf[9], hif[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { hf[k] = (float)a.box.h[k]; hif[k] = (float)a.box.hinv[k]; }
    // FP32 positions carry ~1e-5 A rounding at 100 A: the 2e-3 A band around rc goes to FP64
    const float rlo = (float)(a.rc - 2e-3), rhi = (float)(a.rc + 2e-3);
    const float rlo2 = rlo * rlo, rhi2 = rhi * rhi;
    int c3[3];
    cell_of(a.box, a.nc, pi, c3);
    int64_t out_h = (PASS == 1) ? a.offset[i] : 0, out_f = (PASS == 1 && b.off_f) ? b.off_f[i] : 0;
    int cnt_h = 0, cnt_f = 0;
    const unsigned lt = (1u << lane) - 1u;
    for (int dx = -1; dx <= 1; ++dx) {
        const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
        for (int dy = -1; dy <= 1; ++dy) {
            const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
            for (int dz = -1; dz <= 1; ++dz) {
                const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
                const int c = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                const int cs = a.cell_start[c], ce = a.cell_start[c + 1];
                for (int base = cs; base < ce; base += 32) {
                    const int k = base + lane;
                    bool keep = false;
                    int j = -1;
                    if (k < ce) {
                        j = a.cell_atoms[k];
                        if (j != i) {
                            const float d0 = b.posf[4 * j] - pix, d1 = b.posf[4 * j + 1] - piy, d2 = b.posf[4 * j + 2] - piz;
                            bool amb = false;
                            float sf[3];
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                float t = d0 * hif[q] + d1 * hif[3 + q] + d2 * hif[6 + q];
                                float nn = floorf(t + 0.5f);
                                sf[q] = t - nn;
                                amb |= fabsf(sf[q]) > 0.4999f;
                            }
                            const float e0 = sf[0] * hf[0] + sf[1] * hf[3] + sf[2] * hf[6];
                            const float e1 = sf[0] * hf[1] + sf[1] * hf[4] + sf[2] * hf[7];
                            const float e2 = sf[0] * hf[2] + sf[1] * hf[5] + sf[2] * hf[8];
                            const float r2 = e0 * e0 + e1 * e1 + e2 * e2;
                            if (!amb && r2 < rlo2) keep = true;
                            else if (!amb && r2 > rhi2) keep = false;
                            // exact test on the (lower, higher) orientation, as the half list defines it
                            else keep = j > i ? within_rc(a.box, pi, a.pos + 3 * j, a.rc)
                                              : within_rc(a.box, a.pos + 3 * j, pi, a.rc);
                        }
                    }
                    const bool up = keep && j > i;
                    const unsigned mf = __ballot_sync(0xffffffffu, keep);
                    const unsigned mh = __ballot_sync(0xffffffffu, up);
                    if (PASS == 1) {
                        if (keep) {
                            const int nbd = j > i ? lookup_nbond(a, i, j) : lookup_nbond(a, j, i);
                            int sidx = nbd - 1;
                            if (sidx < 0) sidx += 6;
                            const int64_t sf_ = out_f + __popc(mf & lt);
                            if (b.ent && sf_ < b.cap_f) b.ent[sf_] = j | (sidx << 28);
                            if (up) {
                                const int64_t sh = out_h + __popc(mh & lt);
                                if (sh < a.cap) {
                                    a.pairs[3 * sh] = i;
                                    a.pairs[3 * sh + 1] = j;
                                    a.pairs[3 * sh + 2] = nbd;
                                }
                            }
                        }
                        out_f += __popc(mf);
                        out_h += __popc(mh);
                    } else {
                        cnt_f += __popc(mf);
                        cnt_h += __popc(mh);
                    }
                }
            }
        }
    }
    if (PASS == 0 && lane == 0) {
        a.count[i] = cnt_h;
        if (b.count_f) b.count_f[i] = cnt_f;
    }
}

// k_pairs_warp2 over a finer cell grid: cells at least rc / S wide and a (2S + 1)^3 stencil
// (S = 2: 125 cells of half width, about 0.58 of the 27-cell search volume).  The warp first
// lays the stencil's cells out as one concatenated candidate list (cell starts and a prefix sum of
// their counts in shared memory, in the dx, dy, dz order of the 27-cell scan), then walks it in
// full 32-lane batches; each lane finds its candidate's cell by advancing a cursor (lanes move
// forward monotonically).  Rows come out grouped by i like the coarse scan's.
constexpr int kNbWarps = 8;  // warps per block of k_pairs_warp3
constexpr size_t kNbStageBytes = 44u << 10;  // largest candidate stage of k_pairs_cell: with its static
                                              // shared arrays it stays under the 48 KB default

template <int PASS, int S>
__global__ void __launch_bounds__(32 * kNbWarps) k_pairs_warp3(Nb2Args b) {
    constexpr int W = 2 * S + 1, NQ = W * W * W;
    __shared__ int s_beg[kNbWarps][NQ];
    __shared__ int s_off[kNbWarps][NQ + 1];
    const NbArgs& a = b.a;
    const int wl = threadIdx.x >> 5;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= a.n) return;  // whole warps leave together
    const double* pi = a.pos + 3 * i;
    const float pix = b.posf[4 * i], piy = b.posf[4 * i + 1], piz = b.posf[4 * i + 2];
    float hf[9], hif[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { hf[k] = (float)a.box.h[k]; hif[k] = (float)a.box.hinv[k]; }
    const float rlo = (float)(a.rc - 2e-3), rhi = (float)(a.rc + 2e-3);
    const float rlo2 = rlo * rlo, rhi2 = rhi * rhi;
    int c3[3];
    cell_of(a.box, a.nc, pi, c3);
    // stencil cells -> (start, count), prefix-summed in q order
    int carry = 0;
    if (lane == 0) s_off[wl][0] = 0;
    for (int q0 = 0; q0 < NQ; q0 += 32) {
        const int q = q0 + lane;
        int cnt = 0;
        if (q < NQ) {
            const int dx = q / (W * W) - S, dy = (q / W) % W - S, dz = q % W - S;
            const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
            const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
            const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
            const int cc = (cx * a.nc[1] + cy) * a.nc[2] + cz;
            const int cs = a.cell_start[cc];
            cnt = a.cell_start[cc + 1] - cs;
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
    int64_t out_h = (PASS == 1) ? a.offset[i] : 0, out_f = (PASS == 1 && b.off_f) ? b.off_f[i] : 0;
    int cnt_h = 0, cnt_f = 0;
    const unsigned lt = (1u << lane) - 1u;
    int qc = 0;
    // both passes see the same candidate list, so the masks are complete exactly when it fits
    const bool use_mask = b.mask && (total + 31) / 32 <= b.mask_stride;
    uint32_t* mrow = use_mask ? b.mask + (size_t)i * b.mask_stride : nullptr;
    for (int base = 0; base < total; base += 32) {
        const int t = base + lane;
        bool keep = false;
        int j = -1;
        if (PASS == 1 && use_mask) {
            const uint32_t mk = mrow[base >> 5];
            if (mk == 0u) continue;  // warp-uniform: no candidate of this batch is kept
            if ((mk >> lane) & 1u) {
                while (t >= s_off[wl][qc + 1]) ++qc;
                j = a.cell_atoms[s_beg[wl][qc] + (t - s_off[wl][qc])];
                keep = true;
            }
        } else if (t < total) {
            while (t >= s_off[wl][qc + 1]) ++qc;
            j = a.cell_atoms[s_beg[wl][qc] + (t - s_off[wl][qc])];
            if (j != i) {
                const float d0 = b.posf[4 * j] - pix, d1 = b.posf[4 * j + 1] - piy, d2 = b.posf[4 * j + 2] - piz;
                bool amb = false;
                float sf[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    float tt = d0 * hif[q] + d1 * hif[3 + q] + d2 * hif[6 + q];
                    float nn = floorf(tt + 0.5f);
                    sf[q] = tt - nn;
                    amb |= fabsf(sf[q]) > 0.4999f;
                }
                const float e0 = sf[0] * hf[0] + sf[1] * hf[3] + sf[2] * hf[6];
                const float e1 = sf[0] * hf[1] + sf[1] * hf[4] + sf[2] * hf[7];
                const float e2 = sf[0] * hf[2] + sf[1] * hf[5] + sf[2] * hf[8];
                const float r2 = e0 * e0 + e1 * e1 + e2 * e2;
                if (!amb && r2 < rlo2) keep = true;
                else if (!amb && r2 > rhi2) keep = false;
                else keep = j > i ? within_rc(a.box, pi, a.pos + 3 * j, a.rc)
                                  : within_rc(a.box, a.pos + 3 * j, pi, a.rc);
            }
        }
        const bool up = keep && j > i;
        const unsigned mf = __ballot_sync(0xffffffffu, keep);
        const unsigned mh = __ballot_sync(0xffffffffu, up);
        if (PASS == 0 && use_mask && lane == 0) mrow[base >> 5] = mf;
        if (PASS == 1) {
            if (keep) {
                const int nbd = j > i ? lookup_nbond(a, i, j) : lookup_nbond(a, j, i);
                int sidx = nbd - 1;
                if (sidx < 0) sidx += 6;
                const int64_t sf_ = out_f + __popc(mf & lt);
                if (b.ent && sf_ < b.cap_f) b.ent[sf_] = j | (sidx << 28);
                if (up) {
                    const int64_t sh = out_h + __popc(mh & lt);
                    if (sh < a.cap) {
                        a.pairs[3 * sh] = i;
                        a.pairs[3 * sh + 1] = j;
                        a.pairs[3 * sh + 2] = nbd;
                    }
                }
            }
            out_f += __popc(mf);
            out_h += __popc(mh);
        } else {
            cnt_f += __popc(mf);
            cnt_h += __popc(mh);
        }
    }
    if (PASS == 0 && lane == 0) {
        a.count[i] = cnt_h;
        if (b.count_f) b.count_f[i] = cnt_f;
    }
}

// Block-per-cell form of k_pairs_warp3 (same stencil, candidate order, tests and outputs): one
// CTA takes every atom of one cell.  The cell's (2S + 1)^3 neighbourhood is laid out once per CTA
// and, when it fits in `chmax` entries, staged in shared memory as (x, y, z, j) float4s, so the
// cell's atoms read their candidates from shared memory instead of each gathering them from L2;
// neighbourhoods larger than the stage fall back to the global gathers.  The NW warps of the CTA
// take the cell's atoms in turn.  ORTHO: the box is orthorhombic and the FP32 prefilter's minimum
// image is three multiplies per axis (candidates near rc still take the exact FP64 test).
template <int PASS, int S, int NW, bool ORTHO>
__global__ void __launch_bounds__(32 * NW) k_pairs_cell(Nb2Args b, int chmax) {
    constexpr int W = 2 * S + 1, NQ = W * W * W;
    __shared__ int s_beg[NQ];
    __shared__ int s_off[NQ + 1];
    extern __shared__ __align__(16) float4 s_cand[];
    const NbArgs& a = b.a;
    const int c = blockIdx.x;
    const int cs0 = a.cell_start[c], m = a.cell_start[c + 1] - cs0;
    if (m == 0) return;  // whole CTA
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c3[3] = {c / (a.nc[2] * a.nc[1]), (c / a.nc[2]) % a.nc[1], c % a.nc[2]};
    if (wl == 0) {
        int carry = 0;
        if (lane == 0) s_off[0] = 0;
        for (int q0 = 0; q0 < NQ; q0 += 32) {
            const int q = q0 + lane;
            int cnt = 0;
            if (q < NQ) {
                const int dx = q / (W * W) - S, dy = (q / W) % W - S, dz = q % W - S;
                const int cx = (c3[0] + dx + a.nc[0]) % a.nc[0];
                const int cy = (c3[1] + dy + a.nc[1]) % a.nc[1];
                const int cz = (c3[2] + dz + a.nc[2]) % a.nc[2];
                const int cc = (cx * a.nc[1] + cy) * a.nc[2] + cz;
                const int cs = a.cell_start[cc];
                cnt = a.cell_start[cc + 1] - cs;
                s_beg[q] = cs;
            }
            int incl = cnt;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (q < NQ) s_off[q + 1] = carry + incl;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
    __syncthreads();
    const int total = s_off[NQ];
    const bool staged = total <= chmax;
    if (staged) {
        int qc = 0;
        for (int t = threadIdx.x; t < total; t += blockDim.x) {
            while (t >= s_off[qc + 1]) ++qc;
            const int j = a.cell_atoms[s_beg[qc] + (t - s_off[qc])];
            s_cand[t] = make_float4(b.posf[4 * j], b.posf[4 * j + 1], b.posf[4 * j + 2], __int_as_float(j));
        }
    }
    __syncthreads();
    float hf[9], hif[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) { hf[k] = (float)a.box.h[k]; hif[k] = (float)a.box.hinv[k]; }
    const float rlo = (float)(a.rc - 2e-3), rhi = (float)(a.rc + 2e-3);
    const float rlo2 = rlo * rlo, rhi2 = rhi * rhi;
    const unsigned lt = (1u << lane) - 1u;
    for (int ai = wl; ai < m; ai += NW) {
        const int i = a.cell_atoms[cs0 + ai];
        const double* pi = a.pos + 3 * i;
        const float pix = b.posf[4 * i], piy = b.posf[4 * i + 1], piz = b.posf[4 * i + 2];
        const int64_t base_h = PASS == 2 ? (int64_t)i * b.ell_cap_h : 0, base_f = PASS == 2 ? (int64_t)i * b.ell_cap_f : 0;
        int64_t out_h = (PASS == 1) ? a.offset[i] : base_h, out_f = (PASS == 1 && b.off_f) ? b.off_f[i] : base_f;
        // where this pass writes: the final rows / CSR (pass 1) or the atom's slots (pass 2)
        int32_t* const rows_out = PASS == 2 ? b.ell_rows : a.pairs;
        int32_t* const ent_out = PASS == 2 ? b.ell_ent : b.ent;
        const int64_t lim_h = PASS == 2 ? base_h + b.ell_cap_h : a.cap;
        const int64_t lim_f = PASS == 2 ? base_f + b.ell_cap_f : b.cap_f;
        int cnt_h = 0, cnt_f = 0;
        int qc = 0;
        // covalent partners of i lie in [plo, phi]: the map is read only for those
        const int plo = a.cov_lo ? a.cov_lo[i] : 0, phi = a.cov_hi ? a.cov_hi[i] : a.n;
        const bool use_mask = b.mask && (total + 31) / 32 <= b.mask_stride;
        uint32_t* mrow = use_mask ? b.mask + (size_t)i * b.mask_stride : nullptr;
        for (int base = 0; base < total; base += 32) {
            const int t = base + lane;
            bool keep = false;
            int j = -1;
            if (PASS == 1 && use_mask) {
                const uint32_t mk = mrow[base >> 5];
                if (mk == 0u) continue;  // warp-uniform: no candidate of this batch is kept
                if ((mk >> lane) & 1u) {
                    if (staged) {
                        j = __float_as_int(s_cand[t].w);
                    } else {
                        while (t >= s_off[qc + 1]) ++qc;
                        j = a.cell_atoms[s_beg[qc] + (t - s_off[qc])];
                    }
                    keep = true;
                }
            } else if (t < total) {
                float pjx, pjy, pjz;
                if (staged) {
                    const float4 cv = s_cand[t];
                    pjx = cv.x;
                    pjy = cv.y;
                    pjz = cv.z;
                    j = __float_as_int(cv.w);
                } else {
                    while (t >= s_off[qc + 1]) ++qc;
                    j = a.cell_atoms[s_beg[qc] + (t - s_off[qc])];
                    pjx = b.posf[4 * j];
                    pjy = b.posf[4 * j + 1];
                    pjz = b.posf[4 * j + 2];
                }
                if (j != i) {
                    const float d0 = pjx - pix, d1 = pjy - piy, d2 = pjz - piz;
                    bool amb = false;
                    float r2;
                    if (ORTHO) {
                        const float dd[3] = {d0, d1, d2};
                        r2 = 0.f;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            const float tt = dd[q] * hif[4 * q];
                            const float sq = tt - floorf(tt + 0.5f);
                            amb |= fabsf(sq) > 0.4999f;
                            const float e = sq * hf[4 * q];
                            r2 = fmaf(e, e, r2);
                        }
                    } else {
                        float sf[3];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            float tt = d0 * hif[q] + d1 * hif[3 + q] + d2 * hif[6 + q];
                            float nn = floorf(tt + 0.5f);
                            sf[q] = tt - nn;
                            amb |= fabsf(sf[q]) > 0.4999f;
                        }
                        const float e0 = sf[0] * hf[0] + sf[1] * hf[3] + sf[2] * hf[6];
                        const float e1 = sf[0] * hf[1] + sf[1] * hf[4] + sf[2] * hf[7];
                        const float e2 = sf[0] * hf[2] + sf[1] * hf[5] + sf[2] * hf[8];
                        r2 = e0 * e0 + e1 * e1 + e2 * e2;
                    }
                    if (!amb && r2 < rlo2) keep = true;
                    else if (!amb && r2 > rhi2) keep = false;
                    else keep = j > i ? within_rc(a.box, pi, a.pos + 3 * j, a.rc)
                                      : within_rc(a.box, a.pos + 3 * j, pi, a.rc);
                }
            }
            const bool up = keep && j > i;
            const unsigned mf = __ballot_sync(0xffffffffu, keep);
            const unsigned mh = __ballot_sync(0xffffffffu, up);
            if (PASS == 0 && use_mask && lane == 0) mrow[base >> 5] = mf;
            if (PASS == 1 || PASS == 2) {
                if (keep) {
                    const int nbd = (j < plo || j > phi) ? 0 : (j > i ? lookup_nbond(a, i, j) : lookup_nbond(a, j, i));
                    int sidx = nbd - 1;
                    if (sidx < 0) sidx += 6;
                    const int64_t sf_ = out_f + __popc(mf & lt);
                    if (ent_out && sf_ < lim_f) ent_out[sf_] = j | (sidx << 28);
                    if (up) {
                        const int64_t sh = out_h + __popc(mh & lt);
                        if (sh < lim_h) {
                            rows_out[3 * sh] = i;
                            rows_out[3 * sh + 1] = j;
                            rows_out[3 * sh + 2] = nbd;
                        }
                    }
                }
                out_f += __popc(mf);
                out_h += __popc(mh);
            } else {
                cnt_f += __popc(mf);
                cnt_h += __popc(mh);
            }
        }
        if (PASS == 2) {
            cnt_h = (int)(out_h - base_h);
            cnt_f = (int)(out_f - base_f);
        }
        if (PASS != 1 && lane == 0) {
            a.count[i] = cnt_h;
            if (b.count_f) b.count_f[i] = cnt_f;
            if (b.maxdeg) {
                atomicMax(b.maxdeg, cnt_h);
                atomicMax(b.maxdeg + 1, cnt_f);
            }
        }
    }
}

// Copies each atom's slots of the single-pass build to its offsets in the half rows and the CSR
// (one warp per atom); nothing is written past the capacities, which the caller checks against
// the totals before it uses the lists.
static __global__ void k_ell_compact(int n, const int32_t* count_h, const int32_t* count_f, const int64_t* off_h,
                                     const int64_t* off_f, const int32_t* ell_rows, int cap_h, const int32_t* ell_ent,
                                     int cap_f, int32_t* rows, int64_t rows_cap, int32_t* ent, int64_t ent_cap) {
    const int i = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;
    const int nh = min(count_h[i], cap_h);
    const int64_t bh = off_h[i];
    for (int k = lane; k < nh; k += 32) {
        if (bh + k >= rows_cap) break;
        const int32_t* src = ell_rows + 3 * ((int64_t)i * cap_h + k);
        int32_t* dst = rows + 3 * (bh + k);
        dst[0] = src[0];
        dst[1] = src[1];
        dst[2] = src[2];
    }
    if (!ent) return;
    const int nf = min(count_f[i], cap_f);
    const int64_t bf = off_f[i];
    for (int k = lane; k < nf; k += 32) {
        if (bf + k >= ent_cap) break;
        ent[bf + k] = ell_ent[(int64_t)i * cap_f + k];
    }
}

// cell-ordered float4 copy of the positions (x, y, z, atom index as int bits)
static __global__ void k_pos_cells(int n, const double* pos, const int32_t* cell_atoms, float4* posc) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int a = cell_atoms[k];
    posc[k] = make_float4((float)pos[3 * a], (float)pos[3 * a + 1], (float)pos[3 * a + 2], __int_as_float(a));
}

static __global__ void k_pos_f32(int n, const double* pos, float* posf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    posf[4 * i] = (float)pos[3 * i];
    posf[4 * i + 1] = (float)pos[3 * i + 1];
    posf[4 * i + 2] = (float)pos[3 * i + 2];
    posf[4 * i + 3] = 0.f;
}

}  // namespace dmffb
