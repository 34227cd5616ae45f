// The whole induced-dipole CG solve in one persistent cooperative launch (FP32 engines, meshes of
// at most 64 points per axis).
//
// The dipole solve of the reference (pme.py:342-423 solves A U = -E_perm by fixed-point steps;
// the engine uses preconditioned CG on the same linear system) repeats, per iteration, a chain of
// dependent passes on data that sits in L2: direction update, real-space matvec and dipole spread,
// 3-D FFT, influence multiply, inverse FFT, field gather, CG update.  Launched one kernel per pass
// (and the convergence test on the host every few iterations), a small box spends ~60 us per
// iteration in launch gaps and host round trips.  Here one cooperative grid runs every iteration
// and decides convergence on the device; the passes are separated by a grid barrier:
//   A  p = z + beta p                                   (beta = rz_k-1 / rz_k-2)
//   B  matvec warps (fmv = A_real p, p . fmv) and spread warps (p onto the mesh)
//   C  forward x-plane FFT passes        D  spectrum columns (x FFT, * G, inverse x FFT)
//   E  inverse x-plane FFT passes        F  field gather (Ap, p . Ap)
//   G  alpha = rz / pAp, x += alpha p, r -= alpha (Ap + fmv), z = M r, rz and rr reduced
// (with phase_ns set, block 0 adds the device-clock time of each pass, barrier included)
// then rr decides: stop when sqrt(rr / 3n) <= tol sqrt(bb / 3n) or at max_iter.
//
// The four reduced scalars of iteration k accumulate in slot k mod 4 of acc[4][4] and are read
// after the barriers of iteration k (each CTA keeps the rz of the two previous iterations in
// registers); slot k + 1 is cleared in pass A of iteration k, three iterations after its last
// reads.
//
// The grid barrier is an arrival counter and a generation word (release on arrival, acquire on
// the wait).  Every wait is bounded by the device clock: past `wait_ns` the CTA records
// DMFFB_CG_TIMEOUT in the status word and leaves; the others leave at their next barrier (which
// can no longer complete, so their own waits run out as well), and the host reads the status.
#pragma once
#include <cuda/atomic>

#include "admp_fftconv.cuh"
#include "admp_real.cuh"
#include "admp_recip.cuh"
#include "common.cuh"

namespace dmffb {

constexpr int kCgThreads = 512;
constexpr int DMFFB_CG_TIMEOUT = 1;    // a grid barrier wait ran out
constexpr int DMFFB_CG_NONFINITE = 2;  // non-finite residual

struct CgBarrier {
    unsigned* count;  // arrivals of the current generation
    unsigned* gen;    // generation
    int* status;      // 0, or DMFFB_CG_* of the first failure
    long long wait_ns;
    unsigned phantom;  // arrivals expected beyond the grid's CTAs (0; a test sets 1 to make waits run out)
};

struct CgStatus {
    int iters;
    int converged;
    int status;
    int pad;
    double rr;  // r . r at exit
};

__device__ __forceinline__ long long cg_clock_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// grid-wide barrier of nblocks co-resident CTAs; false when this CTA must leave (a wait ran out
// here or a failure was recorded anywhere)
__device__ inline bool cg_grid_sync(const CgBarrier& b, unsigned nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> cnt(*b.count), gen(*b.gen);
        cuda::atomic_ref<int, cuda::thread_scope_device> st(*b.status);
        const unsigned g = gen.load(cuda::memory_order_relaxed);
        int ok = 1;
        if (cnt.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks + b.phantom - 1) {
            cnt.store(0u, cuda::memory_order_relaxed);
            gen.store(g + 1u, cuda::memory_order_release);
        } else {
            const long long t0 = cg_clock_ns();
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (st.load(cuda::memory_order_relaxed) != 0 || cg_clock_ns() - t0 > b.wait_ns) {
                    int expect = 0;
                    st.compare_exchange_strong(expect, DMFFB_CG_TIMEOUT, cuda::memory_order_relaxed);
                    ok = 0;
                    break;
                }
                __nanosleep(40);
            }
        }
        if (st.load(cuda::memory_order_acquire) != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

struct CgSolveArgs {
    int n;
    // CG vectors [3n] (double) and the polarizabilities [n]
    double *x, *r, *z, *p, *Ap, *fmv;
    const double* pol;
    // real-space matvec
    CsrArgs csr;
    const MvCoef<float>* coef;
    const float* pos4;
    BoxT<float> bxT;
    // spread / gather
    StencilCache<float> st;
    MeshGeom g;
    int perm_mul;
    double gscale;  // 2 * DIELECTRIC
    double self1;
    // convolution (grid_in: the spread mesh, grid_out: the convolved mesh)
    FftConvArgs fc;
    // scalars
    double* acc;         // [4][4] {p.Ap recip, p.fmv, rz, rr}, zero at launch
    const double* init;  // [0] r.z, [3] r.r, [4] b.b of the initial residual
    double tol;
    int max_iter;
    CgBarrier bar;
    CgStatus* out;
    unsigned long long* phase_ns;  // [8] time per pass summed over the iterations (block 0), or null
};

__global__ void __launch_bounds__(kCgThreads) k_cg_solve(CgSolveArgs a) {
    extern __shared__ float2 sm[];
    const unsigned nb = gridDim.x;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int lane = tid & 31;
    const int warps_cta = nth >> 5;
    const int gwarp = blockIdx.x * warps_cta + (tid >> 5), nwarps = nb * warps_cta;
    const int m3 = 3 * a.n;
    // stage twiddles of the three line lengths stay in shared memory for the whole solve
    const size_t work = fc_plane_work(a.fc.K) > fc_col_work(a.fc.K) ? fc_plane_work(a.fc.K) : fc_col_work(a.fc.K);
    float2* twx = sm + work / sizeof(float2);
    float2* twy = twx + kFcTw;
    float2* twz = twy + kFcTw;
    fc_load_twiddles(twx, a.fc.tw[0], tid, nth);
    fc_load_twiddles(twy, a.fc.tw[1], tid, nth);
    fc_load_twiddles(twz, a.fc.tw[2], tid, nth);
    __syncthreads();
    SpreadArgs<float> sa;
    sa.n = a.n;
    sa.pos = nullptr;
    sa.Qg = nullptr;
    sa.U = a.p;
    sa.q1 = nullptr;
    sa.lmax = 1;
    sa.g = a.g;
    sa.grid = a.fc.grid_in;
    sa.perm_mul = a.perm_mul;
    FieldCombine cmb;
    cmb.U = a.p;
    cmb.pol = a.pol;
    cmb.self1 = a.self1;
    cmb.dot_out = a.acc;  // only tested for non-null; the sum goes through block_reduce_add
    const double rms_b = sqrt(a.init[4] / (double)m3);
    double rr = a.init[3];
    int it = 0, conv = 0, status = 0;
    double rz1 = a.init[0], rz2 = 0.0;  // rz of iterations k - 1 and k - 2
    const int ncol = a.fc.K[1] * a.fc.Kh;
    const int ncb = (ncol + kFcCols - 1) / kFcCols;
    // pass timing on block 0 (device clock at each barrier exit)
    const bool timed = a.phase_ns && blockIdx.x == 0 && tid == 0;
    long long tp = timed ? cg_clock_ns() : 0;
    auto mark = [&](int ph) {
        if (timed) {
            const long long t = cg_clock_ns();
            a.phase_ns[ph] += (unsigned long long)(t - tp);
            tp = t;
        }
    };
    while (true) {
        const double rms = sqrt(rr / (double)m3);
        if (!isfinite(rms)) {
            status = DMFFB_CG_NONFINITE;
            break;
        }
        if (rms <= a.tol * rms_b) {
            conv = 1;
            break;
        }
        if (it >= a.max_iter) break;
        double* acc = a.acc + 4 * (it & 3);
        // A: direction; clear the next iteration's scalars
        const double beta = rz2 != 0.0 ? rz1 / rz2 : 0.0;
        for (int k = blockIdx.x * nth + tid; k < m3; k += nb * nth) a.p[k] = a.z[k] + beta * a.p[k];
        if (blockIdx.x == 0 && tid < 4) a.acc[4 * ((it + 1) & 3) + tid] = 0.0;
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(0);
        // B: real-space matvec warps [0, n), spread warps [n, 2n)
        {
            double d[1] = {0.0};
            for (int w = gwarp; w < 2 * a.n; w += nwarps) {
                if (w < a.n) d[0] += matvec_atom<float>(a.csr, a.coef, a.pos4, a.bxT, a.p, a.fmv, w, lane);
                else spread_dip_atom<float>(sa, a.st, w - a.n, lane);
            }
            block_reduce_add<1>(d, acc + 1);
        }
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(1);
        // C, D, E: the convolution
        for (int x = blockIdx.x; x < a.fc.K[0]; x += nb) fc_fwd_plane(a.fc, x, sm, twy, twz);
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(2);
        for (int c = blockIdx.x; c < ncb; c += nb) fc_column_block(a.fc, c * kFcCols, sm, twx);
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(3);
        for (int x = blockIdx.x; x < a.fc.K[0]; x += nb) fc_inv_plane(a.fc, x, sm, twy, twz);
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(4);
        // F: field gather, Ap = recip field of p + (1/pol + self) p
        {
            double d[1] = {0.0};
            for (int w = gwarp; w < a.n; w += nwarps)
                d[0] += gather_field_atom<float>(a.st, a.g, a.fc.grid_out, a.gscale, a.Ap, cmb, w, lane);
            block_reduce_add<1>(d, acc + 0);
        }
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(5);
        // G: update
        {
            const double pAp = acc[0] + acc[1];
            const double alpha = pAp != 0.0 ? rz1 / pAp : 0.0;
            double v[2] = {0.0, 0.0};
            for (int k = blockIdx.x * nth + tid; k < m3; k += nb * nth) {
                double pp = a.pol[k / 3];
                pp = pp < 1e-8 ? 1e-8 : pp;
                a.x[k] += alpha * a.p[k];
                const double rv = a.r[k] - alpha * (a.Ap[k] + a.fmv[k]);
                a.r[k] = rv;
                const double zv = rv * pp / DMFFB_DIELECTRIC;
                a.z[k] = zv;
                v[0] += rv * zv;
                v[1] += rv * rv;
            }
            block_reduce_add<2>(v, acc + 2);
        }
        if (!cg_grid_sync(a.bar, nb)) break;
        mark(6);
        rz2 = rz1;
        rz1 = acc[2];
        rr = acc[3];
        ++it;
    }
    if (blockIdx.x == 0 && tid == 0) {
        cuda::atomic_ref<int, cuda::thread_scope_device> st(*a.bar.status);
        const int bst = st.load(cuda::memory_order_acquire);
        a.out->iters = it;
        a.out->converged = conv;
        a.out->status = bst != 0 ? bst : status;
        a.out->rr = rr;
    }
}

// dynamic shared memory of k_cg_solve: the larger FFT working area + three twiddle tables
__host__ inline size_t cg_solve_smem(const int K[3]) {
    const size_t pw = fc_plane_work(K), cw = fc_col_work(K);
    return (pw > cw ? pw : cw) + 3 * kFcTw * sizeof(float2);
}

}  // namespace dmffb
