// libdmffb200: ADMP multipolar PME engine for B200 (sm_100a) behind the C ABI in
// include/dmffb200.h.  The handle owns every device workspace (allocated in create /
// reserve, never inside compute); callers own their inputs and outputs.
#include <cuda_runtime.h>
#include <cufft.h>
#include <cub/cub.cuh>

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <string>
#include <array>
#include <map>
#include <vector>

#include "../../include/dmffb200.h"
#include "admp_frames.cuh"
#include "admp_real.cuh"
#include "admp_recip.cuh"
#include "common.cuh"
#include "nblist.cuh"
#include "disp.cuh"
#include "classical.cuh"
#include "nbcells.cuh"
#include "admp_fftconv.cuh"
#include "admp_cgsolve.cuh"
#include "pairwise.cuh"

using namespace dmffb;

namespace {

enum {
    S_EREAL = 0,    // [0] energy, [1..9] box grad (pair kernel)
    S_RECIP = 16,   // [0] energy, [1..6] k-space tensor (conv kernel)
    S_GATHER = 24,  // [0] energy check, [1..9] X_NA
    S_SELF = 40,    // [0] E_self, [1] E_pol, [2..10] frame box grad
    S_CG = 56,      // CG scalars
    N_SCAL = 80
};

}  // namespace

struct dmffb_engine {
    // ---- static description
    int n = 0, lmax = 0, lpol = 0, lpme = 1, prec = DMFFB_FP32;
    double rc = 0, kappa = 0;
    int K[3] = {0, 0, 0};
    double ms[6], ps[6], dsc[6];
    int solver = DMFFB_SOLVER_CG;
    double cg_tol = 1e-6;
    int max_iter = 500, steps_pol = 0;
    std::string err;
    bool params_set = false;
    // ---- device data
    int32_t* d_axis_type = nullptr;
    int32_t* d_axis_idx = nullptr;
    int32_t *d_cov_ptr = nullptr, *d_cov_j = nullptr, *d_cov_nb = nullptr;
    double* d_Qloc = nullptr;
    double* d_pol = nullptr;
    void* d_thole = nullptr;
    void* d_polsix = nullptr;
    double* d_pos = nullptr;  // host-path staging
    double* d_U = nullptr;    // host-path staging / internal dipoles
    double* d_forces = nullptr;
    void* d_posT = nullptr;
    double* d_Qg = nullptr;
    void* d_QgT = nullptr;
    void* d_gpair = nullptr;
    void* d_torque = nullptr;
    void* d_fieldT = nullptr;
    double* d_grad = nullptr;
    double* d_scal = nullptr;
    double *d_b = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr, *d_Ap = nullptr, *d_fr = nullptr;
    double* d_gQ = nullptr;
    double* d_fmv = nullptr;  // CSR matvec output [3n]
    // slots of the single-pass neighbour build (k_pairs_cell pass 2): capacities per atom from
    // the largest counts of the last two-pass build (0: no slots yet)
    int32_t* d_ell_rows = nullptr;  // [n_cap * ell_cap_h * 3]
    int32_t* d_ell_ent = nullptr;   // [n_cap * ell_cap_f]
    int ell_cap_h = 0, ell_cap_f = 0;
    int* d_maxdeg = nullptr;        // [2]
    // a single-pass build whose totals are still on their way to the host: nb_finish waits for
    // them when the list is first used (and rebuilds with two passes if a slot overflowed)
    bool nb_pending = false, nb_want_csr = false;
    cudaEvent_t e_nbtot = nullptr;
    int64_t* h_nbtot = nullptr;     // pinned [4]: half rows, CSR entries, largest counts (2 x int32)
    cudaStream_t nb_stream = nullptr;
    const double* nb_pos = nullptr;
    double nb_box[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int64_t* d_csr_off = nullptr;
    int32_t *d_csr_ent = nullptr, *d_csr_deg = nullptr;
    int64_t csr_cap = 0;
    bool csr_from_build = false;     // CSR built together with the internal pair list
    const int32_t* csr_pairs = nullptr;  // the half list the current CSR belongs to
    float* d_posf = nullptr;
    void* d_mvcoef = nullptr;  // [csr_cap] MvCoef<T>
    int64_t mv_cap = 0;
    int32_t* d_pcount_f = nullptr;
    void* d_cub2 = nullptr;
    size_t cub2_bytes = 0;
    void* d_grid = nullptr;
    void* d_grid2 = nullptr;  // spread target of the dipole-only field pass, kept zero between passes
    void* d_cgrid = nullptr;
    double* d_bmod = nullptr;
    cufftHandle plan_f = 0, plan_b = 0;
    bool have_plans = false;
    // ---- neighbour list
    int32_t* d_pairs = nullptr;
    int64_t pair_cap = 0, npairs = 0;
    bool have_pairs = false;
    int32_t *d_atom_cell = nullptr, *d_cell_count = nullptr, *d_cell_start = nullptr, *d_cell_cursor = nullptr,
            *d_cell_atoms = nullptr, *d_pcount = nullptr;
    int64_t* d_poff = nullptr;
    int ncell_cap = 0;
    void* d_cub = nullptr;
    size_t cub_bytes = 0;
    double* h_scal = nullptr;  // pinned
    // ---- timing
    bool timing = false;
    cudaEvent_t ev[8];
    double t_ms[6] = {0, 0, 0, 0, 0, 0};
    // ---- per-kernel-class instrumentation (events around every launch when enabled)
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, int>> prof_marks;  // (class, event index of start)
    double kstat_ms[32] = {0};  // indexed by kernel class (KC_*), KC_COUNT <= 32
    int64_t kstat_n[32] = {0};
    int64_t n_launch = 0, n_fft = 0;
    int64_t cg_graph_launches = 0, cg_graph_ffts = 0;  // per replay of the two-iteration CG graph
    // ---- last result book-keeping
    Box last_box;
    const double* cur_pos = nullptr;  // FP64 positions of the evaluation in flight
    int perm_mul = 1;
    // ---- CG iteration graph (two iterations per launch) and the side stream of the matvec
    cudaStream_t s1 = nullptr, s2 = nullptr;  // engine work stream (capturable) and matvec side stream
    cudaEvent_t e_fork = nullptr, e_join = nullptr, e_in = nullptr, e_out = nullptr;
    cudaEvent_t e_build = nullptr;  // end of the last neighbour build on its stream (no host wait)
    cudaGraphExec_t cg_exec = nullptr;   // two CG steps
    cudaGraphExec_t cg_exec1 = nullptr;  // one CG step (fused path: an odd last segment)
    int64_t cg_graph1_launches = 0, cg_graph1_ffts = 0;
    std::vector<double> cg_key;       // what the instantiated graph bakes in
    std::vector<double> cg_seen_key;  // the previous solve's key
    bool use_graphs = true;
    // ---- dispersion PME / TT damping (engines made by dmffb_disp_create)
    int kind = 0;  // 0 ADMP multipolar PME, 1 dispersion
    int pmax = 10, tt = 0;
    void *d_c = nullptr, *d_tta = nullptr, *d_ttb = nullptr, *d_ttq = nullptr;  // kernel precision
    void *d_glr = nullptr, *d_gsr = nullptr;
    double* d_dc = nullptr;  // [3n] dE_lr/dc per channel (reciprocal part)
    double e_self_disp = 0.0;
    // ---- classical terms (engines made by dmffb_classical_create, kind 2)
    int ntypes = 0, coul = 0, pbc = 1;
    double krf = 0.0, crf = 0.0, e_self_coul = 0.0;
    double mlj[6] = {0, 0, 0, 0, 0, 0};
    double* d_q = nullptr;       // [n] FP64 charges
    void* d_qT = nullptr;        // [n] charges in kernel precision
    int32_t* d_type = nullptr;   // [n]
    void *d_sigtt = nullptr, *d_epstt = nullptr;  // [ntypes^2] kernel precision
    double *d_dq = nullptr, *d_dsig = nullptr, *d_deps = nullptr;
    int64_t nterm[3] = {0, 0, 0};
    int32_t* d_tidx[3] = {nullptr, nullptr, nullptr};
    double* d_tprm[3] = {nullptr, nullptr, nullptr};
    double* d_tdprm[3] = {nullptr, nullptr, nullptr};
    bool want_pgrad = false, charges_set = false;
    bool cell_pass = false;  // dmffb_classical_set_cell_pass: pairs from the cell grid, no list
    // dipole-solve convolution in one thread-block cluster (FP32, meshes up to 64 per axis)
    bool fc_enabled = false;  // dmffb_set_fused_fft
    int fc_ok = -1;          // the engine's FFT convolution serves this mesh (1), not (0), not decided (-1)
    float2* d_fcW = nullptr;  // [K1][K2][K3/2+1] half spectrum between its passes
    int pcg_mode = 2;         // dmffb_set_persistent_cg: 0 off, 1 on, 2 for systems of at most pcg_auto_atoms
    int pcg_auto_atoms = 4096;
    int pcg_max_blocks = -1;  // co-resident k_cg_solve CTAs for the current mesh (0: unavailable, -1: not decided)
    void* d_pcg = nullptr;    // persistent solve scalars, barrier words and status
    double pcg_wait_s = 2.0;  // limit of one grid-barrier wait
    int pcg_phantom = 0;      // arrivals the next persistent solve's barrier waits for beyond its CTAs (tests)
    double pcg_phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // pass times of the persistent solves run while profiling
    float* d_fcG = nullptr;  // [K1*K2*Kh] influence function of the half spectrum
    int64_t fcG_cap = 0;
    int32_t* d_covrows = nullptr;  // [n_covrows*3] covalent rows (i < j, nbond)
    int64_t n_covrows = 0;
    int32_t *d_cov_lo = nullptr, *d_cov_hi = nullptr;  // [n] covalent partner index range
    float4* d_posc = nullptr;  // [n] cell-ordered positions of the cell pass
    // ---- short-range pairwise terms (engines made by dmffb_pairwise_create, kind 3)
    int sr_kind = 0;
    double sr_sign = 1.0;
    void* d_srp = nullptr;      // [4n] per-atom parameters in kernel precision, channel-major
    double* d_srdp = nullptr;   // [4n] dE/dparameter
    void* d_srgrad = nullptr;   // [3n] dE/dpos in kernel precision
    bool zero_guess = false;  // dipole solves start from U = 0 (dmffb_admp_set_zero_guess)
    bool u_zeroed = false;    // this call's U was zeroed by the host-buffer entry point
    // ---- ADMP parameter adjoints (dmffb_admp_set_param_grads)
    bool admp_pgrad = false, have_pgrad = false;
    double *d_dQloc = nullptr, *d_dpa = nullptr, *d_dth = nullptr, *d_dpol = nullptr;
    double* d_dsr = nullptr;  // [4n] dE_sr/d(a, b, q, c6) (dispersion engines)
    // ---- rows with nbond != 0 (the FP64 scaled-rows launches visit only these)
    int32_t* d_srows = nullptr;
    int64_t srows_cap = 0, n_srows = 0;
    int* d_nsel = nullptr;
    int* h_nsel = nullptr;  // pinned
    void* d_cubsel = nullptr;
    size_t cubsel_bytes = 0;
    const int32_t* srows_pairs = nullptr;  // the pair list the row map belongs to
    int64_t srows_npairs = -1, srows_gen = -1, pairs_gen = 0;
    // ---- per-atom mesh stencils of the evaluation in progress (cached dipole spread / gather)
    int4* d_stc_org = nullptr;
    void* d_stc_w = nullptr;
    int64_t stc_cap = 0;
    bool stencils_ready = false;
    // ---- capacities (dmffb_admp_reconfigure reuses the allocations for systems that fit)
    int n_cap = 0;
    int64_t cov_cap = 0, grid_cap = 0, cgrid_cap = 0;
    int bmod_cap = 0;
    uint32_t* d_nbmask = nullptr;  // candidate keep masks of the neighbour count pass
    int64_t nbmask_cap = 0;
    // ---- second-order pass (dmffb_admp_backward): the point of the last compute and scratch
    bool fixed_U = false;  // compute_impl takes U as given (no dipole solve)
    bool have_last = false;
    const int32_t* last_pairs = nullptr;
    int64_t last_npairs = 0;
    double* last_U = nullptr;
    std::vector<double> h_Qloc, h_pol, h_thole;  // host copies of the last set_params
    double* d_bk = nullptr;  // [52 n] scratch of the second-order pass
    int64_t bk_cap = 0;
    std::map<std::array<int, 3>, std::pair<cufftHandle, cufftHandle>> plan_cache;  // mesh -> (R2C, C2R)
};

// completion of a single-pass neighbour build (defined after the kernels)
int nb_finish(dmffb_engine* h);
void nb_discard(dmffb_engine* h);

namespace {

int fail(dmffb_engine* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

#define CK(call)                                                                           \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return fail(h, DMFFB_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CKFFT(call)                                                                        \
    do {                                                                                   \
        cufftResult r_ = (call);                                                           \
        if (r_ != CUFFT_SUCCESS) return fail(h, DMFFB_CUFFT_ERROR, std::string(#call) + " failed"); \
    } while (0)

template <typename P>
int dalloc(dmffb_engine* h, P** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) return fail(h, DMFFB_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    // zeroed on the engine stream and waited for: the engine's streams are non-blocking, so a
    // zeroing on the legacy default stream would not be ordered before their kernels
    if (h->s1) {
        cudaMemsetAsync(*p, 0, bytes, h->s1);
        e = cudaStreamSynchronize(h->s1);
    } else {
        cudaMemset(*p, 0, bytes);
        e = cudaDeviceSynchronize();
    }
    if (e != cudaSuccess) return fail(h, DMFFB_CUDA_ERROR, std::string("zeroing: ") + cudaGetErrorString(e));
    return DMFFB_OK;
}

void make_box(const double* b, Box& bx) {
    for (int k = 0; k < 9; ++k) bx.h[k] = b[k];
    const double* m = b;
    double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
    double inv[9];
    inv[0] = (m[4] * m[8] - m[5] * m[7]) / det;
    inv[1] = (m[2] * m[7] - m[1] * m[8]) / det;
    inv[2] = (m[1] * m[5] - m[2] * m[4]) / det;
    inv[3] = (m[5] * m[6] - m[3] * m[8]) / det;
    inv[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    inv[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    inv[6] = (m[3] * m[7] - m[4] * m[6]) / det;
    inv[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    inv[8] = (m[0] * m[4] - m[1] * m[3]) / det;
    // diagonal boxes: exact reciprocals, as a LU inverse would give
    if (m[1] == 0 && m[2] == 0 && m[3] == 0 && m[5] == 0 && m[6] == 0 && m[7] == 0) {
        for (int k = 0; k < 9; ++k) inv[k] = 0.0;
        inv[0] = 1.0 / m[0];
        inv[4] = 1.0 / m[4];
        inv[8] = 1.0 / m[8];
    }
    for (int k = 0; k < 9; ++k) bx.hinv[k] = inv[k];
}

double det3(const double* m) {
    return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) + m[2] * (m[3] * m[7] - m[4] * m[6]);
}

template <typename T>
BoxT<T> boxT(const Box& b) {
    BoxT<T> r;
    for (int k = 0; k < 9; ++k) {
        r.h[k] = (T)b.h[k];
        r.hinv[k] = (T)b.hinv[k];
    }
    return r;
}

MeshGeom mesh_geom(const Box& b, const int K[3]) {
    MeshGeom g;
    // NA[j][c] = K_j * hinv[c][j]
    for (int j = 0; j < 3; ++j)
        for (int c = 0; c < 3; ++c) g.NA[3 * j + c] = K[j] * b.hinv[3 * c + j];
    for (int j = 0; j < 3; ++j)
        for (int c = 0; c < 3; ++c) g.B[3 * j + c] = g.NA[3 * c + j];
    for (int k = 0; k < 3; ++k) g.K[k] = K[k];
    return g;
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// kernel classes for dmffb_get_kernel_stats
enum { KC_PREP = 0, KC_PAIR_FULL, KC_PAIR_FIELD, KC_PAIR_MATVEC, KC_SPREAD, KC_FFT, KC_CONV, KC_GATHER_FULL,
       KC_GATHER_FIELD, KC_SELF, KC_VEC, KC_NBLIST, KC_MVCOEF,
       // FP64 launches over the topologically scaled rows, parameter-adjoint pair kernels, bonded terms
       KC_PAIR_FULL_SCALED, KC_PAIR_FIELD_SCALED, KC_PGRAD, KC_BONDED,
       KC_FFTCONV,  // the dipole solve's forward FFT + influence multiply + inverse FFT (engine FFT)
       KC_CGSOLVE,  // the whole CG solve in one persistent cooperative launch
       KC_COUNT };
static_assert(KC_COUNT <= 32, "kernel-class statistics arrays hold 32 classes");

inline void prof_begin(dmffb_engine* h, cudaStream_t s, int cls) {
    if (!h->prof) return;
    const size_t k = h->prof_marks.size() * 2;
    while (h->ev_pool.size() < k + 2) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->ev_pool.push_back(e);
    }
    cudaEventRecord(h->ev_pool[k], s);
    h->prof_marks.push_back({cls, (int)k});
}
inline void prof_end(dmffb_engine* h, cudaStream_t s) {
    if (!h->prof) return;
    cudaEventRecord(h->ev_pool[h->prof_marks.back().second + 1], s);
}
inline void prof_collect(dmffb_engine* h) {
    if (!h->prof) return;
    for (auto& m : h->prof_marks) {
        float ms = 0.f;
        cudaEventSynchronize(h->ev_pool[m.second + 1]);
        cudaEventElapsedTime(&ms, h->ev_pool[m.second], h->ev_pool[m.second + 1]);
        h->kstat_ms[m.first] += ms;
        h->kstat_n[m.first] += 1;
    }
    h->prof_marks.clear();
}
// launch one of our kernels with accounting: LAUNCH(h, stream, class, kernel<<<...>>>(args))
#define LAUNCH(H, S, CLS, ...)   \
    do {                         \
        prof_begin(H, S, CLS);   \
        __VA_ARGS__;             \
        prof_end(H, S);          \
        (H)->n_launch++;         \
    } while (0)
#define FFTCALL(H, S, ...)        \
    do {                          \
        prof_begin(H, S, KC_FFT); \
        CKFFT(__VA_ARGS__);       \
        prof_end(H, S);           \
        (H)->n_fft++;             \
    } while (0)

// ------------------------------------------------------------------ small vector kernels
// out = recip + fT + mv + (1/pol + self) U [+ self * permanent dipole]; with dot_out, also
// accumulates dot(dotv, out) into *dot_out (the p.Ap of a CG step)
template <typename T>
__global__ void k_field_combine(int n, const double* recip, const T* fT, const double* mv, const double* U,
                                const double* Qg, const double* pol, double self1, int include_perm, double* out,
                                const double* dotv, double* dot_out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double d[1] = {0.0};
    if (k < 3 * n) {
        const int a = k / 3, c = k % 3;
        double p = pol[a];
        p = p < 1e-8 ? 1e-8 : p;
        double v = recip ? recip[k] : 0.0;
        if (fT) v += (double)fT[k];
        if (mv) v += mv[k];
        if (U) v += (DMFFB_DIELECTRIC / p + self1) * U[k];
        if (include_perm) {
            const int hidx = c == 0 ? 2 : (c == 1 ? 3 : 1);
            v += self1 * Qg[9 * a + hidx];
        }
        out[k] = v;
        if (dot_out) d[0] = dotv[k] * v;
    }
    if (dot_out) block_reduce_add<1>(d, dot_out);
}

// CG helpers; scalars live in s[]: [0] rz(even) [1] rz(odd) [2] pAp [3] rr
__global__ void k_dot2(int m, const double* a, const double* b, const double* c, const double* d, double* s0,
                       double* s1) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double v0[1] = {0.0}, v1[1] = {0.0};
    if (k < m) {
        v0[0] = a[k] * b[k];
        if (c) v1[0] = c[k] * d[k];
    }
    block_reduce_add<1>(v0, s0);
    if (s1) block_reduce_add<1>(v1, s1);
}

__global__ void k_cg_init(int n, const double* b, const double* Ax, const double* pol, double* r, double* z,
                          double* p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    double pp = pol[k / 3];
    pp = pp < 1e-8 ? 1e-8 : pp;
    const double rv = -(b[k] + (Ax ? Ax[k] : 0.0));
    r[k] = rv;
    z[k] = rv * pp / DMFFB_DIELECTRIC;
    p[k] = z[k];
}

// Ap may come in two parts (Ap + Ap2, p.Ap = s[2] + s[5]); s[5] stays 0 when Ap2 is null.
// With ctr (the CG step counter, already advanced for this step), slot = (*ctr - 1) mod 2 and
// rz_new points at the slot pair s[0..1], this step's r.z going to rz_new[1 - slot].
__global__ void k_cg_update(int n, const double* s, int slot, double* x, double* r, double* z, const double* p,
                            const double* Ap, const double* pol, double* rz_new, double* rr,
                            const double* Ap2 = nullptr, const unsigned long long* ctr = nullptr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (ctr) {
        slot = (int)((*ctr - 1ull) & 1ull);
        rz_new += 1 - slot;
    }
    const double pAp = s[2] + s[5];
    const double alpha = pAp != 0.0 ? s[slot] / pAp : 0.0;
    double v[1] = {0.0}, w[1] = {0.0};
    if (k < 3 * n) {
        double pp = pol[k / 3];
        pp = pp < 1e-8 ? 1e-8 : pp;
        x[k] += alpha * p[k];
        const double ap = Ap2 ? Ap[k] + Ap2[k] : Ap[k];
        const double rv = r[k] - alpha * ap;
        r[k] = rv;
        const double zv = rv * pp / DMFFB_DIELECTRIC;
        z[k] = zv;
        v[0] = rv * zv;
        w[0] = rv * rv;
    }
    block_reduce_add<1>(v, rz_new);
    block_reduce_add<1>(w, rr);
}

// with ctr (the CG step counter, not yet advanced for this step), slot_new = *ctr mod 2
__global__ void k_cg_p(int n, const double* s, int slot_old, int slot_new, const double* z, double* p,
                       double* zero = nullptr, const unsigned long long* ctr = nullptr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (ctr) {
        slot_new = (int)(*ctr & 1ull);
        slot_old = 1 - slot_new;
    }
    if (k == 0 && zero) *zero = 0.0;
    if (k >= 3 * n) return;
    const double beta = s[slot_old] != 0.0 ? s[slot_new] / s[slot_old] : 0.0;
    p[k] = z[k] + beta * p[k];
}

__global__ void k_ref_step(int n, const double* f, const double* pol, double* U, double* maxf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    const double p = pol[k / 3];
    U[k] -= f[k] * p / DMFFB_DIELECTRIC;
    (void)maxf;
}

__global__ void k_absmax(int n, const double* f, const double* pol, double thresh_pol, unsigned long long* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    if (pol[k / 3] > thresh_pol) {
        const double v = fabs(f[k]);
        atomicMax(out, (unsigned long long)__double_as_longlong(v));
    }
}

template <typename T>
__global__ void k_set_thole(int n, const double* pol, const double* thole, T* th, T* psix) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    th[a] = thole ? (T)thole[a] : T(0);
    psix[a] = pol ? (T)pow(pol[a] > 0 ? pol[a] : 0.0, 1.0 / 6.0) : T(0);
}

// ------------------------------------------------------------------ engine pieces
// predicate of the scaled-rows selection: a valid row (i < j) with a topological scale
struct ScaledRow {
    const int32_t* p;
    __device__ __forceinline__ bool operator()(const int32_t r) const {
        return p[3 * (int64_t)r + 2] != 0 && p[3 * (int64_t)r] < p[3 * (int64_t)r + 1];
    }
};

// Indices of the rows with nbond != 0 (stable, so still sorted by i), rebuilt when the pair
// list changes: the FP64 scaled-rows launches run over these (about one row in a hundred)
// instead of over every row.
int scaled_rows(dmffb_engine* h, cudaStream_t s, const int32_t* pairs, int64_t npairs) {
    const bool internal = pairs == h->d_pairs;
    if (internal && h->srows_pairs == pairs && h->srows_npairs == npairs && h->srows_gen == h->pairs_gen)
        return DMFFB_OK;
    int st;
    if (npairs > 0x7fffffff) return fail(h, DMFFB_BAD_ARG, "too many pair rows");
    if (!h->d_nsel) {
        if ((st = dalloc(h, &h->d_nsel, sizeof(int)))) return st;
        if (cudaMallocHost((void**)&h->h_nsel, sizeof(int)) != cudaSuccess) return fail(h, DMFFB_OOM, "cudaMallocHost");
    }
    const int64_t cap_need = std::max<int64_t>(npairs, 1);
    if (cap_need > h->srows_cap) {  // capacity for every row: selection output cannot overflow
        if (h->d_srows) cudaFree(h->d_srows);
        h->d_srows = nullptr;
        h->srows_cap = cap_need + cap_need / 4;
        if ((st = dalloc(h, &h->d_srows, h->srows_cap * sizeof(int32_t)))) return st;
    }
    size_t need = 0;
    cub::CountingInputIterator<int32_t> it(0);
    cub::DeviceSelect::If(nullptr, need, it, h->d_srows, h->d_nsel, (int)npairs, ScaledRow{pairs}, s);
    if (need > h->cubsel_bytes) {
        if (h->d_cubsel) cudaFree(h->d_cubsel);
        h->d_cubsel = nullptr;
        h->cubsel_bytes = need;
        if ((st = dalloc(h, &h->d_cubsel, need))) return st;
    }
    size_t tb = h->cubsel_bytes;
    CK(cub::DeviceSelect::If(h->d_cubsel, tb, it, h->d_srows, h->d_nsel, (int)npairs, ScaledRow{pairs}, s));
    CK(cudaMemcpyAsync(h->h_nsel, h->d_nsel, sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    h->n_srows = *h->h_nsel;
    h->srows_pairs = pairs;
    h->srows_npairs = npairs;
    h->srows_gen = internal ? h->pairs_gen : -1;
    return DMFFB_OK;
}

template <typename T>
PairArgs<T> pair_args(dmffb_engine* h, const Box& bx, const int32_t* pairs, int64_t npairs, const double* U) {
    PairArgs<T> a;
    a.n = h->n;
    a.npairs = npairs;
    a.pairs = pairs;
    a.pos = (const T*)h->d_posT;
    a.posd = h->cur_pos;
    a.Qg = (const T*)h->d_QgT;
    a.Qgd = h->d_Qg;
    a.U = U;
    a.thole = (const T*)h->d_thole;
    a.polsix = (const T*)h->d_polsix;
    for (int k = 0; k < 6; ++k) {
        a.ms[k] = (T)h->ms[k];
        a.ps[k] = (T)h->ps[k];
        a.dsc[k] = (T)h->dsc[k];
    }
    a.kappa = (T)(h->lpme ? h->kappa : 0.0);
    a.boxd = bx;
    a.grad = (T*)h->d_gpair;
    a.torque = (T*)h->d_torque;
    a.field = (T*)h->d_fieldT;
    a.scal = h->d_scal + S_EREAL;
    a.want_box = 1;
    return a;
}

int lmax_eff(const dmffb_engine* h) { return (h->lmax == 0 && h->lpol) ? 1 : h->lmax; }

// reciprocal pass: spread (Qg and/or U) -> FFT -> convolution -> inverse FFT -> gather
// per-atom wrapped stencil origins and spline weights at these positions, for the cached dipole
// spread and field gather of the dipole solve
// The dynamic shared memory limit of a kernel is a property of the function, shared by every
// engine of the process (and by the server's slot threads): it is set to what the largest mesh
// served (64 points per axis) needs, the same value from every caller, never to one engine's own
// need, which another engine's smaller setting would undercut at its next launch.
const int kFcMaxMesh[3] = {kFcMaxK, kFcMaxK, kFcMaxK};

bool fc_grant_smem() {
    return cudaFuncSetAttribute(k_fc_fwd_planes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fc_plane_smem(kFcMaxMesh)) == cudaSuccess &&
           cudaFuncSetAttribute(k_fc_inv_planes, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fc_plane_smem(kFcMaxMesh)) == cudaSuccess &&
           cudaFuncSetAttribute(k_fc_columns, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)fc_col_smem(kFcMaxMesh)) == cudaSuccess &&
           cudaFuncSetAttribute(k_cg_solve, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)cg_solve_smem(kFcMaxMesh)) == cudaSuccess;
}

// Whether the engine's FFT convolution serves the current mesh: FP32, extents of at most 64 points
// and the kernels' shared memory granted; otherwise the cuFFT path runs.
int fc_decide(dmffb_engine* h) {
    if (h->fc_ok >= 0) return h->fc_ok;
    h->fc_ok = 0;
    if (h->prec != DMFFB_FP32 || !h->lpme) return 0;
    for (int k = 0; k < 3; ++k) {
        bool ok = false;
        fc_plan(h->K[k], &ok);
        if (!ok) return 0;
    }
    if (!fc_grant_smem()) {
        cudaGetLastError();
        return 0;
    }
    h->fc_ok = 1;
    return 1;
}

// influence-function table and spectrum buffer of the engine's FFT convolution for this box (once
// per dipole solve)
int fc_prepare(dmffb_engine* h, cudaStream_t s, const Box& bx) {
    const int Kh = h->K[2] / 2 + 1;
    const int64_t m = (int64_t)h->K[0] * h->K[1] * Kh;
    int st;
    if (m > h->fcG_cap) {
        if (h->d_fcG) cudaFree(h->d_fcG);
        if (h->d_fcW) cudaFree(h->d_fcW);
        h->d_fcG = nullptr;
        h->d_fcW = nullptr;
        h->fcG_cap = m;
        if ((st = dalloc(h, &h->d_fcG, m * sizeof(float)))) return st;
        if ((st = dalloc(h, &h->d_fcW, m * sizeof(float2)))) return st;
    }
    LAUNCH(h, s, KC_VEC, k_fc_gtable<<<nblk(m, 256), 256, 0, s>>>(h->K[0], h->K[1], h->K[2], Kh, bx, h->d_bmod,
                                                                  h->kappa, fabs(det3(bx.h)), h->d_fcG));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

FftConvArgs fc_args(dmffb_engine* h, float* in, float* out) {
    FftConvArgs a = {};
    for (int k = 0; k < 3; ++k) a.K[k] = h->K[k];
    a.Kh = h->K[2] / 2 + 1;
    a.grid_in = in;
    a.grid_out = out;
    a.spec = h->d_fcW;
    a.G = h->d_fcG;
    a.px = fc_plan(h->K[0]);
    a.py = fc_plan(h->K[1]);
    a.pz = fc_plan(h->K[2]);
    fc_host_twiddles(a.px, a.tw[0]);
    fc_host_twiddles(a.py, a.tw[1]);
    fc_host_twiddles(a.pz, a.tw[2]);
    return a;
}

int fc_launch(dmffb_engine* h, cudaStream_t s, float* in, float* out) {
    static_assert(sizeof(FftConvArgs) <= 4000, "launch arguments of the FFT convolution");
    FftConvArgs a = fc_args(h, in, out);
    const size_t sp = fc_plane_smem(h->K), sc = fc_col_smem(h->K);
    const int ncb = (h->K[1] * a.Kh + kFcCols - 1) / kFcCols;
    LAUNCH(h, s, KC_FFTCONV, k_fc_fwd_planes<<<h->K[0], kFcPlaneThreads, sp, s>>>(a));
    LAUNCH(h, s, KC_FFTCONV, k_fc_columns<<<ncb, kFcColThreads, sc, s>>>(a));
    LAUNCH(h, s, KC_FFTCONV, k_fc_inv_planes<<<h->K[0], kFcPlaneThreads, sp, s>>>(a));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// Co-resident CTAs of the persistent CG solve for the current mesh (0: the graph-replayed solve
// runs instead): needs the engine-FFT convolution for the mesh, the kernel's shared memory and a
// device that takes cooperative launches.
bool pcg_wanted(const dmffb_engine* h) {
    return h->pcg_mode == 1 || (h->pcg_mode == 2 && h->n <= h->pcg_auto_atoms);
}

int pcg_decide(dmffb_engine* h) {
    if (h->pcg_max_blocks >= 0) return h->pcg_max_blocks;
    h->pcg_max_blocks = 0;
    if (fc_decide(h) <= 0) return 0;
    int dev = 0, coop = 0, nsm = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop ||
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const size_t smem = cg_solve_smem(h->K);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_solve, kCgThreads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    h->pcg_max_blocks = per_sm * nsm;
    return h->pcg_max_blocks;
}


template <typename T>
int stencil_prep(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx) {
    const int n = h->n;
    int st;
    if (n > h->stc_cap) {
        if (h->d_stc_org) cudaFree(h->d_stc_org);
        if (h->d_stc_w) cudaFree(h->d_stc_w);
        h->d_stc_org = nullptr;
        h->d_stc_w = nullptr;
        h->stc_cap = n;
        if ((st = dalloc(h, &h->d_stc_org, (size_t)n * sizeof(int4)))) return st;
        if ((st = dalloc(h, &h->d_stc_w, (size_t)n * 36 * sizeof(double)))) return st;
    }
    LAUNCH(h, s, KC_VEC, k_stencil_prep<T><<<nblk(n, 128), 128, 0, s>>>(n, pos, mesh_geom(bx, h->K), h->d_stc_org,
                                                                        (T*)h->d_stc_w));
    if (sizeof(T) == 4 && (h->fc_enabled || (pcg_wanted(h) && pcg_decide(h) > 0)) && fc_decide(h) > 0 &&
        (st = fc_prepare(h, s, bx)))
        return st;
    h->stencils_ready = true;
    return DMFFB_OK;
}

template <typename T>
StencilCache<T> stencil_cache(dmffb_engine* h) {
    StencilCache<T> c;
    c.org = h->d_stc_org;
    c.w = (const T*)h->d_stc_w;
    return c;
}

template <typename T>
int recip_pass(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, bool use_Qg, const double* U,
               int mode, double* field_out, int field_acc, double* const* zero_scal = nullptr) {
    const MeshGeom g = mesh_geom(bx, h->K);
    const int64_t K3 = (int64_t)h->K[0] * h->K[1] * h->K[2];
    // the dipole-only field pass (the CG matvec) spreads into d_grid2, which the convolution
    // clears again once the forward transform has read it: no memset per pass
    const bool dip = mode == GATHER_FIELD && !use_Qg && U;
    void* spread_grid = dip ? h->d_grid2 : h->d_grid;
    if (!dip) CK(cudaMemsetAsync(h->d_grid, 0, K3 * sizeof(T), s));
    SpreadArgs<T> sa;
    sa.n = h->n;
    sa.pos = pos;
    sa.Qg = use_Qg ? (const T*)h->d_QgT : nullptr;
    sa.U = U;
    sa.q1 = nullptr;
    sa.lmax = lmax_eff(h);
    sa.g = g;
    sa.grid = (T*)spread_grid;
    sa.perm_mul = h->perm_mul;
    if (zero_scal)
        for (int k = 0; k < 3; ++k) sa.zero_scal[k] = zero_scal[k];
    if (dip && h->stencils_ready) {
        LAUNCH(h, s, KC_SPREAD, k_spread_dip_cached<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(sa, stencil_cache<T>(h)));
    } else {
        // the general spread (dipoles alone when Qg is null) clears no scalars itself
        if (zero_scal)
            for (int k = 0; k < 3; ++k)
                if (zero_scal[k]) CK(cudaMemsetAsync(zero_scal[k], 0, sizeof(double), s));
        LAUNCH(h, s, KC_SPREAD, k_spread<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(sa));
    }
    CKFFT(cufftSetStream(h->plan_f, s));
    CKFFT(cufftSetStream(h->plan_b, s));
    if (sizeof(T) == 4) {
        FFTCALL(h, s, cufftExecR2C(h->plan_f, (cufftReal*)spread_grid, (cufftComplex*)h->d_cgrid));
    } else {
        FFTCALL(h, s, cufftExecD2Z(h->plan_f, (cufftDoubleReal*)spread_grid, (cufftDoubleComplex*)h->d_cgrid));
    }
    ConvArgs<T> ca;
    for (int k = 0; k < 3; ++k) ca.K[k] = h->K[k];
    ca.Kh = h->K[2] / 2 + 1;
    ca.S = (T*)h->d_cgrid;
    ca.bmod = h->d_bmod;
    for (int k = 0; k < 9; ++k) ca.hinv[k] = bx.hinv[k];
    ca.V = fabs(det3(bx.h));
    ca.kappa = h->kappa;
    ca.escale = DMFFB_DIELECTRIC;
    ca.kind = CK_COUL;
    ca.scal = h->d_scal + S_RECIP;
    ca.want_energy = (mode == GATHER_FULL) ? 1 : 0;
    if (dip) {
        ca.zero_real = (T*)h->d_grid2;
        ca.nzero = K3;
    }
    const int64_t nk = (int64_t)h->K[0] * h->K[1] * ca.Kh;
    LAUNCH(h, s, KC_CONV, k_conv<T><<<nblk(nk, 256), 256, 0, s>>>(ca));
    if (sizeof(T) == 4) {
        FFTCALL(h, s, cufftExecC2R(h->plan_b, (cufftComplex*)h->d_cgrid, (cufftReal*)h->d_grid));
    } else {
        FFTCALL(h, s, cufftExecZ2D(h->plan_b, (cufftDoubleComplex*)h->d_cgrid, (cufftDoubleReal*)h->d_grid));
    }
    GatherArgs<T> ga;
    ga.n = h->n;
    ga.pos = pos;
    ga.Qg = use_Qg ? (const T*)h->d_QgT : nullptr;
    ga.U = U;
    ga.q1 = nullptr;
    ga.lmax = lmax_eff(h);
    ga.g = g;
    ga.phi = (const T*)h->d_grid;
    ga.scale = 2.0 * DMFFB_DIELECTRIC;
    ga.grad = h->d_grad;
    ga.torque = (T*)h->d_torque;
    ga.field = field_out;
    ga.field_accumulate = field_acc;
    ga.gQ = (mode == GATHER_FULL) ? h->d_gQ : nullptr;
    ga.dq1 = nullptr;
    ga.scal = h->d_scal + S_GATHER;
    ga.want_box = 1;
    ga.mode = mode;
    if (mode == GATHER_FIELD && !field_acc && h->stencils_ready)
        LAUNCH(h, s, KC_GATHER_FIELD, k_gather_field_cached<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(
                                          h->n, stencil_cache<T>(h), g, (const T*)h->d_grid, 2.0 * DMFFB_DIELECTRIC, field_out,
                                          FieldCombine()));
    else if (mode == GATHER_FIELD && !field_acc)
        LAUNCH(h, s, KC_GATHER_FIELD, k_gather_field<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(
                                          h->n, pos, g, (const T*)h->d_grid, 2.0 * DMFFB_DIELECTRIC, field_out));
    else
        LAUNCH(h, s, (mode == GATHER_FULL ? KC_GATHER_FULL : KC_GATHER_FIELD), k_gather<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(ga));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// One CG step's direction update and matvec A p on the PME path with the stencil cache.  The
// step's r.z slot comes from the step counter in sc[7] (zero at the start of the solve), so a
// captured step runs right whatever the parity of the step it is replayed as: k_cg_p reads the
// counter (slot = count mod 2), forms p = z + beta p (beta from the previous step's r.z) and
// clears sc[5]; the real-space matvec forks onto the side stream, writes d_fmv and reduces p.fmv
// into sc[5], overlapping the whole reciprocal pass; the dipole spread clears sc[2] and sc[3]
// (rr) and advances the counter; the gather writes d_Ap = recip + diagonal p, reduces p.d_Ap into
// sc[2] and clears sc[1 - slot], the r.z slot this step's update writes.  A p = d_Ap + d_fmv; the
// caller joins the side stream (h->e_join) before the update reads them.
template <typename T>
int cg_matvec_fused(dmffb_engine* h, cudaStream_t s, const Box& bx, double* sc) {
    unsigned long long* ctr = (unsigned long long*)(sc + 7);
    const MeshGeom g = mesh_geom(bx, h->K);
    SpreadArgs<T> sa;
    sa.n = h->n;
    sa.pos = nullptr;
    sa.Qg = nullptr;
    sa.U = h->d_p;
    sa.q1 = nullptr;
    sa.lmax = 1;
    sa.g = g;
    sa.grid = (T*)h->d_grid2;
    sa.perm_mul = h->perm_mul;
    sa.zero_scal[0] = sc + 2;
    sa.zero_scal[1] = sc + 3;
    sa.ctr_inc = ctr;
    LAUNCH(h, s, KC_VEC, k_cg_p<<<nblk(3 * h->n, 256), 256, 0, s>>>(h->n, sc, 1, 0, h->d_z, h->d_p, sc + 5, ctr));
    const bool fork = h->s2 && !h->prof;
    {
        CsrArgs c;
        c.n = h->n;
        c.off = h->d_csr_off;
        c.ent = h->d_csr_ent;
        cudaStream_t sm = s;
        if (fork) {
            CK(cudaEventRecord(h->e_fork, s));
            CK(cudaStreamWaitEvent(h->s2, h->e_fork, 0));
            sm = h->s2;
        }
        LAUNCH(h, sm, KC_PAIR_MATVEC, k_matvec_apply<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, sm>>>(
                                          c, (const MvCoef<T>*)h->d_mvcoef, (const T*)h->d_posT, boxT<T>(bx), h->d_p, h->d_fmv,
                                          sc + 5));
        if (fork) CK(cudaEventRecord(h->e_join, h->s2));
    }
    LAUNCH(h, s, KC_SPREAD, k_spread_dip_cached<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(sa, stencil_cache<T>(h)));
    if (sizeof(T) == 4 && h->fc_enabled && h->fc_ok > 0) {
        // forward FFT, influence multiply and inverse FFT in one cluster; it also clears grid2
        int stc = fc_launch(h, s, (float*)h->d_grid2, (float*)h->d_grid);
        if (stc) return stc;
    } else {
    const int64_t K3 = (int64_t)h->K[0] * h->K[1] * h->K[2];
    CKFFT(cufftSetStream(h->plan_f, s));
    CKFFT(cufftSetStream(h->plan_b, s));
    if (sizeof(T) == 4)
        FFTCALL(h, s, cufftExecR2C(h->plan_f, (cufftReal*)h->d_grid2, (cufftComplex*)h->d_cgrid));
    else
        FFTCALL(h, s, cufftExecD2Z(h->plan_f, (cufftDoubleReal*)h->d_grid2, (cufftDoubleComplex*)h->d_cgrid));
    ConvArgs<T> ca;
    for (int k = 0; k < 3; ++k) ca.K[k] = h->K[k];
    ca.Kh = h->K[2] / 2 + 1;
    ca.S = (T*)h->d_cgrid;
    ca.bmod = h->d_bmod;
    for (int k = 0; k < 9; ++k) ca.hinv[k] = bx.hinv[k];
    ca.V = fabs(det3(bx.h));
    ca.kappa = h->kappa;
    ca.escale = DMFFB_DIELECTRIC;
    ca.kind = CK_COUL;
    ca.scal = h->d_scal + S_RECIP;
    ca.want_energy = 0;
    ca.zero_real = (T*)h->d_grid2;
    ca.nzero = K3;
    const int64_t nk = (int64_t)h->K[0] * h->K[1] * ca.Kh;
    LAUNCH(h, s, KC_CONV, k_conv<T><<<nblk(nk, 256), 256, 0, s>>>(ca));
    if (sizeof(T) == 4)
        FFTCALL(h, s, cufftExecC2R(h->plan_b, (cufftComplex*)h->d_cgrid, (cufftReal*)h->d_grid));
    else
        FFTCALL(h, s, cufftExecZ2D(h->plan_b, (cufftDoubleComplex*)h->d_cgrid, (cufftDoubleReal*)h->d_grid));
    }
    FieldCombine cmb;
    const double k = h->kappa;
    cmb.U = h->d_p;
    cmb.pol = h->d_pol;
    cmb.self1 = -2.0 * DMFFB_DIELECTRIC * (k / 1.7724538509055159) * 2.0 * k * k / 3.0;
    cmb.dot_out = sc + 2;
    cmb.zero_pair = sc;
    cmb.ctr = ctr;
    LAUNCH(h, s, KC_GATHER_FIELD, k_gather_field_cached<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(
                                      h->n, stencil_cache<T>(h), g, (const T*)h->d_grid, 2.0 * DMFFB_DIELECTRIC, h->d_Ap,
                                      cmb));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// pair tensors of every CSR entry for the solve at these positions
template <typename T>
int matvec_alloc(dmffb_engine* h) {
    int st;
    if (h->csr_cap > h->mv_cap) {
        if (h->d_mvcoef) cudaFree(h->d_mvcoef);
        h->mv_cap = h->csr_cap;
        if ((st = dalloc(h, &h->d_mvcoef, h->mv_cap * sizeof(MvCoef<T>)))) return st;
    }
    return DMFFB_OK;
}

// pair tensors of every CSR entry (the buffer is sized by matvec_alloc)
template <typename T>
int matvec_coef_launch(dmffb_engine* h, cudaStream_t s, const Box& bx, const int32_t* pairs, int64_t npairs) {
    PairArgs<T> a = pair_args<T>(h, bx, pairs, npairs, nullptr);
    CsrArgs c;
    c.n = h->n;
    c.off = h->d_csr_off;
    c.ent = h->d_csr_ent;
    LAUNCH(h, s, KC_MVCOEF, k_matvec_coef<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(
                                     a, c, (MvCoef<T>*)h->d_mvcoef));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// full both-direction CSR of the half-list rows (for the atomics-free CG matvec)
int build_csr(dmffb_engine* h, cudaStream_t s, const int32_t* pairs, int64_t npairs) {
    const int n = h->n;
    int st;
    if (h->csr_from_build && pairs == h->d_pairs) return DMFFB_OK;  // made by the neighbour build
    h->csr_from_build = false;
    if (!h->d_csr_off) {
        const int nc = h->n_cap;
        if ((st = dalloc(h, &h->d_csr_off, (nc + 1) * sizeof(int64_t)))) return st;
        if ((st = dalloc(h, &h->d_csr_deg, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_fmv, 3 * nc * sizeof(double)))) return st;
        size_t need = 0;
        cub::DeviceScan::InclusiveSum(nullptr, need, (int32_t*)nullptr, (int64_t*)nullptr, nc);
        h->cub2_bytes = need;
        if ((st = dalloc(h, &h->d_cub2, need))) return st;
    }
    if (2 * npairs > h->csr_cap) {
        if (h->d_csr_ent) cudaFree(h->d_csr_ent);
        h->csr_cap = 2 * npairs + 1024;
        if ((st = dalloc(h, &h->d_csr_ent, h->csr_cap * sizeof(int32_t)))) return st;
    }
    CK(cudaMemsetAsync(h->d_csr_deg, 0, n * sizeof(int32_t), s));
    if (npairs > 0)
        LAUNCH(h, s, KC_VEC, k_csr_count<<<nblk(npairs, 256), 256, 0, s>>>(npairs, pairs, n, h->d_csr_deg));
    CK(cudaMemsetAsync(h->d_csr_off, 0, sizeof(int64_t), s));
    size_t tb = h->cub2_bytes;
    LAUNCH(h, s, KC_VEC, cub::DeviceScan::InclusiveSum(h->d_cub2, tb, h->d_csr_deg, h->d_csr_off + 1, n, s));
    CK(cudaMemsetAsync(h->d_csr_deg, 0, n * sizeof(int32_t), s));
    if (npairs > 0)
        LAUNCH(h, s, KC_VEC, k_csr_fill<<<nblk(npairs, 256), 256, 0, s>>>(npairs, pairs, n, h->d_csr_off, h->d_csr_deg,
                                                                          h->d_csr_ent));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// dE/dU at U (include_perm) or its linear part A U (!include_perm), into out.  With dot_out,
// dot(dotv, out) is accumulated into *dot_out; zero_scal names three scalars set to 0 before
// the combine (by the first kernel of the reciprocal pass when there is one)
template <typename T>
int field_eval(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, const int32_t* pairs,
               int64_t npairs, const double* U, bool include_perm, double* out, const double* dotv = nullptr,
               double* dot_out = nullptr, double* const* zero_scal = nullptr, bool with_mvcoef = false) {
    const bool recip_on = h->lpme && h->have_plans;
    if (zero_scal && !recip_on)
        for (int k = 0; k < 3; ++k)
            if (zero_scal[k]) CK(cudaMemsetAsync(zero_scal[k], 0, sizeof(double), s));
    if (include_perm) CK(cudaMemsetAsync(h->d_fieldT, 0, (size_t)3 * h->n * sizeof(T), s));
    // the real-space work (permanent pair field, matvec) runs on a side stream, overlapping the
    // reciprocal pass; both write their own arrays and meet in the combine
    const bool real_work = (include_perm && npairs > 0) || U || with_mvcoef;
    const bool fork = real_work && h->s2 && !h->prof;
    cudaStream_t sr = s;
    if (fork) {
        CK(cudaEventRecord(h->e_fork, s));
        CK(cudaStreamWaitEvent(h->s2, h->e_fork, 0));
        sr = h->s2;
    }
    // the CG matvec's pair tensors, needed only after this pass: also beside the reciprocal pass
    if (with_mvcoef) {
        int stc = matvec_coef_launch<T>(h, sr, bx, pairs, npairs);
        if (stc) return stc;
    }
    if (include_perm && npairs > 0) {
        PairArgs<T> a = pair_args<T>(h, bx, pairs, npairs, nullptr);
        if (sizeof(T) == 4) {
            LAUNCH(h, sr, KC_PAIR_FIELD, k_admp_pair<T, true, PAIR_FIELD, ROWS_UNSCALED><<<nblk(npairs, 128), 128, 0, sr>>>(a));
            a.rowmap = h->d_srows;
            a.nrowmap = h->n_srows;
            if (h->n_srows > 0)
                LAUNCH(h, sr, KC_PAIR_FIELD_SCALED, k_admp_pair<T, true, PAIR_FIELD, ROWS_SCALED><<<nblk(h->n_srows, 128), 128, 0, sr>>>(a));
        } else {
            LAUNCH(h, sr, KC_PAIR_FIELD, k_admp_pair<T, true, PAIR_FIELD><<<nblk(npairs, 128), 128, 0, sr>>>(a));
        }
    }
    if (U) {
        CsrArgs c;
        c.n = h->n;
        c.off = h->d_csr_off;
        c.ent = h->d_csr_ent;
        cudaStream_t sm = sr;
        LAUNCH(h, sm, KC_PAIR_MATVEC, k_matvec_apply<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, sm>>>(
                                          c, (const MvCoef<T>*)h->d_mvcoef, (const T*)h->d_posT, boxT<T>(bx), U, h->d_fmv));
    }
    if (fork) CK(cudaEventRecord(h->e_join, h->s2));
    const double* recip = nullptr;
    if (recip_on) {
        int st = recip_pass<T>(h, s, pos, bx, include_perm, U, GATHER_FIELD, h->d_fr, 0, zero_scal);
        if (st) return st;
        recip = h->d_fr;
    }
    if (fork) CK(cudaStreamWaitEvent(s, h->e_join, 0));
    const double k = h->kappa;
    const double self1 = h->lpme ? -2.0 * DMFFB_DIELECTRIC * (k / 1.7724538509055159) * 2.0 * k * k / 3.0 : 0.0;
    LAUNCH(h, s, KC_VEC, k_field_combine<T><<<nblk(3 * h->n, 256), 256, 0, s>>>(
                             h->n, recip, include_perm ? (const T*)h->d_fieldT : nullptr, U ? h->d_fmv : nullptr, U,
                             h->d_Qg, h->d_pol, self1, include_perm ? 1 : 0, out, dotv, dot_out));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

// Solves A U = -b for the induced dipoles, b the permanent field (dE/dU at U = 0), A = d2E/dU2.
// With rhs (the second-order pass) it solves A U = -rhs from U = 0 by CG instead.
// layout of d_pcg: acc[4][4] doubles, barrier words {count, gen, status, pad}, CgStatus
constexpr size_t kPcgAcc = 0, kPcgBar = 16 * sizeof(double), kPcgOut = kPcgBar + 4 * sizeof(unsigned);
constexpr size_t kPcgPhase = kPcgOut + 32;  // CgStatus padded to 32 B, then 8 pass timers
constexpr size_t kPcgBytes = kPcgPhase + 8 * sizeof(unsigned long long);

// The CG iterations after k_cg_init (sc[0] = r.z, sc[3] = r.r, sc[4] = b.b on the device) in one
// cooperative launch of k_cg_solve; convergence is decided on the device and read back once.
int cg_persistent(dmffb_engine* h, cudaStream_t s, const Box& bx, double* U, const double* sc,
                  dmffb_admp_result* res) {
    int st;
    if (!h->d_pcg && (st = dalloc(h, (char**)&h->d_pcg, kPcgBytes))) return st;
    char* base = (char*)h->d_pcg;
    CK(cudaMemsetAsync(base, 0, kPcgBytes, s));
    CgSolveArgs a = {};
    a.n = h->n;
    a.x = U;
    a.r = h->d_r;
    a.z = h->d_z;
    a.p = h->d_p;
    a.Ap = h->d_Ap;
    a.fmv = h->d_fmv;
    a.pol = h->d_pol;
    a.csr.n = h->n;
    a.csr.off = h->d_csr_off;
    a.csr.ent = h->d_csr_ent;
    a.coef = (const MvCoef<float>*)h->d_mvcoef;
    a.pos4 = (const float*)h->d_posT;
    a.bxT = boxT<float>(bx);
    a.st = stencil_cache<float>(h);
    a.g = mesh_geom(bx, h->K);
    a.perm_mul = h->perm_mul;
    a.gscale = 2.0 * DMFFB_DIELECTRIC;
    const double k = h->kappa;
    a.self1 = -2.0 * DMFFB_DIELECTRIC * (k / 1.7724538509055159) * 2.0 * k * k / 3.0;
    a.fc = fc_args(h, (float*)h->d_grid2, (float*)h->d_grid);
    a.acc = (double*)(base + kPcgAcc);
    a.init = sc;
    a.tol = h->cg_tol;
    a.max_iter = h->max_iter;
    unsigned* bw = (unsigned*)(base + kPcgBar);
    a.bar.count = bw;
    a.bar.gen = bw + 1;
    a.bar.status = (int*)(bw + 2);
    a.bar.wait_ns = (long long)(h->pcg_wait_s * 1e9);
    a.bar.phantom = (unsigned)h->pcg_phantom;
    h->pcg_phantom = 0;
    a.out = (CgStatus*)(base + kPcgOut);
    a.phase_ns = h->prof ? (unsigned long long*)(base + kPcgPhase) : nullptr;
    // CTAs: enough warps for the matvec + spread pass (two warps per atom), the x-planes and the
    // spectrum column blocks, within what the device holds at once
    const int ncb = (h->K[1] * (h->K[2] / 2 + 1) + kFcCols - 1) / kFcCols;
    int grid = (int)((2 * (int64_t)h->n + kCgThreads / 32 - 1) / (kCgThreads / 32));
    grid = std::max(grid, std::max(h->K[0], ncb));
    grid = std::min(grid, h->pcg_max_blocks);
    void* args[] = {&a};
    LAUNCH(h, s, KC_CGSOLVE, CK(cudaLaunchCooperativeKernel((const void*)k_cg_solve, dim3(grid), dim3(kCgThreads),
                                                            args, cg_solve_smem(h->K), s)));
    static_assert(sizeof(CgStatus) <= 32, "status block of the persistent solve");
    CK(cudaMemcpyAsync(h->h_scal, a.out, a.phase_ns ? kPcgBytes - kPcgOut : sizeof(CgStatus),
                       cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CgStatus cs;
    memcpy(&cs, h->h_scal, sizeof(cs));
    if (a.phase_ns) {
        unsigned long long ph[8];
        memcpy(ph, (char*)h->h_scal + (kPcgPhase - kPcgOut), sizeof(ph));
        for (int k = 0; k < 8; ++k) h->pcg_phase_ms[k] += ph[k] * 1e-6;
    }
    const int n3 = 3 * h->n;
    res->n_iter = cs.iters;
    res->converged = cs.converged;
    res->residual_rms = sqrt(cs.rr / n3);
    if (cs.status == DMFFB_CG_TIMEOUT)
        return fail(h, DMFFB_TIMEOUT, "dipole solve: a grid barrier wait of the persistent CG kernel ran out");
    if (cs.status == DMFFB_CG_NONFINITE) return fail(h, DMFFB_NONFINITE, "non-finite residual in the dipole solve");
    return DMFFB_OK;
}

template <typename T>
int solve_dipoles(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, const int32_t* pairs,
                  int64_t npairs, double* U, dmffb_admp_result* res, const double* rhs = nullptr) {
    const int n = h->n;
    const unsigned nb3 = nblk(3 * n, 256);
    double* sc = h->d_scal + S_CG;
    int st;
    if ((st = build_csr(h, s, pairs, npairs))) return st;
    if ((st = matvec_alloc<T>(h))) return st;
    if (h->solver == DMFFB_SOLVER_REFERENCE && !rhs) {
        if ((st = matvec_coef_launch<T>(h, s, bx, pairs, npairs))) return st;
        int it = 0;
        bool conv = false;
        const int maxit = h->steps_pol > 0 ? h->steps_pol : h->max_iter;
        for (it = 0; it < maxit; ++it) {
            if ((st = field_eval<T>(h, s, pos, bx, pairs, npairs, U, true, h->d_b))) return st;
            if (h->steps_pol <= 0) {
                CK(cudaMemsetAsync(sc + 8, 0, sizeof(double), s));
                LAUNCH(h, s, KC_VEC, k_absmax<<<nb3, 256, 0, s>>>(n, h->d_b, h->d_pol, 0.001, (unsigned long long*)(sc + 8)));
                CK(cudaMemcpyAsync(h->h_scal, sc + 8, sizeof(double), cudaMemcpyDeviceToHost, s));
                CK(cudaStreamSynchronize(s));
                if (h->h_scal[0] < h->cg_tol) {
                    conv = true;
                    break;
                }
            }
            LAUNCH(h, s, KC_VEC, k_ref_step<<<nb3, 256, 0, s>>>(n, h->d_b, h->d_pol, U, nullptr));
        }
        if (h->steps_pol > 0) {
            conv = true;
            it = h->steps_pol;
        }
        res->n_iter = it;
        res->converged = conv ? 1 : 0;
        res->residual_rms = conv && h->steps_pol <= 0 ? h->h_scal[0] : -1.0;
        return DMFFB_OK;
    }
    // CG on A U = -b.  The dipole-only field passes keep d_grid2 zero between passes; clear it
    // here so that an earlier solve that stopped part-way leaves nothing behind
    // the stencil cache holds for these positions only: it is dropped when the solve returns
    struct StencilScope {
        dmffb_engine* h;
        ~StencilScope() { h->stencils_ready = false; }
    } stencil_scope{h};
    if (h->lpme && h->have_plans) {
        CK(cudaMemsetAsync(h->d_grid2, 0, (size_t)h->K[0] * h->K[1] * h->K[2] * sizeof(T), s));
        if ((st = stencil_prep<T>(h, s, pos, bx))) return st;
    }
    if (rhs) {
        if ((st = matvec_coef_launch<T>(h, s, bx, pairs, npairs))) return st;
        CK(cudaMemcpyAsync(h->d_b, rhs, (size_t)3 * n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    } else if ((st = field_eval<T>(h, s, pos, bx, pairs, npairs, nullptr, true, h->d_b, nullptr, nullptr, nullptr,
                                   true))) {
        return st;
    }
    // from U = 0 the residual is -b: no A U pass
    const bool u0 = h->zero_guess || h->u_zeroed || rhs;
    if (h->zero_guess || rhs) CK(cudaMemsetAsync(U, 0, (size_t)3 * n * sizeof(double), s));
    if (!u0 && (st = field_eval<T>(h, s, pos, bx, pairs, npairs, U, false, h->d_Ap))) return st;
    LAUNCH(h, s, KC_VEC, k_cg_init<<<nb3, 256, 0, s>>>(n, h->d_b, u0 ? nullptr : h->d_Ap, h->d_pol, h->d_r, h->d_z,
                                                     h->d_p));
    CK(cudaMemsetAsync(sc, 0, 8 * sizeof(double), s));
    LAUNCH(h, s, KC_VEC, k_dot2<<<nb3, 256, 0, s>>>(3 * n, h->d_r, h->d_z, h->d_r, h->d_r, sc + 0, sc + 3));
    LAUNCH(h, s, KC_VEC, k_dot2<<<nb3, 256, 0, s>>>(3 * n, h->d_b, h->d_b, nullptr, nullptr, sc + 4, nullptr));
    const bool fused = h->lpme && h->have_plans && h->stencils_ready;
    if (sizeof(T) == 4 && fused && pcg_wanted(h) && h->d_fcW && pcg_decide(h) > 0)
        return cg_persistent(h, s, bx, U, sc, res);
    int it = 0;
    bool conv = false;
    double rms = 0.0, rms_b = 0.0;
    // one CG iteration; slot = parity of the r.z scalar it reads
    auto iteration = [&](int slot) -> int {
        int st2;
        if (fused) {
            if ((st2 = cg_matvec_fused<T>(h, s, bx, sc))) return st2;
            if (h->s2 && !h->prof) CK(cudaStreamWaitEvent(s, h->e_join, 0));
            LAUNCH(h, s, KC_VEC, k_cg_update<<<nb3, 256, 0, s>>>(n, sc, 0, U, h->d_r, h->d_z, h->d_p, h->d_Ap,
                                                               h->d_pol, sc, sc + 3, h->d_fmv,
                                                               (const unsigned long long*)(sc + 7)));
            return DMFFB_OK;
        }
        // Ap = A p with p.Ap reduced into sc[2]; pAp, rr and the r.z slot this step writes are
        // cleared at the head of the pass (the previous step has read them by then)
        double* const zs[3] = {sc + 2, sc + 3, sc + (1 - slot)};
        if ((st2 = field_eval<T>(h, s, pos, bx, pairs, npairs, h->d_p, false, h->d_Ap, h->d_p, sc + 2, zs))) return st2;
        LAUNCH(h, s, KC_VEC, k_cg_update<<<nb3, 256, 0, s>>>(n, sc, slot, U, h->d_r, h->d_z, h->d_p, h->d_Ap,
                                                           h->d_pol, sc + (1 - slot), sc + 3));
        LAUNCH(h, s, KC_VEC, k_cg_p<<<nb3, 256, 0, s>>>(n, sc, slot, 1 - slot, h->d_z, h->d_p));
        return DMFFB_OK;
    };
    // two iterations (slot 0 then 1) are captured once into a CUDA graph and replayed; the graph
    // bakes in pointers and the box, so it is captured on the second solve in a row with the same
    // ones (a one-off solve, such as a serving request of a new size, runs its launches directly
    // and pays no capture and instantiation) and replayed while they stay the same.  The fused
    // step takes its parity from the device step counter, so a one-step graph is captured beside
    // it for a last segment of odd length.
    bool graphs = h->use_graphs && !h->prof;
    if (graphs) {
        std::vector<double> key = {(double)(uintptr_t)pos, (double)(uintptr_t)pairs, (double)npairs,
                                   (double)(uintptr_t)U, (double)(uintptr_t)h->d_csr_ent, (double)sizeof(T),
                                   (double)(uintptr_t)h->d_mvcoef, (double)(uintptr_t)h->d_csr_off,
                                   (double)(h->fc_enabled ? h->fc_ok : 0), (double)(uintptr_t)h->d_fcG,
                                   (double)fused};
        for (int k = 0; k < 9; ++k) key.push_back(bx.h[k]);
        const bool repeat = key == h->cg_seen_key;
        h->cg_seen_key = key;
        if ((!h->cg_exec || key != h->cg_key) && !repeat) graphs = false;
    }
    auto capture = [&](int steps, cudaGraphExec_t* exec, int64_t* launches, int64_t* ffts) -> int {
        if (*exec) { cudaGraphExecDestroy(*exec); *exec = nullptr; }
        cudaGraph_t g;
        const int64_t l0 = h->n_launch, f0 = h->n_fft;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        int st0 = iteration(0);
        if (!st0 && steps == 2) st0 = iteration(1);
        cudaError_t ce = cudaStreamEndCapture(s, &g);
        // captured launches run on replay: count them there
        *launches = h->n_launch - l0;
        *ffts = h->n_fft - f0;
        h->n_launch = l0;
        h->n_fft = f0;
        if (st0) return st0;
        if (ce != cudaSuccess) return fail(h, DMFFB_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(exec, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return fail(h, DMFFB_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ce));
        return DMFFB_OK;
    };
    if (graphs) {
        const std::vector<double>& key = h->cg_seen_key;
        if (!h->cg_exec || key != h->cg_key) {
            if ((st = capture(2, &h->cg_exec, &h->cg_graph_launches, &h->cg_graph_ffts))) return st;
            if (h->cg_exec1) { cudaGraphExecDestroy(h->cg_exec1); h->cg_exec1 = nullptr; }
            if (fused && (st = capture(1, &h->cg_exec1, &h->cg_graph1_launches, &h->cg_graph1_ffts))) return st;
            h->cg_key = key;
        }
    }
    // The host reads the residual every few steps (no per-step sync).  On the fused path, from the
    // second read on, the residual's decay over the last segment predicts the steps still needed:
    // a segment shorter than check_every then ends at the first step expected to converge.
    const int check_every = 4;
    double r_prev = -1.0;
    int it_prev = 0;
    auto run_steps = [&](int k) -> int {
        int st2;
        for (; k >= 2; k -= 2) {
            if (graphs) {
                CK(cudaGraphLaunch(h->cg_exec, s));
                h->n_launch += h->cg_graph_launches;
                h->n_fft += h->cg_graph_ffts;
            } else {
                if ((st2 = iteration(0))) return st2;
                if ((st2 = iteration(1))) return st2;
            }
        }
        if (k == 1) {
            if (graphs) {
                CK(cudaGraphLaunch(h->cg_exec1, s));
                h->n_launch += h->cg_graph1_launches;
                h->n_fft += h->cg_graph1_ffts;
            } else if ((st2 = iteration(0))) {
                return st2;
            }
        }
        return DMFFB_OK;
    };
    while (true) {
        CK(cudaMemcpyAsync(h->h_scal, sc + 3, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        rms = sqrt(h->h_scal[0] / (3.0 * n));
        if (it == 0) rms_b = sqrt(h->h_scal[1] / (3.0 * n));
        if (!std::isfinite(rms)) return fail(h, DMFFB_NONFINITE, "non-finite residual in the dipole solve");
        // relative criterion: RMS(dE/dU) below cg_tol times the RMS permanent field
        if (rms <= h->cg_tol * rms_b) {
            conv = true;
            break;
        }
        if (it >= h->max_iter) break;
        int k = check_every;
        if (fused && r_prev > 0.0 && rms < r_prev && it > it_prev) {
            const double rate = std::pow(rms / r_prev, 1.0 / (double)(it - it_prev));
            const double need = std::log(h->cg_tol * rms_b / rms) / std::log(rate);
            if (need > 0.0 && need < (double)check_every) k = std::max(1, (int)std::ceil(need));
        }
        r_prev = rms;
        it_prev = it;
        if ((st = run_steps(k))) return st;
        it += k;
    }
    res->n_iter = it;
    res->converged = conv ? 1 : 0;
    res->residual_rms = rms;
    return DMFFB_OK;
}

template <typename T>
int ensure_pairs(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx);

template <typename T>
int compute_impl(dmffb_engine* h, cudaStream_t s, const double* pos, const double* box, const int32_t* pairs,
                 int64_t npairs, double* U, double* forces, dmffb_admp_result* res) {
    if (!h->params_set) return fail(h, DMFFB_BAD_ARG, "dmffb_admp_set_params was not called");
    if (!pos || !box || !res) return fail(h, DMFFB_BAD_ARG, "null pos/box/result");
    if (h->lpol && !U) return fail(h, DMFFB_BAD_ARG, "polarizable system needs U_inout");
    Box bx;
    make_box(box, bx);
    h->last_box = bx;
    h->cur_pos = pos;
    memset(res, 0, sizeof(*res));
    const int n = h->n;
    int st;
    const bool own_list = !pairs;
    if (own_list && !h->have_pairs)
        if ((st = dmffb_admp_build_neighbors(h, (void*)s, pos, box))) return st;
    if (own_list && h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
    if (h->timing) CK(cudaEventRecord(h->ev[0], s));
    CK(cudaMemsetAsync(h->d_scal, 0, N_SCAL * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_gpair, 0, (size_t)3 * n * sizeof(T), s));
    CK(cudaMemsetAsync(h->d_torque, 0, (size_t)3 * n * sizeof(T), s));
    CK(cudaMemsetAsync(h->d_grad, 0, (size_t)3 * n * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_gQ, 0, (size_t)9 * n * sizeof(double), s));
    PrepArgs<T> pa;
    pa.f.n = n;
    pa.f.pos = pos;
    pa.f.axis_type = h->d_axis_type;
    pa.f.axis_idx = h->d_axis_idx;
    pa.f.box = bx;
    pa.Qloc = h->d_Qloc;
    pa.lmax = h->lmax;
    pa.posT = (T*)h->d_posT;
    pa.QgT = (T*)h->d_QgT;
    pa.Qg = h->d_Qg;
    LAUNCH(h, s, KC_PREP, k_prepare<T><<<nblk(n, 128), 128, 0, s>>>(pa));
    CK(cudaGetLastError());
    // the work above needs no pair list: it runs while a single-pass build's totals come back
    if (own_list) {
        if ((st = nb_finish(h))) return st;
        if (h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
        pairs = h->d_pairs;
        npairs = h->npairs;
    }
    res->n_pairs = npairs;
    h->last_pairs = pairs;
    h->last_npairs = npairs;
    h->last_U = U;
    h->have_last = true;
    if (sizeof(T) == 4 && npairs > 0)
        if ((st = scaled_rows(h, s, pairs, npairs))) return st;
    if (h->timing) CK(cudaEventRecord(h->ev[1], s));
    if (h->lpol && !h->fixed_U) {
        if ((st = solve_dipoles<T>(h, s, pos, bx, pairs, npairs, U, res))) return st;
    } else {
        res->converged = 1;
    }
    if (h->timing) CK(cudaEventRecord(h->ev[2], s));
    // the real-space FULL pass runs on the side stream beside the reciprocal FULL pass (both add
    // torques with atomics; the gradients, energies and virials they write are separate)
    const bool fork_full = npairs > 0 && h->lpme && h->have_plans && h->s2 && !h->prof && !h->timing;
    cudaStream_t sp = s;
    if (fork_full) {
        CK(cudaEventRecord(h->e_fork, s));
        CK(cudaStreamWaitEvent(h->s2, h->e_fork, 0));
        sp = h->s2;
    }
    if (npairs > 0) {
        PairArgs<T> a = pair_args<T>(h, bx, pairs, npairs, h->lpol ? U : nullptr);
        const unsigned nbk = nblk(npairs, 128);
        if (sizeof(T) == 4) {
            const unsigned nbs = nblk(h->n_srows, 128);
            if (h->lpol) {
                LAUNCH(h, sp, KC_PAIR_FULL, k_admp_pair<T, true, PAIR_FULL, ROWS_UNSCALED><<<nbk, 128, 0, sp>>>(a));
                a.rowmap = h->d_srows;
                a.nrowmap = h->n_srows;
                if (nbs) LAUNCH(h, sp, KC_PAIR_FULL_SCALED, k_admp_pair<T, true, PAIR_FULL, ROWS_SCALED><<<nbs, 128, 0, sp>>>(a));
            } else {
                LAUNCH(h, sp, KC_PAIR_FULL, k_admp_pair<T, false, PAIR_FULL, ROWS_UNSCALED><<<nbk, 128, 0, sp>>>(a));
                a.rowmap = h->d_srows;
                a.nrowmap = h->n_srows;
                if (nbs) LAUNCH(h, sp, KC_PAIR_FULL_SCALED, k_admp_pair<T, false, PAIR_FULL, ROWS_SCALED><<<nbs, 128, 0, sp>>>(a));
            }
        } else {
            if (h->lpol) LAUNCH(h, sp, KC_PAIR_FULL, k_admp_pair<T, true, PAIR_FULL><<<nbk, 128, 0, sp>>>(a));
            else LAUNCH(h, sp, KC_PAIR_FULL, k_admp_pair<T, false, PAIR_FULL><<<nbk, 128, 0, sp>>>(a));
        }
        CK(cudaGetLastError());
    }
    if (fork_full) CK(cudaEventRecord(h->e_join, h->s2));
    if (h->timing) CK(cudaEventRecord(h->ev[3], s));
    if (h->lpme && h->have_plans) {
        if ((st = recip_pass<T>(h, s, pos, bx, true, h->lpol ? U : nullptr, GATHER_FULL, nullptr, 0))) return st;
    }
    if (fork_full) CK(cudaStreamWaitEvent(s, h->e_join, 0));
    if (h->timing) CK(cudaEventRecord(h->ev[4], s));
    SelfArgs<T> sa;
    sa.f = pa.f;
    sa.Qg = h->d_Qg;
    sa.U = h->lpol ? U : nullptr;
    sa.pol = h->lpol ? h->d_pol : nullptr;
    sa.torque = (const T*)h->d_torque;
    sa.kappa = h->kappa;
    sa.lmax_eff = lmax_eff(h);
    sa.lpme = h->lpme;
    sa.want_box = 1;
    sa.grad = h->d_grad;
    sa.scal = h->d_scal + S_SELF;
    sa.tau_out = nullptr;
    if (h->lmax == 0) sa.f.axis_idx = nullptr;
    LAUNCH(h, s, KC_SELF, k_self_frames<T><<<nblk((int64_t)n * kSelfTasks, 128), 128, 0, s>>>(sa));
    if (forces) LAUNCH(h, s, KC_VEC, k_finalize_forces<T><<<nblk(3 * n, 256), 256, 0, s>>>(n, (const T*)h->d_gpair, h->d_grad, forces));
    CK(cudaGetLastError());
    h->have_pgrad = false;
    if (h->admp_pgrad) {  // parameter adjoints at the converged dipoles (E is stationary in U)
        CK(cudaMemsetAsync(h->d_dpa, 0, (size_t)n * sizeof(double), s));
        CK(cudaMemsetAsync(h->d_dth, 0, (size_t)n * sizeof(double), s));
        if (npairs > 0) {
            PgradArgs<T> g;
            g.p = pair_args<T>(h, bx, pairs, npairs, h->lpol ? U : nullptr);
            g.dQ = h->d_gQ;
            g.dpa = h->d_dpa;
            g.dth = h->d_dth;
            const unsigned nbk = nblk(npairs, 128);
            if (sizeof(T) == 4) {
                const unsigned nbs = nblk(h->n_srows, 128);
                if (h->lpol) {
                    LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, true, ROWS_UNSCALED><<<nbk, 128, 0, s>>>(g));
                    g.p.rowmap = h->d_srows;
                    g.p.nrowmap = h->n_srows;
                    if (nbs) LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, true, ROWS_SCALED><<<nbs, 128, 0, s>>>(g));
                } else {
                    LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, false, ROWS_UNSCALED><<<nbk, 128, 0, s>>>(g));
                    g.p.rowmap = h->d_srows;
                    g.p.nrowmap = h->n_srows;
                    if (nbs) LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, false, ROWS_SCALED><<<nbs, 128, 0, s>>>(g));
                }
            } else {
                if (h->lpol) LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, true><<<nbk, 128, 0, s>>>(g));
                else LAUNCH(h, s, KC_PGRAD, k_admp_pgrad<T, false><<<nbk, 128, 0, s>>>(g));
            }
        }
        LocalGradArgs la;
        la.f = pa.f;
        la.Qg = h->d_Qg;
        la.U = h->lpol ? U : nullptr;
        la.pol = h->lpol ? h->d_pol : nullptr;
        la.dpa = h->lpol ? h->d_dpa : nullptr;
        la.kappa = h->kappa;
        la.lmax = h->lmax;
        la.lmax_eff = lmax_eff(h);
        la.lpme = h->lpme;
        la.dQ = h->d_gQ;
        la.dQloc = h->d_dQloc;
        la.dpol = h->lpol ? h->d_dpol : nullptr;
        LAUNCH(h, s, KC_SELF, k_local_grad<<<nblk(n, 128), 128, 0, s>>>(la));
        CK(cudaGetLastError());
        h->have_pgrad = true;
    }
    if (h->timing) CK(cudaEventRecord(h->ev[5], s));
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, N_SCAL * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    prof_collect(h);
    const double* sc = h->h_scal;
    res->e_real = sc[S_EREAL];
    res->e_recip = sc[S_RECIP];
    res->e_self = sc[S_SELF];
    res->e_pol = sc[S_SELF + 1];
    res->energy = res->e_real + res->e_recip + res->e_self + res->e_pol;
    // box gradient: pair images + frame images + reciprocal (k-space and mesh-coordinate parts)
    double bg[9];
    for (int k = 0; k < 9; ++k) bg[k] = sc[S_EREAL + 1 + k] + sc[S_SELF + 2 + k];
    if (h->lpme && h->have_plans) {
        const double* hi = bx.hinv;  // h^-T[a][b] = hinv[b][a]
        const double E = sc[S_RECIP];
        const double* t = sc + S_RECIP + 1;
        const double Tkk[9] = {t[0], t[3], t[4], t[3], t[1], t[5], t[4], t[5], t[2]};
        const MeshGeom g = mesh_geom(bx, h->K);
        const double* X = sc + S_GATHER + 1;  // X_NA[j][c]
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                double v = -E * hi[3 * b + a];
                double s2 = 0.0;
                for (int k = 0; k < 3; ++k) s2 += hi[3 * k + a] * Tkk[3 * k + b];
                v -= 2.0 * s2;
                // -(h^-T X^T NA)[a][b] = -sum_{k,j} hinv[k][a] X[j][k] NA[j][b]
                double s3 = 0.0;
                for (int k = 0; k < 3; ++k)
                    for (int j = 0; j < 3; ++j) s3 += hi[3 * k + a] * X[3 * j + k] * g.NA[3 * j + b];
                v -= s3;
                bg[3 * a + b] += v;
            }
    }
    for (int k = 0; k < 9; ++k) res->box_grad[k] = bg[k];
    if (h->timing) {
        float ms;
        for (int k = 0; k < 5; ++k) {
            cudaEventElapsedTime(&ms, h->ev[k], h->ev[k + 1]);
            h->t_ms[k] = ms;
        }
        cudaEventElapsedTime(&ms, h->ev[0], h->ev[5]);
        h->t_ms[5] = ms;
    }
    if (!std::isfinite(res->energy)) return fail(h, DMFFB_NONFINITE, "non-finite energy");
    if (h->lpol && !res->converged) {
        h->err = "induced dipoles did not converge";
        return DMFFB_NOT_CONVERGED;
    }
    return DMFFB_OK;
}


// reciprocal pass of one point-charge-like channel (dispersion: c_k with the C_k influence
// function including k = 0), accumulating energy / k-space tensor / mesh box term into scal
template <typename T>
int recip_pass_channel(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, const T* q, int kind,
                       double escale, double* grad, double* dq, double* scal_conv, double* scal_gather) {
    const MeshGeom g = mesh_geom(bx, h->K);
    const int64_t K3 = (int64_t)h->K[0] * h->K[1] * h->K[2];
    CK(cudaMemsetAsync(h->d_grid, 0, K3 * sizeof(T), s));
    SpreadArgs<T> sa;
    sa.n = h->n;
    sa.pos = pos;
    sa.Qg = nullptr;
    sa.U = nullptr;
    sa.q1 = q;
    sa.lmax = 0;
    sa.g = g;
    sa.grid = (T*)h->d_grid;
    sa.perm_mul = h->perm_mul;
    LAUNCH(h, s, KC_SPREAD, k_spread<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(sa));
    CKFFT(cufftSetStream(h->plan_f, s));
    CKFFT(cufftSetStream(h->plan_b, s));
    if (sizeof(T) == 4) FFTCALL(h, s, cufftExecR2C(h->plan_f, (cufftReal*)h->d_grid, (cufftComplex*)h->d_cgrid));
    else FFTCALL(h, s, cufftExecD2Z(h->plan_f, (cufftDoubleReal*)h->d_grid, (cufftDoubleComplex*)h->d_cgrid));
    ConvArgs<T> ca;
    for (int k = 0; k < 3; ++k) ca.K[k] = h->K[k];
    ca.Kh = h->K[2] / 2 + 1;
    ca.S = (T*)h->d_cgrid;
    ca.bmod = h->d_bmod;
    for (int k = 0; k < 9; ++k) ca.hinv[k] = bx.hinv[k];
    ca.V = fabs(det3(bx.h));
    ca.kappa = h->kappa;
    ca.escale = escale;
    ca.kind = kind;
    ca.scal = scal_conv;
    ca.want_energy = 1;
    LAUNCH(h, s, KC_CONV, k_conv<T><<<nblk((int64_t)h->K[0] * h->K[1] * ca.Kh, 256), 256, 0, s>>>(ca));
    if (sizeof(T) == 4) FFTCALL(h, s, cufftExecC2R(h->plan_b, (cufftComplex*)h->d_cgrid, (cufftReal*)h->d_grid));
    else FFTCALL(h, s, cufftExecZ2D(h->plan_b, (cufftDoubleComplex*)h->d_cgrid, (cufftDoubleReal*)h->d_grid));
    GatherArgs<T> ga;
    ga.n = h->n;
    ga.pos = pos;
    ga.Qg = nullptr;
    ga.U = nullptr;
    ga.q1 = q;
    ga.lmax = 0;
    ga.g = g;
    ga.phi = (const T*)h->d_grid;
    ga.scale = 2.0 * escale;
    ga.grad = grad;
    ga.torque = nullptr;
    ga.field = nullptr;
    ga.field_accumulate = 0;
    ga.gQ = nullptr;
    ga.dq1 = dq;
    ga.scal = scal_gather;
    ga.want_box = 1;
    ga.mode = GATHER_FULL;
    LAUNCH(h, s, KC_GATHER_FULL, k_gather<T><<<nblk((int64_t)h->n * 32, 256), 256, 0, s>>>(ga));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

template <typename T>
__global__ void k_disp_finalize(int n, const T* glr, const T* gsr, const double* gd, double* flr, double* fsr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= 3 * n) return;
    if (flr) flr[k] = -((double)glr[k] + gd[k]);
    if (fsr) fsr[k] = gsr ? -(double)gsr[k] : 0.0;
}

// box gradient of the reciprocal part: -E h^-T - 2 h^-T Tkk - h^-T X^T NA
void recip_box_grad(const Box& bx, const int K[3], const double* conv, const double* X, double* out) {
    const double* hi = bx.hinv;
    const double E = conv[0];
    const double* t = conv + 1;
    const double Tkk[9] = {t[0], t[3], t[4], t[3], t[1], t[5], t[4], t[5], t[2]};
    const MeshGeom g = mesh_geom(bx, K);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double v = -E * hi[3 * b + a];
            double s2 = 0.0, s3 = 0.0;
            for (int k = 0; k < 3; ++k) s2 += hi[3 * k + a] * Tkk[3 * k + b];
            for (int k = 0; k < 3; ++k)
                for (int j = 0; j < 3; ++j) s3 += hi[3 * k + a] * X[3 * j + k] * g.NA[3 * j + b];
            out[3 * a + b] += v - 2.0 * s2 - s3;
        }
}

template <typename T>
int disp_compute_impl(dmffb_engine* h, cudaStream_t s, const double* pos, const double* box, const int32_t* pairs,
                      int64_t npairs, double* f_lr, double* f_sr, dmffb_disp_result* res) {
    if (!h->params_set) return fail(h, DMFFB_BAD_ARG, "dmffb_disp_set_params was not called");
    Box bx;
    make_box(box, bx);
    memset(res, 0, sizeof(*res));
    const int n = h->n;
    int st;
    if (!pairs) {
        if (!h->have_pairs)
            if ((st = dmffb_admp_build_neighbors(h, (void*)s, pos, box))) return st;
        if ((st = nb_finish(h))) return st;
        if (h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
        pairs = h->d_pairs;
        npairs = h->npairs;
    }
    res->n_pairs = npairs;
    CK(cudaMemsetAsync(h->d_scal, 0, N_SCAL * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_glr, 0, (size_t)3 * n * sizeof(T), s));
    CK(cudaMemsetAsync(h->d_gsr, 0, (size_t)3 * n * sizeof(T), s));
    CK(cudaMemsetAsync(h->d_grad, 0, (size_t)3 * n * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_dc, 0, (size_t)3 * n * sizeof(double), s));
    DispArgs<T> a;
    a.n = n;
    a.npairs = npairs;
    a.pairs = pairs;
    a.pos = pos;
    a.c = (const T*)h->d_c;
    a.a = (const T*)h->d_tta;
    a.b = (const T*)h->d_ttb;
    a.q = (const T*)h->d_ttq;
    for (int k = 0; k < 6; ++k) a.ms[k] = (T)h->ms[k];
    a.kappa = (T)h->kappa;
    a.pmax = h->pmax;
    a.boxd = bx;
    a.grad_lr = (T*)h->d_glr;
    a.grad_sr = (T*)h->d_gsr;
    a.scal = h->d_scal;  // [0] E_lr real [1] E_sr [2..10] box lr [11..19] box sr
    const bool pg = h->want_pgrad;
    a.dlr = pg ? h->d_dc : nullptr;
    a.dsr = (pg && h->tt) ? h->d_dsr : nullptr;
    if (pg && h->tt) CK(cudaMemsetAsync(h->d_dsr, 0, (size_t)4 * n * sizeof(double), s));
    if (npairs > 0) {
        const unsigned nbk = nblk(npairs, 128);
        if (sizeof(T) == 4) {
            if ((st = scaled_rows(h, s, pairs, npairs))) return st;
            const unsigned nbs = nblk(h->n_srows, 128);
            if (h->tt) {
                LAUNCH(h, s, KC_PAIR_FULL, k_disp_pair<T, 1, true><<<nbk, 128, 0, s>>>(a));
                a.rowmap = h->d_srows;
                a.nrowmap = h->n_srows;
                if (nbs) LAUNCH(h, s, KC_PAIR_FULL_SCALED, k_disp_pair<T, 2, true><<<nbs, 128, 0, s>>>(a));
            } else {
                LAUNCH(h, s, KC_PAIR_FULL, k_disp_pair<T, 1, false><<<nbk, 128, 0, s>>>(a));
                a.rowmap = h->d_srows;
                a.nrowmap = h->n_srows;
                if (nbs) LAUNCH(h, s, KC_PAIR_FULL_SCALED, k_disp_pair<T, 2, false><<<nbs, 128, 0, s>>>(a));
            }
        } else {
            if (h->tt) LAUNCH(h, s, KC_PAIR_FULL, k_disp_pair<T, 0, true><<<nbk, 128, 0, s>>>(a));
            else LAUNCH(h, s, KC_PAIR_FULL, k_disp_pair<T, 0, false><<<nbk, 128, 0, s>>>(a));
        }
        CK(cudaGetLastError());
    }
    const int npass = h->pmax >= 10 ? 3 : (h->pmax >= 8 ? 2 : 1);
    if (h->lpme && h->have_plans) {
        const int kinds[3] = {CK_DISP6, CK_DISP8, CK_DISP10};
        for (int k = 0; k < npass; ++k) {
            if ((st = recip_pass_channel<T>(h, s, pos, bx, (const T*)h->d_c + (size_t)k * n, kinds[k], 1.0, h->d_grad,
                                            h->d_dc + (size_t)k * n, h->d_scal + 24, h->d_scal + 32)))
                return st;
        }
    }
    if (pg && h->lpme)
        LAUNCH(h, s, KC_SELF, k_disp_self_dc<T><<<nblk(n, 256), 256, 0, s>>>(n, h->pmax, h->kappa, (const T*)h->d_c,
                                                                         h->d_dc));
    h->have_pgrad = pg;
    LAUNCH(h, s, KC_VEC, k_disp_finalize<T><<<nblk(3 * n, 256), 256, 0, s>>>(
                             n, (const T*)h->d_glr, h->tt ? (const T*)h->d_gsr : nullptr, h->d_grad, f_lr, f_sr));
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, N_SCAL * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    prof_collect(h);
    const double* sc = h->h_scal;
    res->e_real = sc[0];
    res->e_sr = sc[1];
    res->e_recip = (h->lpme && h->have_plans) ? sc[24] : 0.0;
    res->e_self = h->lpme ? h->e_self_disp : 0.0;
    res->energy = res->e_real + res->e_recip + res->e_self;
    for (int k = 0; k < 9; ++k) {
        res->box_grad[k] = sc[2 + k];
        res->box_grad_sr[k] = sc[11 + k];
    }
    if (h->lpme && h->have_plans) recip_box_grad(bx, h->K, sc + 24, sc + 33, res->box_grad);
    if (!std::isfinite(res->energy) || !std::isfinite(res->e_sr)) return fail(h, DMFFB_NONFINITE, "non-finite energy");
    return DMFFB_OK;
}

// dE/dq of the Ewald self term, -2 D kappa / sqrt(pi) q_i (pme.py:1183-1222 at lmax 0)
__global__ void k_self_dq(int n, const double* q, double c, double* dq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dq[i] += c * q[i];
}

// Half-width cell grid of the cell pass: at least 5 cells of width >= rc/2 per axis (the 5^3
// stencil then covers every pair within rc), at most 64 per axis.
bool half_cells(const dmffb_engine* h, const Box& bx, int nc[3]) {
    const double* m = bx.h;
    const double V = fabs(det3(m));
    for (int k = 0; k < 3; ++k) {
        const double* u = m + 3 * ((k + 1) % 3);
        const double* w = m + 3 * ((k + 2) % 3);
        const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        nc[k] = (int)floor(V / sqrt(cx * cx + cy * cy + cz * cz) / (0.5 * h->rc));
        if (nc[k] > 64) nc[k] = 64;
        if (nc[k] < 5) return false;
    }
    return true;
}

// Counting sort of the atoms into the cells nc (the binning of the list build): cell_start /
// cell_atoms, and the cell-ordered float4 positions of the cell pass.
int bin_cells(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, const int nc[3]) {
    const int n = h->n;
    int st;
    if (!h->d_pcount) {
        const int cap = h->n_cap;
        if ((st = dalloc(h, &h->d_pcount, cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_poff, (cap + 1) * sizeof(int64_t)))) return st;
        if ((st = dalloc(h, &h->d_atom_cell, cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_atoms, cap * sizeof(int32_t)))) return st;
    }
    const int ncell = nc[0] * nc[1] * nc[2];
    if (ncell + 1 > h->ncell_cap) {
        if (h->d_cell_count) { cudaFree(h->d_cell_count); cudaFree(h->d_cell_start); cudaFree(h->d_cell_cursor); }
        h->ncell_cap = ncell + 1;
        if ((st = dalloc(h, &h->d_cell_count, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_start, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_cursor, h->ncell_cap * sizeof(int32_t)))) return st;
    }
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, (int32_t*)nullptr, (int32_t*)nullptr, ncell + 1);
    if (need > h->cub_bytes) {
        if (h->d_cub) cudaFree(h->d_cub);
        h->cub_bytes = need;
        if ((st = dalloc(h, &h->d_cub, need))) return st;
    }
    CK(cudaMemsetAsync(h->d_cell_count, 0, (ncell + 1) * sizeof(int32_t), s));
    CK(cudaMemsetAsync(h->d_cell_cursor, 0, (ncell + 1) * sizeof(int32_t), s));
    LAUNCH(h, s, KC_NBLIST, k_cell_count<<<nblk(n, 256), 256, 0, s>>>(n, pos, bx, nc[0], nc[1], nc[2], h->d_atom_cell,
                                                                     h->d_cell_count));
    size_t tb = h->cub_bytes;
    LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::ExclusiveSum(h->d_cub, tb, h->d_cell_count, h->d_cell_start, ncell + 1, s));
    LAUNCH(h, s, KC_NBLIST, k_cell_fill<<<nblk(n, 256), 256, 0, s>>>(n, h->d_atom_cell, h->d_cell_start,
                                                                    h->d_cell_cursor, h->d_cell_atoms));
    if (!h->d_posc && (st = dalloc(h, &h->d_posc, (size_t)h->n_cap * sizeof(float4)))) return st;
    LAUNCH(h, s, KC_NBLIST, k_pos_cells<<<nblk(n, 256), 256, 0, s>>>(n, pos, h->d_cell_atoms, h->d_posc));
    CK(cudaGetLastError());
    return DMFFB_OK;
}

template <typename T>
int classical_compute_impl(dmffb_engine* h, cudaStream_t s, const double* pos, const double* box,
                           const int32_t* pairs, int64_t npairs, double* forces, dmffb_classical_result* res) {
    const bool nonbonded = h->coul != COUL_NONE || h->ntypes > 0;
    if (nonbonded && !h->params_set) return fail(h, DMFFB_BAD_ARG, "dmffb_classical_set_params was not called");
    Box bx;
    make_box(box, bx);
    memset(res, 0, sizeof(*res));
    const int n = h->n;
    int st;
    // the cell pass: every pair within rc straight from the cell grid of these positions
    int ncf[3] = {0, 0, 0};
    const bool cellpass = nonbonded && !pairs && h->cell_pass && h->pbc && !h->want_pgrad && half_cells(h, bx, ncf);
    if (nonbonded && !pairs && !cellpass) {
        if (!h->have_pairs)
            if ((st = dmffb_admp_build_neighbors(h, (void*)s, pos, box))) return st;
        if ((st = nb_finish(h))) return st;
        if (h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
        pairs = h->d_pairs;
        npairs = h->npairs;
    }
    if (!nonbonded) npairs = 0;
    res->n_pairs = npairs;
    const bool pg = h->want_pgrad;
    CK(cudaMemsetAsync(h->d_scal, 0, N_SCAL * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_glr, 0, (size_t)3 * n * sizeof(T), s));
    CK(cudaMemsetAsync(h->d_grad, 0, (size_t)3 * n * sizeof(double), s));
    if (pg) {
        CK(cudaMemsetAsync(h->d_dq, 0, (size_t)n * sizeof(double), s));
        if (h->ntypes > 0) {
            CK(cudaMemsetAsync(h->d_dsig, 0, (size_t)h->ntypes * h->ntypes * sizeof(double), s));
            CK(cudaMemsetAsync(h->d_deps, 0, (size_t)h->ntypes * h->ntypes * sizeof(double), s));
        }
    }
    if (cellpass) {
        if ((st = bin_cells(h, s, pos, bx, ncf))) return st;
        NbCellArgs<T> c;
        c.n = n;
        c.pos = pos;
        c.posc = h->d_posc;
        c.boxd = bx;
        c.rc = h->rc;
        for (int k = 0; k < 3; ++k) c.nc[k] = ncf[k];
        c.cell_start = h->d_cell_start;
        c.cov.cov_ptr = h->d_cov_ptr;
        c.cov.cov_j = h->d_cov_j;
        c.cov.cov_nb = h->d_cov_nb;
        c.cov_lo = h->d_cov_lo;
        c.cov_hi = h->d_cov_hi;
        c.qT = (const T*)h->d_qT;
        c.type = h->ntypes > 0 ? h->d_type : nullptr;
        c.ntypes = h->ntypes;
        c.sig_tt = (const T*)h->d_sigtt;
        c.eps_tt = (const T*)h->d_epstt;
        c.mc = (T)h->ms[5];
        c.ml = (T)h->mlj[5];
        c.kappa = (T)h->kappa;
        c.krf = (T)h->krf;
        c.crf = (T)h->crf;
        c.coul = h->coul;
        c.grad = (T*)h->d_glr;
        c.scal = h->d_scal;
        {
            const double* m = bx.h;
            const double V = fabs(det3(m));
            for (int k = 0; k < 3; ++k) {
                const double* u = m + 3 * ((k + 1) % 3);
                const double* w = m + 3 * ((k + 2) % 3);
                const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
                c.width[k] = V / sqrt(cx * cx + cy * cy + cz * cz);
            }
        }
        LAUNCH(h, s, KC_PAIR_FULL, k_nb_cells<T><<<nblk((int64_t)n * 32, 32 * kNbWarps), 32 * kNbWarps, 0, s>>>(c));
        CK(cudaGetLastError());
        // rows with a topological scale: the covalent rows within rc, FP64 for FP32 engines
        pairs = h->d_covrows;
        npairs = h->n_covrows;
    }
    if (npairs > 0) {
        NbPairArgs<T> a;
        a.n = n;
        a.npairs = npairs;
        a.pairs = pairs;
        a.pos = pos;
        a.q = h->d_q;
        a.qT = (const T*)h->d_qT;
        a.type = h->ntypes > 0 ? h->d_type : nullptr;
        a.ntypes = h->ntypes;
        a.sig_tt = (const T*)h->d_sigtt;
        a.eps_tt = (const T*)h->d_epstt;
        for (int k = 0; k < 6; ++k) {
            a.mc[k] = (T)h->ms[k];
            a.ml[k] = (T)h->mlj[k];
        }
        a.kappa = (T)h->kappa;
        a.krf = (T)h->krf;
        a.crf = (T)h->crf;
        a.coul = h->coul;
        a.pbc = h->pbc;
        a.boxd = bx;
        a.grad = (T*)h->d_glr;
        a.dq = (pg && h->coul != COUL_NONE) ? h->d_dq : nullptr;
        a.dsig = (pg && h->ntypes > 0) ? h->d_dsig : nullptr;
        a.deps = (pg && h->ntypes > 0) ? h->d_deps : nullptr;
        a.scal = h->d_scal;
        const unsigned nbk = nblk(npairs, 128);
        if (cellpass) {
            a.cut = h->rc;
            a.dq = a.dsig = a.deps = nullptr;
            LAUNCH(h, s, KC_PAIR_FULL_SCALED, k_nb_pair<T, 2><<<nbk, 128, 0, s>>>(a));
        } else if (sizeof(T) == 4) {
            if ((st = scaled_rows(h, s, pairs, npairs))) return st;
            LAUNCH(h, s, KC_PAIR_FULL, k_nb_pair<T, 1><<<nbk, 128, 0, s>>>(a));
            a.rowmap = h->d_srows;
            a.nrowmap = h->n_srows;
            if (h->n_srows > 0) LAUNCH(h, s, KC_PAIR_FULL_SCALED, k_nb_pair<T, 2><<<nblk(h->n_srows, 128), 128, 0, s>>>(a));
        } else {
            LAUNCH(h, s, KC_PAIR_FULL, k_nb_pair<T, 0><<<nbk, 128, 0, s>>>(a));
        }
        CK(cudaGetLastError());
    }
    const bool recip = h->coul == COUL_PME && h->lpme && h->have_plans;
    if (recip) {
        if ((st = recip_pass_channel<T>(h, s, pos, bx, (const T*)h->d_qT, CK_COUL, DMFFB_DIELECTRIC, h->d_grad,
                                        pg ? h->d_dq : nullptr, h->d_scal + 24, h->d_scal + 32)))
            return st;
        if (pg)
            LAUNCH(h, s, KC_SELF, k_self_dq<<<nblk(n, 256), 256, 0, s>>>(
                                      n, h->d_q, -2.0 * DMFFB_DIELECTRIC * h->kappa / sqrt(M_PI), h->d_dq));
    }
    for (int kind = 0; kind < 3; ++kind) {
        if (h->nterm[kind] <= 0) continue;
        BondedArgs b;
        b.nterm = (int)h->nterm[kind];
        b.idx = h->d_tidx[kind];
        b.prm = h->d_tprm[kind];
        b.pos = pos;
        b.grad = h->d_grad;
        b.dprm = pg ? h->d_tdprm[kind] : nullptr;
        b.scal = h->d_scal + 12 + kind;
        const unsigned nbk = nblk(h->nterm[kind], 128);
        if (kind == 0) LAUNCH(h, s, KC_BONDED, k_bonds<<<nbk, 128, 0, s>>>(b));
        else if (kind == 1) LAUNCH(h, s, KC_BONDED, k_angles<<<nbk, 128, 0, s>>>(b));
        else LAUNCH(h, s, KC_BONDED, k_torsions<<<nbk, 128, 0, s>>>(b));
        CK(cudaGetLastError());
    }
    if (forces)
        LAUNCH(h, s, KC_VEC, k_disp_finalize<T><<<nblk(3 * n, 256), 256, 0, s>>>(
                                 n, (const T*)h->d_glr, (const T*)nullptr, h->d_grad, forces, (double*)nullptr));
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, N_SCAL * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    prof_collect(h);
    const double* sc = h->h_scal;
    if (cellpass) res->n_pairs = (int64_t)llround(sc[11]);
    res->e_coul_real = sc[0];
    res->e_lj = sc[1];
    res->e_bond = sc[12];
    res->e_angle = sc[13];
    res->e_torsion = sc[14];
    res->e_coul_recip = recip ? sc[24] : 0.0;
    res->e_coul_self = (h->coul == COUL_PME && h->lpme) ? h->e_self_coul : 0.0;
    res->energy = res->e_coul_real + res->e_coul_recip + res->e_coul_self + res->e_lj + res->e_bond + res->e_angle +
                  res->e_torsion;
    for (int k = 0; k < 9; ++k) res->box_grad[k] = sc[2 + k];
    if (recip) recip_box_grad(bx, h->K, sc + 24, sc + 33, res->box_grad);
    if (!std::isfinite(res->energy)) return fail(h, DMFFB_NONFINITE, "non-finite energy");
    return DMFFB_OK;
}

template <typename T>
__global__ void k_to_t(int m, const double* src, T* dst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < m) dst[k] = (T)src[k];
}

// description -> scalar state (n, cut-off, Ewald, scales, solver, spread order)
void set_scalars(dmffb_engine* h, const dmffb_admp_desc* d) {
    h->n = d->n_atoms;
    h->rc = d->rc;
    h->kappa = d->lpme ? d->kappa : 0.0;
    for (int k = 0; k < 3; ++k) h->K[k] = d->lpme ? d->K[k] : 0;
    for (int k = 0; k < 6; ++k) {
        h->ms[k] = d->mscales[k];
        h->ps[k] = d->pscales[k];
        h->dsc[k] = d->dscales[k];
    }
    h->solver = d->solver;
    {  // a multiplier coprime with n near n / 148 (one stride per SM) for the spread order
        auto gcd = [](int64_t a, int64_t b) { while (b) { int64_t t = a % b; a = b; b = t; } return a; };
        int64_t m = std::max<int64_t>(1, d->n_atoms / 148) | 1;
        while (gcd(m, d->n_atoms) != 1) m += 2;
        h->perm_mul = (int)(m % std::max(1, d->n_atoms));
        if (h->perm_mul == 0) h->perm_mul = 1;
    }
    h->cg_tol = d->cg_tol > 0 ? d->cg_tol : 1e-6;
    h->max_iter = d->max_iter > 0 ? d->max_iter : 500;
    h->steps_pol = d->steps_pol;
}

// validate and upload local-axis data and the covalent map (CSR of j > i rows) of the description
int upload_topology(dmffb_engine* h, const dmffb_admp_desc* d) {
    const int n = d->n_atoms;
    std::vector<int32_t> at(n, DMFFB_NOAXISTYPE), ai(3 * n, -1);
    if (d->axis_types) for (int i = 0; i < n; ++i) at[i] = d->axis_types[i];
    if (d->axis_indices) for (int i = 0; i < 3 * n; ++i) ai[i] = d->axis_indices[i];
    for (int i = 0; i < n; ++i) {
        if (at[i] < 0 || at[i] > 5) return fail(h, DMFFB_BAD_ARG, "bad axis type");
        for (int k = 0; k < 3; ++k)
            if (ai[3 * i + k] >= n) return fail(h, DMFFB_BAD_ARG, "axis index out of range");
        // every axis atom the frame type reads must exist
        const int need = (at[i] == DMFFB_ZBISECT || at[i] == DMFFB_THREEFOLD) ? 3
                         : (at[i] == DMFFB_ZONLY ? 1 : (at[i] == DMFFB_NOAXISTYPE ? 0 : 2));
        if (d->lmax > 0)
            for (int k = 0; k < need; ++k)
                if (ai[3 * i + k] < 0) return fail(h, DMFFB_BAD_ARG, "missing axis atom");
    }
    std::vector<int32_t> cnt(n + 1, 0);
    for (int64_t r = 0; r < d->n_cov; ++r) {
        int i = d->cov_rows[3 * r], j = d->cov_rows[3 * r + 1];
        if (i < 0 || j < 0 || i >= n || j >= n || i == j) return fail(h, DMFFB_BAD_ARG, "bad covalent row");
        cnt[std::min(i, j) + 1]++;
    }
    for (int i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
    const int64_t nc = std::max<int64_t>(d->n_cov, 1);
    std::vector<int32_t> cj(nc), cn(nc), cur(cnt.begin(), cnt.end() - 1);
    // each atom's smallest and largest covalent partner index (lo > hi: none): the neighbour
    // build skips the map lookup for partners outside the range
    std::vector<int32_t> plo(n, n), phi(n, -1);
    for (int64_t r = 0; r < d->n_cov; ++r) {
        int i = d->cov_rows[3 * r], j = d->cov_rows[3 * r + 1];
        int lo = std::min(i, j), hi = std::max(i, j);
        int k = cur[lo]++;
        cj[k] = hi;
        cn[k] = d->cov_rows[3 * r + 2];
        plo[lo] = std::min(plo[lo], hi);
        phi[lo] = std::max(phi[lo], hi);
        plo[hi] = std::min(plo[hi], lo);
        phi[hi] = std::max(phi[hi], lo);
    }
    int st;
    if (nc > h->cov_cap) {
        if (h->d_cov_j) cudaFree(h->d_cov_j);
        if (h->d_cov_nb) cudaFree(h->d_cov_nb);
        h->d_cov_j = h->d_cov_nb = nullptr;
        h->cov_cap = nc;
        if ((st = dalloc(h, &h->d_cov_j, nc * sizeof(int32_t))) || (st = dalloc(h, &h->d_cov_nb, nc * sizeof(int32_t))))
            return st;
    }
    CK(cudaMemcpyAsync(h->d_axis_type, at.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_axis_idx, ai.data(), 3 * n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_cov_ptr, cnt.data(), (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_cov_j, cj.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_cov_nb, cn.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    if (!h->d_cov_lo) {
        if ((st = dalloc(h, &h->d_cov_lo, (size_t)h->n_cap * sizeof(int32_t))) ||
            (st = dalloc(h, &h->d_cov_hi, (size_t)h->n_cap * sizeof(int32_t))))
            return st;
    }
    CK(cudaMemcpyAsync(h->d_cov_lo, plo.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_cov_hi, phi.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaStreamSynchronize(h->s1));  // the host vectors go out of scope
    return DMFFB_OK;
}

// PME mesh of h->K: grids grown to fit, B-spline moduli, cuFFT plans (cached per mesh shape)
int setup_mesh(dmffb_engine* h) {
    h->fc_ok = -1;  // whether the engine's FFT convolution serves the mesh is decided again
    h->pcg_max_blocks = -1;
    const size_t ts = h->prec == DMFFB_FP32 ? 4 : 8;
    const int64_t K3 = (int64_t)h->K[0] * h->K[1] * h->K[2];
    const int64_t Kc = (int64_t)h->K[0] * h->K[1] * (h->K[2] / 2 + 1);
    int st;
    if (K3 > h->grid_cap) {
        if (h->d_grid) cudaFree(h->d_grid);
        h->d_grid = nullptr;
        if (h->d_grid2) cudaFree(h->d_grid2);
        h->d_grid2 = nullptr;
        h->grid_cap = K3;
        if ((st = dalloc(h, &h->d_grid, K3 * ts))) return st;
        if ((st = dalloc(h, &h->d_grid2, K3 * ts))) return st;
    }
    if (Kc > h->cgrid_cap) {
        if (h->d_cgrid) cudaFree(h->d_cgrid);
        h->d_cgrid = nullptr;
        h->cgrid_cap = Kc;
        if ((st = dalloc(h, &h->d_cgrid, 2 * Kc * ts))) return st;
    }
    const int ksum = h->K[0] + h->K[1] + h->K[2];
    if (ksum > h->bmod_cap) {
        if (h->d_bmod) cudaFree(h->d_bmod);
        h->d_bmod = nullptr;
        h->bmod_cap = ksum;
        if ((st = dalloc(h, &h->d_bmod, ksum * sizeof(double)))) return st;
    }
    // per-dimension B-spline moduli, recip.py:440-448: sum_{m=-2..2} M6(m+3) cos(2 pi m k / K)
    const double M6[5] = {1.0 / 120, 26.0 / 120, 66.0 / 120, 26.0 / 120, 1.0 / 120};
    std::vector<double> bm;
    for (int dd = 0; dd < 3; ++dd)
        for (int k = 0; k < h->K[dd]; ++k) {
            const int m = k < (h->K[dd] + 1) / 2 ? k : k - h->K[dd];
            double sm = 0;
            for (int q = -2; q <= 2; ++q) sm += M6[q + 2] * cos(2.0 * M_PI * q * m / h->K[dd]);
            bm.push_back(sm);
        }
    CK(cudaMemcpyAsync(h->d_bmod, bm.data(), bm.size() * sizeof(double), cudaMemcpyHostToDevice, h->s1));
    CK(cudaStreamSynchronize(h->s1));
    const std::array<int, 3> key = {h->K[0], h->K[1], h->K[2]};
    auto it = h->plan_cache.find(key);
    if (it == h->plan_cache.end()) {
        cufftHandle pf = 0, pb = 0;
        cufftType tf = h->prec == DMFFB_FP32 ? CUFFT_R2C : CUFFT_D2Z;
        cufftType tb = h->prec == DMFFB_FP32 ? CUFFT_C2R : CUFFT_Z2D;
        if (cufftPlan3d(&pf, h->K[0], h->K[1], h->K[2], tf) != CUFFT_SUCCESS)
            return fail(h, DMFFB_CUFFT_ERROR, "cufftPlan3d failed");
        if (cufftPlan3d(&pb, h->K[0], h->K[1], h->K[2], tb) != CUFFT_SUCCESS) {
            cufftDestroy(pf);
            return fail(h, DMFFB_CUFFT_ERROR, "cufftPlan3d failed");
        }
        it = h->plan_cache.emplace(key, std::make_pair(pf, pb)).first;
    }
    h->plan_f = it->second.first;
    h->plan_b = it->second.second;
    h->have_plans = true;
    return DMFFB_OK;
}

}  // namespace

// Completes a single-pass build: waits for its totals; if a count or a total outgrew its
// capacity, the list is rebuilt with the two passes (which resize the slots) from the positions
// the build was given, on its stream.
int nb_finish(dmffb_engine* h) {
    if (!h->nb_pending) return DMFFB_OK;
    h->nb_pending = false;
    CK(cudaEventSynchronize(h->e_nbtot));
    const int* md = (const int*)(h->h_nbtot + 2);
    if (md[0] <= h->ell_cap_h && (!h->nb_want_csr || md[1] <= h->ell_cap_f) && h->h_nbtot[0] <= h->pair_cap &&
        (!h->nb_want_csr || h->h_nbtot[1] <= h->csr_cap)) {
        h->npairs = h->h_nbtot[0];
        return DMFFB_OK;
    }
    h->have_pairs = false;
    h->ell_cap_h = h->ell_cap_f = 0;  // the two passes this time
    return dmffb_admp_build_neighbors(h, (void*)h->nb_stream, h->nb_pos, h->nb_box);
}

// Drops a single-pass build whose list will not be used (the engine is reconfigured, staged rows
// replace the list, or it is destroyed) once its copies to the host are done.
void nb_discard(dmffb_engine* h) {
    if (!h->nb_pending) return;
    cudaEventSynchronize(h->e_nbtot);
    h->nb_pending = false;
    h->have_pairs = false;
}

// ====================================================================== C ABI
extern "C" {

const char* dmffb_last_error(const dmffb_engine* h) { return h ? h->err.c_str() : "null handle"; }

int dmffb_admp_create(const dmffb_admp_desc* d, dmffb_engine** out) {
    if (!d || !out) return DMFFB_BAD_ARG;
    *out = nullptr;
    if (d->n_atoms <= 0 || d->lmax < 0 || d->lmax > 2 || (d->precision != DMFFB_FP32 && d->precision != DMFFB_FP64))
        return DMFFB_BAD_ARG;
    if (d->lpme && (d->K[0] <= 0 || d->K[1] <= 0 || d->K[2] <= 0 || !(d->kappa > 0))) return DMFFB_BAD_ARG;
    dmffb_engine* h = new dmffb_engine();
    *out = h;
    // streams and events first: every upload and zeroing below is ordered on the engine stream
    for (int k = 0; k < 8; ++k) cudaEventCreate(&h->ev[k]);
    cudaStreamCreateWithFlags(&h->s1, cudaStreamNonBlocking);
    cudaStreamCreateWithFlags(&h->s2, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&h->e_in, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&h->e_out, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&h->e_fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&h->e_join, cudaEventDisableTiming);
    h->lmax = d->lmax;
    h->lpol = d->lpol ? 1 : 0;
    h->lpme = d->lpme ? 1 : 0;
    h->prec = d->precision;
    h->n_cap = d->n_atoms;
    if (getenv("DMFFB_DISABLE_GRAPHS")) h->use_graphs = false;  // eager launches (debugging, tools)
    set_scalars(h, d);
    const int n = h->n_cap;
    const size_t ts = h->prec == DMFFB_FP32 ? 4 : 8;
    int st = 0;
#define AL(p, b)                                  \
    if ((st = dalloc(h, &(p), (b))) != DMFFB_OK) { \
        return st;                                \
    }
    AL(h->d_axis_type, n * sizeof(int32_t));
    AL(h->d_axis_idx, 3 * n * sizeof(int32_t));
    AL(h->d_cov_ptr, (n + 1) * sizeof(int32_t));
    if ((st = upload_topology(h, d))) return st;
    AL(h->d_Qloc, 9 * n * sizeof(double));
    AL(h->d_pol, n * sizeof(double));
    AL(h->d_thole, n * ts);
    AL(h->d_polsix, n * ts);
    AL(h->d_pos, 3 * n * sizeof(double));
    AL(h->d_U, 3 * n * sizeof(double));
    AL(h->d_forces, 3 * n * sizeof(double));
    AL(h->d_posT, 4 * n * ts);
    AL(h->d_Qg, 9 * n * sizeof(double));
    AL(h->d_QgT, 9 * n * ts);
    AL(h->d_gpair, 3 * n * ts);
    AL(h->d_torque, 3 * n * ts);
    AL(h->d_fieldT, 3 * n * ts);
    AL(h->d_grad, 3 * n * sizeof(double));
    AL(h->d_scal, N_SCAL * sizeof(double));
    AL(h->d_gQ, 9 * n * sizeof(double));
    if (h->lpol) {
        AL(h->d_b, 3 * n * sizeof(double));
        AL(h->d_r, 3 * n * sizeof(double));
        AL(h->d_z, 3 * n * sizeof(double));
        AL(h->d_p, 3 * n * sizeof(double));
        AL(h->d_Ap, 3 * n * sizeof(double));
        AL(h->d_fr, 3 * n * sizeof(double));
    }
#undef AL
    if (cudaMallocHost((void**)&h->h_scal, N_SCAL * sizeof(double)) != cudaSuccess)
        return fail(h, DMFFB_OOM, "cudaMallocHost failed");
    if (h->lpme && (st = setup_mesh(h))) return st;
    cudaError_t e = cudaStreamSynchronize(h->s1);
    if (e != cudaSuccess) return fail(h, DMFFB_CUDA_ERROR, cudaGetErrorString(e));
    return DMFFB_OK;
}

int dmffb_admp_reconfigure(dmffb_engine* h, const dmffb_admp_desc* d) {
    if (!h || !d) return DMFFB_BAD_ARG;
    if (h->kind != 0) return fail(h, DMFFB_BAD_ARG, "reconfigure applies to ADMP engines");
    if (d->n_atoms <= 0 || d->n_atoms > h->n_cap)
        return fail(h, DMFFB_SCRATCH_TOO_SMALL, "n_atoms exceeds the capacity the engine was created with");
    if (d->lmax != h->lmax || (d->lpol ? 1 : 0) != h->lpol || (d->lpme ? 1 : 0) != h->lpme || d->precision != h->prec)
        return fail(h, DMFFB_BAD_ARG, "lmax, lpol, lpme and precision are fixed at create");
    if (d->lpme && (d->K[0] <= 0 || d->K[1] <= 0 || d->K[2] <= 0 || !(d->kappa > 0)))
        return fail(h, DMFFB_BAD_ARG, "bad PME mesh or kappa");
    CK(cudaStreamSynchronize(h->s1));
    set_scalars(h, d);
    int st;
    if ((st = upload_topology(h, d))) return st;
    if (h->lpme && (st = setup_mesh(h))) return st;
    // everything derived from the previous system is stale
    nb_discard(h);
    h->have_pairs = false;
    h->npairs = 0;
    h->csr_from_build = false;
    h->csr_pairs = nullptr;
    if (h->cg_exec) {
        cudaGraphExecDestroy(h->cg_exec);
        h->cg_exec = nullptr;
    }
    if (h->cg_exec1) {
        cudaGraphExecDestroy(h->cg_exec1);
        h->cg_exec1 = nullptr;
    }
    h->cg_key.clear();
    h->cg_seen_key.clear();
    h->params_set = false;
    h->have_last = false;
    return DMFFB_OK;
}

void dmffb_destroy(dmffb_engine* h) {
    if (!h) return;
    nb_discard(h);
    if (h->h_nbtot) cudaFreeHost(h->h_nbtot);
    if (h->e_nbtot) cudaEventDestroy(h->e_nbtot);
    void* ptrs[] = {h->d_axis_type, h->d_axis_idx, h->d_cov_ptr, h->d_cov_j, h->d_cov_nb, h->d_Qloc, h->d_pol,
                    h->d_thole, h->d_polsix, h->d_pos, h->d_U, h->d_forces, h->d_posT, h->d_Qg, h->d_QgT,
                    h->d_gpair, h->d_torque, h->d_fieldT, h->d_grad, h->d_scal, h->d_b, h->d_r, h->d_z, h->d_p,
                    h->d_Ap, h->d_fr, h->d_gQ, h->d_fmv, h->d_posf, h->d_pcount_f, h->d_mvcoef, h->d_csr_off, h->d_csr_ent, h->d_csr_deg, h->d_cub2, h->d_grid, h->d_grid2, h->d_cgrid, h->d_bmod, h->d_pairs, h->d_atom_cell,
                    h->d_cell_count, h->d_cell_start, h->d_cell_cursor, h->d_cell_atoms, h->d_pcount, h->d_poff,
                    h->d_c, h->d_tta, h->d_ttb, h->d_ttq, h->d_glr, h->d_gsr, h->d_dc,
                    h->d_q, h->d_qT, h->d_type, h->d_sigtt, h->d_epstt, h->d_dq, h->d_dsig, h->d_deps,
                    h->d_tidx[0], h->d_tidx[1], h->d_tidx[2], h->d_tprm[0], h->d_tprm[1], h->d_tprm[2],
                    h->d_tdprm[0], h->d_tdprm[1], h->d_tdprm[2], h->d_dQloc, h->d_dpa, h->d_dth, h->d_dpol, h->d_dsr, h->d_srows, h->d_nsel, h->d_cubsel,
                    h->d_cub, h->d_ell_rows, h->d_ell_ent, h->d_maxdeg, h->d_stc_org, h->d_stc_w, h->d_nbmask, h->d_covrows, h->d_cov_lo, h->d_cov_hi, h->d_fcG, h->d_fcW, h->d_pcg, h->d_posc, h->d_srp, h->d_srdp, h->d_srgrad};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->h_nsel) cudaFreeHost(h->h_nsel);
    for (auto& kv : h->plan_cache) {
        cufftDestroy(kv.second.first);
        cufftDestroy(kv.second.second);
    }
    for (int k = 0; k < 8; ++k) cudaEventDestroy(h->ev[k]);
    for (auto e : h->ev_pool) cudaEventDestroy(e);
    if (h->cg_exec) cudaGraphExecDestroy(h->cg_exec);
    if (h->cg_exec1) cudaGraphExecDestroy(h->cg_exec1);
    if (h->s2) cudaStreamDestroy(h->s2);
    if (h->s1) cudaStreamDestroy(h->s1);
    if (h->e_in) cudaEventDestroy(h->e_in);
    if (h->e_out) cudaEventDestroy(h->e_out);
    if (h->e_fork) cudaEventDestroy(h->e_fork);
    if (h->e_build) cudaEventDestroy(h->e_build);
    if (h->e_join) cudaEventDestroy(h->e_join);
    if (h->d_bk) cudaFree(h->d_bk);
    delete h;
}

int dmffb_admp_set_params(dmffb_engine* h, const double* Q_local, const double* pol, const double* thole) {
    if (!h || !Q_local) return fail(h, DMFFB_BAD_ARG, "null handle or Q_local");
    if (h->lpol && (!pol || !thole)) return fail(h, DMFFB_BAD_ARG, "polarizable system needs pol and thole");
    const int n = h->n;
    // ordered on the engine stream (no device-wide synchronisation: other engines keep running)
    cudaStream_t s = h->s1;
    h->h_Qloc.assign(Q_local, Q_local + 9 * (size_t)n);
    if (pol) h->h_pol.assign(pol, pol + n);
    else h->h_pol.assign(n, 0.0);
    if (thole) h->h_thole.assign(thole, thole + n);
    else h->h_thole.assign(n, 0.0);
    CK(cudaMemcpyAsync(h->d_Qloc, Q_local, 9 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (pol) CK(cudaMemcpyAsync(h->d_pol, pol, n * sizeof(double), cudaMemcpyHostToDevice, s));
    else CK(cudaMemsetAsync(h->d_pol, 0, n * sizeof(double), s));
    double* dth = nullptr;
    if (thole) {  // staged in the gradient scratch, which compute() overwrites anyway
        dth = h->d_grad;
        CK(cudaMemcpyAsync(dth, thole, n * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    if (h->prec == DMFFB_FP32)
        k_set_thole<float><<<nblk(n, 128), 128, 0, s>>>(n, h->d_pol, dth, (float*)h->d_thole, (float*)h->d_polsix);
    else
        k_set_thole<double><<<nblk(n, 128), 128, 0, s>>>(n, h->d_pol, dth, (double*)h->d_thole, (double*)h->d_polsix);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    h->params_set = true;
    return DMFFB_OK;
}

int dmffb_admp_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                       int64_t npairs, double* U_inout, double* forces_out, dmffb_admp_result* result) {
    if (!h) return DMFFB_BAD_ARG;
    if (pairs && npairs < 0) return fail(h, DMFFB_BAD_ARG, "negative npairs");
    // the evaluation runs on the engine's own stream (capturable into CUDA graphs), ordered
    // after the caller's prior work on `stream` and before the caller's later work
    cudaStream_t caller = (cudaStream_t)stream;
    CK(cudaEventRecord(h->e_in, caller));
    CK(cudaStreamWaitEvent(h->s1, h->e_in, 0));
    int st = h->prec == DMFFB_FP32
                 ? compute_impl<float>(h, h->s1, pos, box, pairs, npairs, U_inout, forces_out, result)
                 : compute_impl<double>(h, h->s1, pos, box, pairs, npairs, U_inout, forces_out, result);
    cudaEventRecord(h->e_out, h->s1);
    cudaStreamWaitEvent(caller, h->e_out, 0);
    return st;
}

int dmffb_admp_compute_host(dmffb_engine* h, const double* pos, const double* box, const int32_t* pairs,
                            int64_t npairs, double* U_inout, double* forces_out, dmffb_admp_result* result) {
    if (!h || !pos) return fail(h, DMFFB_BAD_ARG, "null handle or positions");
    if (pairs && npairs < 0) return fail(h, DMFFB_BAD_ARG, "negative npairs");
    const int n = h->n;
    cudaStream_t s = h->s1;  // engine stream: host-buffer calls of different engines overlap on the GPU
    CK(cudaMemcpyAsync(h->d_pos, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    int32_t* dp = nullptr;
    if (pairs) {  // staged in the engine's pair buffer (grown when short)
        nb_discard(h);
        if (npairs > h->pair_cap) {
            CK(cudaStreamSynchronize(s));
            if (h->d_pairs) cudaFree(h->d_pairs);
            h->d_pairs = nullptr;
            h->pair_cap = npairs + 64;
            int sa = dalloc(h, &h->d_pairs, h->pair_cap * 3 * sizeof(int32_t));
            if (sa) return sa;
        }
        h->have_pairs = false;
        h->csr_from_build = false;
        h->pairs_gen++;
        dp = h->d_pairs;
        CK(cudaMemcpyAsync(dp, pairs, npairs * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    }
    if (h->lpol) {
        // with a zero initial guess the input dipoles are not read: no copy in
        if (U_inout && !h->zero_guess)
            CK(cudaMemcpyAsync(h->d_U, U_inout, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
        else CK(cudaMemsetAsync(h->d_U, 0, 3 * n * sizeof(double), s));
    }
    if (!pairs) {  // host callers hold no device pair list: rebuild for these positions
        int sb = dmffb_admp_build_neighbors(h, (void*)s, h->d_pos, box);
        if (sb) return sb;
    }
    h->u_zeroed = h->lpol && !U_inout;  // this call starts from U = 0
    int st = dmffb_admp_compute(h, s, h->d_pos, box, dp, npairs, h->lpol ? h->d_U : nullptr, h->d_forces, result);
    h->u_zeroed = false;
    if (dp) h->have_pairs = false;  // the staged rows are not the engine's own neighbour list
    if (st != DMFFB_OK && st != DMFFB_NOT_CONVERGED) return st;
    if (forces_out) CK(cudaMemcpyAsync(forces_out, h->d_forces, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (h->lpol && U_inout) CK(cudaMemcpyAsync(U_inout, h->d_U, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return st;
}

}  // extern "C"

// dE/dU at (pos, box, U) with the engine's current parameters: frames and global multipoles,
// the CSR and matvec tensors of these positions, then the field pass.
template <typename T>
int field_at(dmffb_engine* h, cudaStream_t s, const double* pos, const Box& bx, const int32_t* pairs, int64_t npairs,
             const double* U, double* field_out) {
    const int n = h->n;
    PrepArgs<T> pa;
    pa.f.n = n;
    pa.f.pos = pos;
    pa.f.axis_type = h->d_axis_type;
    pa.f.axis_idx = h->d_axis_idx;
    pa.f.box = bx;
    pa.Qloc = h->d_Qloc;
    pa.lmax = h->lmax;
    pa.posT = (T*)h->d_posT;
    pa.QgT = (T*)h->d_QgT;
    pa.Qg = h->d_Qg;
    h->cur_pos = pos;
    LAUNCH(h, s, KC_PREP, k_prepare<T><<<nblk(n, 128), 128, 0, s>>>(pa));
    int st;
    if (sizeof(T) == 4 && npairs > 0 && (st = scaled_rows(h, s, pairs, npairs))) return st;
    // the matvec of U needs this call's CSR and pair tensors (not a previous compute's)
    if ((st = build_csr(h, s, pairs, npairs))) return st;
    if ((st = matvec_alloc<T>(h))) return st;
    return field_eval<T>(h, s, pos, bx, pairs, npairs, U, true, field_out, nullptr, nullptr, nullptr, true);
}

__global__ void k_lin(int64_t m, double* out, const double* x0, double a, const double* d) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = x0[i] + (d ? a * d[i] : 0.0);
}

__global__ void k_cdiff(int64_t m, double* out, const double* p, const double* q, double scale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) out[i] = (p[i] - q[i]) * scale;
}

// Second-order pass at the point of the last compute (see dmffb_admp_backward in the header).
// With Phi(z) = E(z, U*(z)), z = (positions, box, Q_local, pol, thole) and U* the converged
// dipoles, the vector-Jacobian product of the first derivatives with a cotangent c is the
// Hessian-vector product H_Phi c (the Hessian is symmetric).  Implicit differentiation of
// dE/dU (z, U*(z)) = 0 gives dU*/dz c = dU with
//     A dU = -g,  A = d2E/dU2 (the dipole-solve matrix),  g = d2E/dU dz c,
// solved by the engine's CG (no unrolling of the solve), and then
//     H_Phi c = d2E/dz2 c + d2E/dz dU dU = d/de [dE/dz (z + e c, U* + e dU)] at e = 0.
// Both directional derivatives are central differences of the engine's analytic first
// derivatives (dE/dU, forces, box gradient, parameter adjoints) over a step e along c with the
// pair list fixed; dE/dU and dE/dz are polynomial in U (E is quadratic in U), so the U
// direction is exact and the truncation error, O(e^2), comes from the z direction alone.
template <typename T>
int admp_backward_impl(dmffb_engine* h, cudaStream_t s, const dmffb_admp_cotangent* c, dmffb_admp_second* out) {
    const int n = h->n;
    const int64_t n3 = 3 * (int64_t)n, n9 = 9 * (int64_t)n;
    int st;
    if ((int64_t)52 * n > h->bk_cap) {
        if (h->d_bk) cudaFree(h->d_bk);
        h->d_bk = nullptr;
        h->bk_cap = (int64_t)52 * n;
        if ((st = dalloc(h, &h->d_bk, (size_t)h->bk_cap * sizeof(double)))) return st;
    }
    double* b = h->d_bk;
    double *pos_s = b, *U_s = b + n3, *g = b + 2 * n3, *dU = b + 3 * n3, *Fp = b + 4 * n3, *Fm = b + 5 * n3;
    double* Q0 = b + 6 * n3;
    double *pol0 = Q0 + n9, *th0 = pol0 + n, *th_s = th0 + n, *Qp = th_s + n, *Qm = Qp + n9;
    double *pp = Qm + n9, *pm = pp + n, *tp = pm + n, *tm = tp + n;
    // the point of the last compute
    const double* pos0 = h->cur_pos;
    const Box bx0 = h->last_box;
    const int32_t* pairs = h->last_pairs;
    const int64_t npairs = h->last_npairs;
    double* U0 = h->last_U;
    // step: at most eps of each quantity's own scale along c (1 A for positions and box)
    std::vector<double> hc;
    auto maxabs_dev = [&](const double* d, int64_t m, double* out_max) -> int {
        *out_max = 0.0;
        if (!d) return DMFFB_OK;
        hc.resize(m);
        CK(cudaMemcpyAsync(hc.data(), d, m * sizeof(double), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (double v : hc) *out_max = std::max(*out_max, fabs(v));
        return DMFFB_OK;
    };
    auto maxabs_host = [](const std::vector<double>& v) {
        double m = 0.0;
        for (double x : v) m = std::max(m, fabs(x));
        return m;
    };
    double mpos, mQ, mpol, mth, mbox = 0.0;
    if ((st = maxabs_dev(c->pos, n3, &mpos)) || (st = maxabs_dev(c->Q_local, n9, &mQ)) ||
        (st = maxabs_dev(h->lpol ? c->pol : nullptr, n, &mpol)) || (st = maxabs_dev(h->lpol ? c->thole : nullptr, n, &mth)))
        return st;
    for (int k = 0; k < 9; ++k) mbox = std::max(mbox, fabs(c->box[k]));
    const double sQ = std::max(maxabs_host(h->h_Qloc), 1e-12);
    const double sp = std::max(maxabs_host(h->h_pol), 1e-12), sth = std::max(maxabs_host(h->h_thole), 1e-12);
    const double rate = std::max(std::max(std::max(mpos, mbox), std::max(mQ / sQ, mpol / sp)), mth / sth);
    out->n_iter = 0;
    out->residual_rms = 0.0;
    auto zero_out = [&]() -> int {
        if (out->pos) CK(cudaMemsetAsync(out->pos, 0, n3 * sizeof(double), s));
        if (out->Q_local) CK(cudaMemsetAsync(out->Q_local, 0, n9 * sizeof(double), s));
        if (out->pol) CK(cudaMemsetAsync(out->pol, 0, n * sizeof(double), s));
        if (out->thole) CK(cudaMemsetAsync(out->thole, 0, n * sizeof(double), s));
        for (int k = 0; k < 9; ++k) out->box[k] = 0.0;
        CK(cudaStreamSynchronize(s));
        return DMFFB_OK;
    };
    if (!(rate > 0.0)) {
        out->step = 0.0;
        return zero_out();
    }
    const double eps = sizeof(T) == 8 ? 1e-4 : 3e-3;
    const double e = eps / rate;
    out->step = e;
    // unperturbed parameters
    CK(cudaMemcpyAsync(Q0, h->d_Qloc, n9 * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(pol0, h->d_pol, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    CK(cudaMemcpyAsync(th0, h->h_thole.data(), n * sizeof(double), cudaMemcpyHostToDevice, s));
    // parameters and positions at z + a c (a = 0 restores the unperturbed parameters)
    double box_s[9];
    auto set_point = [&](double a) -> int {
        LAUNCH(h, s, KC_VEC, k_lin<<<nblk(n3, 256), 256, 0, s>>>(n3, pos_s, pos0, a, c->pos));
        for (int k = 0; k < 9; ++k) box_s[k] = bx0.h[k] + a * c->box[k];
        LAUNCH(h, s, KC_VEC, k_lin<<<nblk(n9, 256), 256, 0, s>>>(n9, h->d_Qloc, Q0, a, c->Q_local));
        if (h->lpol) {
            LAUNCH(h, s, KC_VEC, k_lin<<<nblk(n, 256), 256, 0, s>>>(n, h->d_pol, pol0, a, c->pol));
            LAUNCH(h, s, KC_VEC, k_lin<<<nblk(n, 256), 256, 0, s>>>(n, th_s, th0, a, c->thole));
            LAUNCH(h, s, KC_VEC, k_set_thole<T><<<nblk(n, 128), 128, 0, s>>>(n, h->d_pol, th_s, (T*)h->d_thole,
                                                                             (T*)h->d_polsix));
        }
        CK(cudaGetLastError());
        return DMFFB_OK;
    };
    const bool pg_was = h->admp_pgrad;
    const int solver_was = h->solver;
    double bgp[9], bgm[9];
    auto body = [&]() -> int {
        Box bxs;
        if (h->lpol) {
            // g = d2E/dU dz c: the field at fixed U* on both sides of z
            if ((st = set_point(e))) return st;
            make_box(box_s, bxs);
            if ((st = field_at<T>(h, s, pos_s, bxs, pairs, npairs, U0, Fp))) return st;
            if ((st = set_point(-e))) return st;
            make_box(box_s, bxs);
            if ((st = field_at<T>(h, s, pos_s, bxs, pairs, npairs, U0, Fm))) return st;
            LAUNCH(h, s, KC_VEC, k_cdiff<<<nblk(n3, 256), 256, 0, s>>>(n3, g, Fp, Fm, 0.5 / e));
            // tangent (adjoint) solve at z: A dU = -g, by CG from zero
            if ((st = set_point(0.0))) return st;
            PrepArgs<T> pa;
            pa.f.n = n;
            pa.f.pos = pos0;
            pa.f.axis_type = h->d_axis_type;
            pa.f.axis_idx = h->d_axis_idx;
            pa.f.box = bx0;
            pa.Qloc = h->d_Qloc;
            pa.lmax = h->lmax;
            pa.posT = (T*)h->d_posT;
            pa.QgT = (T*)h->d_QgT;
            pa.Qg = h->d_Qg;
            h->cur_pos = pos0;
            LAUNCH(h, s, KC_PREP, k_prepare<T><<<nblk(n, 128), 128, 0, s>>>(pa));
            if (sizeof(T) == 4 && npairs > 0 && (st = scaled_rows(h, s, pairs, npairs))) return st;
            h->solver = DMFFB_SOLVER_CG;
            dmffb_admp_result r2;
            memset(&r2, 0, sizeof(r2));
            if ((st = solve_dipoles<T>(h, s, pos0, bx0, pairs, npairs, dU, &r2, g))) return st;
            h->solver = solver_was;
            out->n_iter = r2.n_iter;
            out->residual_rms = r2.residual_rms;
        }
        // d/de of (dE/dpos, dE/dbox, dE/dparams) at (z + e c, U* + e dU)
        h->admp_pgrad = true;
        h->fixed_U = true;
        dmffb_admp_result rp, rm;
        for (int side = 0; side < 2; ++side) {
            const double a = side == 0 ? e : -e;
            if ((st = set_point(a))) return st;
            if (h->lpol) LAUNCH(h, s, KC_VEC, k_lin<<<nblk(n3, 256), 256, 0, s>>>(n3, U_s, U0, a, dU));
            dmffb_admp_result* r = side == 0 ? &rp : &rm;
            if ((st = compute_impl<T>(h, s, pos_s, box_s, pairs, npairs, h->lpol ? U_s : nullptr, side == 0 ? Fp : Fm, r)))
                return st;
            double* bg = side == 0 ? bgp : bgm;
            for (int k = 0; k < 9; ++k) bg[k] = r->box_grad[k];
            CK(cudaMemcpyAsync(side == 0 ? Qp : Qm, h->d_dQloc, n9 * sizeof(double), cudaMemcpyDeviceToDevice, s));
            if (h->lpol) {
                CK(cudaMemcpyAsync(side == 0 ? pp : pm, h->d_dpol, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
                CK(cudaMemcpyAsync(side == 0 ? tp : tm, h->d_dth, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
            }
        }
        const double inv = 0.5 / e;
        // forces are -dE/dpos
        if (out->pos) LAUNCH(h, s, KC_VEC, k_cdiff<<<nblk(n3, 256), 256, 0, s>>>(n3, out->pos, Fm, Fp, inv));
        if (out->Q_local) LAUNCH(h, s, KC_VEC, k_cdiff<<<nblk(n9, 256), 256, 0, s>>>(n9, out->Q_local, Qp, Qm, inv));
        if (out->pol) {
            if (h->lpol) LAUNCH(h, s, KC_VEC, k_cdiff<<<nblk(n, 256), 256, 0, s>>>(n, out->pol, pp, pm, inv));
            else CK(cudaMemsetAsync(out->pol, 0, n * sizeof(double), s));
        }
        if (out->thole) {
            if (h->lpol) LAUNCH(h, s, KC_VEC, k_cdiff<<<nblk(n, 256), 256, 0, s>>>(n, out->thole, tp, tm, inv));
            else CK(cudaMemsetAsync(out->thole, 0, n * sizeof(double), s));
        }
        for (int k = 0; k < 9; ++k) out->box[k] = (bgp[k] - bgm[k]) * inv;
        CK(cudaGetLastError());
        return DMFFB_OK;
    };
    st = body();
    // restore the engine: parameters, flags and the point of the last compute
    h->fixed_U = false;
    h->admp_pgrad = pg_was;
    h->solver = solver_was;
    h->have_pgrad = false;  // the last compute's parameter adjoints were overwritten
    int st2 = set_point(0.0);
    h->cur_pos = pos0;
    h->last_box = bx0;
    h->last_pairs = pairs;
    h->last_npairs = npairs;
    h->last_U = U0;
    h->have_last = true;
    if (cudaStreamSynchronize(s) != cudaSuccess && !st) st = fail(h, DMFFB_CUDA_ERROR, "second-order pass");
    return st ? st : st2;
}

extern "C" {

int dmffb_admp_backward(dmffb_engine* h, void* stream, const dmffb_admp_cotangent* c, dmffb_admp_second* out) {
    if (!h || h->kind != 0) return fail(h, DMFFB_BAD_ARG, "ADMP engine required");
    if (!c || !out) return fail(h, DMFFB_BAD_ARG, "null cotangent or output");
    if (!h->have_last || !h->cur_pos) return fail(h, DMFFB_BAD_ARG, "dmffb_admp_backward needs a preceding compute");
    int st;
    if (!h->d_dQloc) {  // allocate the adjoint buffers without switching them on for later computes
        const bool was = h->admp_pgrad;
        if ((st = dmffb_admp_set_param_grads(h, 1))) return st;
        h->admp_pgrad = was;
    }
    cudaStream_t caller = (cudaStream_t)stream;
    CK(cudaEventRecord(h->e_in, caller));
    CK(cudaStreamWaitEvent(h->s1, h->e_in, 0));
    st = h->prec == DMFFB_FP32 ? admp_backward_impl<float>(h, h->s1, c, out) : admp_backward_impl<double>(h, h->s1, c, out);
    cudaEventRecord(h->e_out, h->s1);
    cudaStreamWaitEvent(caller, h->e_out, 0);
    return st;
}

int dmffb_admp_field(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                     int64_t npairs, const double* U, double* field_out) {
    if (!h || !pos || !box || !field_out) return fail(h, DMFFB_BAD_ARG, "null argument");
    if (!h->lpol) return fail(h, DMFFB_BAD_ARG, "field requires a polarizable system");
    cudaStream_t s = (cudaStream_t)stream;
    Box bx;
    make_box(box, bx);
    h->cur_pos = pos;
    if (!pairs) {
        if (!h->have_pairs) {
            int st = dmffb_admp_build_neighbors(h, stream, pos, box);
            if (st) return st;
        }
        {
            int st = nb_finish(h);
            if (st) return st;
        }
        if (h->e_build) CK(cudaStreamWaitEvent((cudaStream_t)stream, h->e_build, 0));
        pairs = h->d_pairs;
        npairs = h->npairs;
    }
    const int n = h->n;
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        PrepArgs<T> pa;
        pa.f.n = n;
        pa.f.pos = pos;
        pa.f.axis_type = h->d_axis_type;
        pa.f.axis_idx = h->d_axis_idx;
        pa.f.box = bx;
        pa.Qloc = h->d_Qloc;
        pa.lmax = h->lmax;
        pa.posT = (T*)h->d_posT;
        pa.QgT = (T*)h->d_QgT;
        pa.Qg = h->d_Qg;
        LAUNCH(h, s, KC_PREP, k_prepare<T><<<nblk(n, 128), 128, 0, s>>>(pa));
        int st;
        if (sizeof(T) == 4 && npairs > 0 && (st = scaled_rows(h, s, pairs, npairs))) return st;
        // the matvec of U needs this call's CSR and pair tensors (not a previous compute's)
        if ((st = build_csr(h, s, pairs, npairs))) return st;
        if ((st = matvec_alloc<T>(h))) return st;
        st = field_eval<T>(h, s, pos, bx, pairs, npairs, U, true, field_out, nullptr, nullptr, nullptr, true);
        if (st) return st;
        CK(cudaStreamSynchronize(s));
        return DMFFB_OK;
    };
    if (h->prec == DMFFB_FP32) return run(float(0));
    return run(double(0));
}

int dmffb_admp_set_zero_guess(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 0) return fail(h, DMFFB_BAD_ARG, "ADMP engine required");
    h->zero_guess = enabled != 0;
    return DMFFB_OK;
}

int dmffb_admp_set_param_grads(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 0) return fail(h, DMFFB_BAD_ARG, "ADMP engine required");
    if (enabled && !h->d_dQloc) {
        const int nc = h->n_cap;
        int st;
        if ((st = dalloc(h, &h->d_dQloc, 9 * (size_t)nc * sizeof(double))) ||
            (st = dalloc(h, &h->d_dpa, (size_t)nc * sizeof(double))) ||
            (st = dalloc(h, &h->d_dth, (size_t)nc * sizeof(double))) ||
            (st = dalloc(h, &h->d_dpol, (size_t)nc * sizeof(double))))
            return st;
    }
    h->admp_pgrad = enabled != 0;
    return DMFFB_OK;
}

int dmffb_admp_multipole_grads(dmffb_engine* h, void* stream, double* dE_dQglobal, double* dE_dQlocal) {
    return dmffb_admp_param_grads(h, stream, dE_dQglobal, dE_dQlocal, nullptr, nullptr);
}

int dmffb_admp_param_grads(dmffb_engine* h, void* stream, double* dE_dQglobal, double* dE_dQlocal, double* dE_dpol,
                           double* dE_dthole) {
    if (!h || h->kind != 0) return fail(h, DMFFB_BAD_ARG, "ADMP engine required");
    if (!h->have_pgrad) return fail(h, DMFFB_BAD_ARG, "enable dmffb_admp_set_param_grads before compute");
    cudaStream_t cs = (cudaStream_t)stream;
    const size_t n = h->n;
    if (dE_dQglobal) CK(cudaMemcpyAsync(dE_dQglobal, h->d_gQ, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (dE_dQlocal) CK(cudaMemcpyAsync(dE_dQlocal, h->d_dQloc, 9 * n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (dE_dpol) {
        if (h->lpol) CK(cudaMemcpyAsync(dE_dpol, h->d_dpol, n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
        else CK(cudaMemsetAsync(dE_dpol, 0, n * sizeof(double), cs));
    }
    if (dE_dthole) {
        if (h->lpol) CK(cudaMemcpyAsync(dE_dthole, h->d_dth, n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
        else CK(cudaMemsetAsync(dE_dthole, 0, n * sizeof(double), cs));
    }
    return DMFFB_OK;
}

int dmffb_admp_param_grads_host(dmffb_engine* h, double* dE_dQlocal, double* dE_dpol, double* dE_dthole) {
    if (!h || h->kind != 0) return fail(h, DMFFB_BAD_ARG, "ADMP engine required");
    if (!h->have_pgrad) return fail(h, DMFFB_BAD_ARG, "enable dmffb_admp_set_param_grads before compute");
    cudaStream_t s = h->s1;
    const size_t n = h->n;
    if (dE_dQlocal) CK(cudaMemcpyAsync(dE_dQlocal, h->d_dQloc, 9 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (dE_dpol) {
        if (h->lpol) CK(cudaMemcpyAsync(dE_dpol, h->d_dpol, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        else memset(dE_dpol, 0, n * sizeof(double));
    }
    if (dE_dthole) {
        if (h->lpol) CK(cudaMemcpyAsync(dE_dthole, h->d_dth, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        else memset(dE_dthole, 0, n * sizeof(double));
    }
    CK(cudaStreamSynchronize(s));
    return DMFFB_OK;
}

int dmffb_build_neighbors(dmffb_engine* h, void* stream, const double* pos, const double* box, double rc,
                          int32_t* pairs_out, int64_t capacity, int64_t* npairs_out) {
    if (!h || !pos || !box || !npairs_out) return fail(h, DMFFB_BAD_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const int n = h->n;
    Box bx;
    make_box(box, bx);
    // cells per axis from the perpendicular widths V / |a_i x a_j|
    const double* m = bx.h;
    const double V = fabs(det3(m));
    int nc[3];
    bool cells = true;
    for (int k = 0; k < 3; ++k) {
        const double* u = m + 3 * ((k + 1) % 3);
        const double* w = m + 3 * ((k + 2) % 3);
        const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        const double width = V / sqrt(cx * cx + cy * cy + cz * cz);
        nc[k] = (int)floor(width / rc);
        if (nc[k] > 64) nc[k] = 64;
        if (nc[k] < 3) cells = false;
    }
    int st;
    if (!h->d_pcount) {
        const int nc = h->n_cap;
        if ((st = dalloc(h, &h->d_pcount, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_poff, (nc + 1) * sizeof(int64_t)))) return st;
        if ((st = dalloc(h, &h->d_atom_cell, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_atoms, nc * sizeof(int32_t)))) return st;
    }
    const int ncell = cells ? nc[0] * nc[1] * nc[2] : 1;
    if (ncell + 1 > h->ncell_cap) {
        if (h->d_cell_count) { cudaFree(h->d_cell_count); cudaFree(h->d_cell_start); cudaFree(h->d_cell_cursor); }
        h->ncell_cap = ncell + 1;
        if ((st = dalloc(h, &h->d_cell_count, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_start, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_cursor, h->ncell_cap * sizeof(int32_t)))) return st;
    }
    // scan workspace
    size_t need = 0, need2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, (int32_t*)nullptr, (int32_t*)nullptr, ncell + 1);
    cub::DeviceScan::InclusiveSum(nullptr, need2, (int32_t*)nullptr, (int64_t*)nullptr, n);
    need = std::max(need, need2);
    if (need > h->cub_bytes) {
        if (h->d_cub) cudaFree(h->d_cub);
        h->cub_bytes = need;
        if ((st = dalloc(h, &h->d_cub, need))) return st;
    }
    NbArgs a;
    a.n = n;
    a.pos = pos;
    a.box = bx;
    a.rc = rc;
    for (int k = 0; k < 3; ++k) a.nc[k] = cells ? nc[k] : 1;
    a.cov_ptr = h->d_cov_ptr;
    a.cov_j = h->d_cov_j;
    a.cov_nb = h->d_cov_nb;
    a.count = h->d_pcount;
    a.offset = h->d_poff;
    a.pairs = pairs_out;
    a.cap = capacity;
    if (cells) {
        CK(cudaMemsetAsync(h->d_cell_count, 0, (ncell + 1) * sizeof(int32_t), s));
        CK(cudaMemsetAsync(h->d_cell_cursor, 0, (ncell + 1) * sizeof(int32_t), s));
        LAUNCH(h, s, KC_NBLIST, k_cell_count<<<nblk(n, 256), 256, 0, s>>>(n, pos, bx, nc[0], nc[1], nc[2], h->d_atom_cell, h->d_cell_count));
        size_t tb = h->cub_bytes;
        LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::ExclusiveSum(h->d_cub, tb, h->d_cell_count, h->d_cell_start, ncell + 1, s));
        LAUNCH(h, s, KC_NBLIST, k_cell_fill<<<nblk(n, 256), 256, 0, s>>>(n, h->d_atom_cell, h->d_cell_start, h->d_cell_cursor, h->d_cell_atoms));
        a.cell_start = h->d_cell_start;
        a.cell_atoms = h->d_cell_atoms;
        LAUNCH(h, s, KC_NBLIST, k_pairs_warp<0><<<nblk((int64_t)n * 32, 256), 256, 0, s>>>(a));
    } else {
        LAUNCH(h, s, KC_NBLIST, k_pairs_all<0><<<nblk(n, 128), 128, 0, s>>>(a));
    }
    {
        size_t tb = h->cub_bytes;
        CK(cudaMemsetAsync(h->d_poff, 0, sizeof(int64_t), s));
        LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::InclusiveSum(h->d_cub, tb, h->d_pcount, h->d_poff + 1, n, s));
    }
    int64_t total = 0;
    CK(cudaMemcpyAsync(&total, h->d_poff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *npairs_out = total;
    if (total > capacity || !pairs_out) {
        h->err = "neighbour capacity too small";
        return DMFFB_NEIGHBOR_OVERFLOW;
    }
    if (cells) LAUNCH(h, s, KC_NBLIST, k_pairs_warp<1><<<nblk((int64_t)n * 32, 256), 256, 0, s>>>(a));
    else LAUNCH(h, s, KC_NBLIST, k_pairs_all<1><<<nblk(n, 128), 128, 0, s>>>(a));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    prof_collect(h);
    return DMFFB_OK;
}

int dmffb_admp_build_neighbors(dmffb_engine* h, void* stream, const double* pos, const double* box) {
    if (!h || !pos || !box) return DMFFB_BAD_ARG;
    if (h->nb_pending) nb_discard(h);  // this build replaces it
    cudaStream_t s = (cudaStream_t)stream;
    const int n = h->n;
    Box bx;
    make_box(box, bx);
    const double* m = bx.h;
    const double V = fabs(det3(m));
    int nc[3], nc2[3];
    bool cells = true, fine = true;  // fine: half-width cells with the 5^3 stencil
    for (int k = 0; k < 3; ++k) {
        const double* u = m + 3 * ((k + 1) % 3);
        const double* w = m + 3 * ((k + 2) % 3);
        const double cx = u[1] * w[2] - u[2] * w[1], cy = u[2] * w[0] - u[0] * w[2], cz = u[0] * w[1] - u[1] * w[0];
        const double width = V / sqrt(cx * cx + cy * cy + cz * cz);
        nc[k] = (int)floor(width / h->rc);
        if (nc[k] > 64) nc[k] = 64;
        if (nc[k] < 3) cells = false;
        nc2[k] = (int)floor(width / (0.5 * h->rc));
        if (nc2[k] > 64) nc2[k] = 64;
        if (nc2[k] < 5) fine = false;
    }
    if (fine && cells)
        for (int k = 0; k < 3; ++k) nc[k] = nc2[k];
    if (!cells) {  // small boxes: the generic builder, CSR later from the rows
        int64_t need = 0;
        int st = dmffb_build_neighbors(h, stream, pos, box, h->rc, h->d_pairs, h->pair_cap, &need);
        if (st == DMFFB_NEIGHBOR_OVERFLOW) {
            if (h->d_pairs) cudaFree(h->d_pairs);
            h->pair_cap = (int64_t)(need * 1.3) + 64;
            if ((st = dalloc(h, &h->d_pairs, h->pair_cap * 3 * sizeof(int32_t)))) return st;
            st = dmffb_build_neighbors(h, stream, pos, box, h->rc, h->d_pairs, h->pair_cap, &need);
        }
        if (st) return st;
        h->npairs = need;
        h->have_pairs = true;
        h->pairs_gen++;
        h->csr_from_build = false;
        return DMFFB_OK;
    }
    int st;
    if (!h->d_pcount) {
        const int nc = h->n_cap;
        if ((st = dalloc(h, &h->d_pcount, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_poff, (nc + 1) * sizeof(int64_t)))) return st;
        if ((st = dalloc(h, &h->d_atom_cell, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_atoms, nc * sizeof(int32_t)))) return st;
    }
    if (!h->d_posf) {
        if ((st = dalloc(h, &h->d_posf, 4 * h->n_cap * sizeof(float)))) return st;
        if ((st = dalloc(h, &h->d_pcount_f, h->n_cap * sizeof(int32_t)))) return st;
    }
    if (!h->d_csr_off) {
        const int nc = h->n_cap;
        if ((st = dalloc(h, &h->d_csr_off, (nc + 1) * sizeof(int64_t)))) return st;
        if ((st = dalloc(h, &h->d_csr_deg, nc * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_fmv, 3 * nc * sizeof(double)))) return st;
        size_t need = 0;
        cub::DeviceScan::InclusiveSum(nullptr, need, (int32_t*)nullptr, (int64_t*)nullptr, nc);
        h->cub2_bytes = need;
        if ((st = dalloc(h, &h->d_cub2, need))) return st;
    }
    const int ncell = nc[0] * nc[1] * nc[2];
    if (ncell + 1 > h->ncell_cap) {
        if (h->d_cell_count) { cudaFree(h->d_cell_count); cudaFree(h->d_cell_start); cudaFree(h->d_cell_cursor); }
        h->ncell_cap = ncell + 1;
        if ((st = dalloc(h, &h->d_cell_count, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_start, h->ncell_cap * sizeof(int32_t)))) return st;
        if ((st = dalloc(h, &h->d_cell_cursor, h->ncell_cap * sizeof(int32_t)))) return st;
    }
    size_t need = 0, need2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, (int32_t*)nullptr, (int32_t*)nullptr, ncell + 1);
    cub::DeviceScan::InclusiveSum(nullptr, need2, (int32_t*)nullptr, (int64_t*)nullptr, n);
    need = std::max(need, need2);
    if (need > h->cub_bytes) {
        if (h->d_cub) cudaFree(h->d_cub);
        h->cub_bytes = need;
        if ((st = dalloc(h, &h->d_cub, need))) return st;
    }
    LAUNCH(h, s, KC_NBLIST, k_pos_f32<<<nblk(n, 256), 256, 0, s>>>(n, pos, h->d_posf));
    CK(cudaMemsetAsync(h->d_cell_count, 0, (ncell + 1) * sizeof(int32_t), s));
    CK(cudaMemsetAsync(h->d_cell_cursor, 0, (ncell + 1) * sizeof(int32_t), s));
    LAUNCH(h, s, KC_NBLIST, k_cell_count<<<nblk(n, 256), 256, 0, s>>>(n, pos, bx, nc[0], nc[1], nc[2], h->d_atom_cell,
                                                                     h->d_cell_count));
    size_t tb = h->cub_bytes;
    LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::ExclusiveSum(h->d_cub, tb, h->d_cell_count, h->d_cell_start, ncell + 1, s));
    LAUNCH(h, s, KC_NBLIST, k_cell_fill<<<nblk(n, 256), 256, 0, s>>>(n, h->d_atom_cell, h->d_cell_start,
                                                                    h->d_cell_cursor, h->d_cell_atoms));
    Nb2Args b;
    b.a.n = n;
    b.a.pos = pos;
    b.a.box = bx;
    b.a.rc = h->rc;
    for (int k = 0; k < 3; ++k) b.a.nc[k] = nc[k];
    b.a.cell_start = h->d_cell_start;
    b.a.cell_atoms = h->d_cell_atoms;
    b.a.cov_ptr = h->d_cov_ptr;
    b.a.cov_j = h->d_cov_j;
    b.a.cov_nb = h->d_cov_nb;
    b.a.cov_lo = h->d_cov_lo;
    b.a.cov_hi = h->d_cov_hi;
    b.a.count = h->d_pcount;
    b.a.offset = h->d_poff;
    b.posf = h->d_posf;
    // the full CSR feeds only the polarizable dipole solve; other engines take the half rows alone
    const bool want_csr = h->kind == 0 && h->lpol;
    b.count_f = want_csr ? h->d_pcount_f : nullptr;
    b.off_f = want_csr ? h->d_csr_off : nullptr;
    b.ent = nullptr;
    b.cap_f = 0;
    if (fine) {
        // keep masks for the fill pass: room for 1.5x the mean candidate count (125 cells of the
        // stencil) per atom, at most 1 GiB; atoms with more candidates repeat the distance tests
        const double mean_cand = 125.0 * (double)n / (double)ncell;
        int64_t stride = (int64_t)ceil(1.5 * mean_cand / 32.0) + 2;
        if ((int64_t)n * stride * 4 > ((int64_t)1 << 30)) stride = 0;
        if (stride > 0 && (int64_t)n * stride > h->nbmask_cap) {
            if (h->d_nbmask) cudaFree(h->d_nbmask);
            h->d_nbmask = nullptr;
            h->nbmask_cap = (int64_t)n * stride;
            if ((st = dalloc(h, &h->d_nbmask, h->nbmask_cap * sizeof(uint32_t)))) return st;
        }
        b.mask = stride > 0 ? h->d_nbmask : nullptr;
        b.mask_stride = (int)stride;
    }
    // small neighbourhoods (staging room for 1.5x the mean candidate count within 44 KB): one CTA
    // per cell with the candidates staged in shared memory; larger ones keep the warp-per-atom
    // kernel, whose L2 gathers run at full occupancy (measured faster there than 100 KB stages)
    const int chmax = (int)(1.5 * 125.0 * (double)n / (double)ncell + 64.0);
    const size_t stage_bytes = (size_t)chmax * sizeof(float4);
    const bool staged = stage_bytes <= kNbStageBytes;
    const bool ortho = m[1] == 0.0 && m[2] == 0.0 && m[3] == 0.0 && m[5] == 0.0 && m[6] == 0.0 && m[7] == 0.0;
    if (!h->d_maxdeg && (st = dalloc(h, &h->d_maxdeg, 2 * sizeof(int)))) return st;
    int maxdeg[2] = {0, 0};
    // Single pass: the distance tests run once, each atom's rows and CSR entries go to its slots,
    // the scans of the counts place them and k_ell_compact copies them there (the same row set
    // and CSR as the two passes below).  Taken when the last two-pass build sized the slots; if a
    // count or a total outgrows its capacity, the two-pass build runs after all.
    if (fine && staged && h->ell_cap_h > 0 && (!want_csr || h->ell_cap_f > 0) && h->d_pairs &&
        (!want_csr || h->d_csr_ent)) {
        Nb2Args e = b;
        e.mask = nullptr;
        e.mask_stride = 0;
        e.ell_rows = h->d_ell_rows;
        e.ell_ent = want_csr ? h->d_ell_ent : nullptr;
        e.ell_cap_h = h->ell_cap_h;
        e.ell_cap_f = h->ell_cap_f;
        e.maxdeg = h->d_maxdeg;
        CK(cudaMemsetAsync(h->d_maxdeg, 0, 2 * sizeof(int), s));
        if (ortho) LAUNCH(h, s, KC_NBLIST, k_pairs_cell<2, 2, kNbWarps, true><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(e, chmax));
        else LAUNCH(h, s, KC_NBLIST, k_pairs_cell<2, 2, kNbWarps, false><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(e, chmax));
        CK(cudaMemsetAsync(h->d_poff, 0, sizeof(int64_t), s));
        tb = h->cub_bytes;
        LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::InclusiveSum(h->d_cub, tb, h->d_pcount, h->d_poff + 1, n, s));
        if (want_csr) {
            CK(cudaMemsetAsync(h->d_csr_off, 0, sizeof(int64_t), s));
            tb = h->cub_bytes;
            LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::InclusiveSum(h->d_cub, tb, h->d_pcount_f, h->d_csr_off + 1, n, s));
        }
        LAUNCH(h, s, KC_NBLIST, k_ell_compact<<<nblk((int64_t)n * 32, 256), 256, 0, s>>>(
                                    n, h->d_pcount, h->d_pcount_f, h->d_poff, h->d_csr_off, h->d_ell_rows, h->ell_cap_h,
                                    want_csr ? h->d_ell_ent : nullptr, h->ell_cap_f, h->d_pairs, h->pair_cap,
                                    want_csr ? h->d_csr_ent : nullptr, h->csr_cap));
        CK(cudaGetLastError());
        // the totals travel to pinned memory behind an event; no host wait here (nb_finish)
        if (!h->h_nbtot && cudaMallocHost((void**)&h->h_nbtot, 4 * sizeof(int64_t)) != cudaSuccess)
            return fail(h, DMFFB_OOM, "cudaMallocHost failed");
        h->h_nbtot[0] = h->h_nbtot[1] = h->h_nbtot[2] = h->h_nbtot[3] = 0;
        if (want_csr) CK(cudaMemcpyAsync(h->h_nbtot + 1, h->d_csr_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(h->h_nbtot, h->d_poff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(h->h_nbtot + 2, h->d_maxdeg, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (!h->e_nbtot) CK(cudaEventCreateWithFlags(&h->e_nbtot, cudaEventDisableTiming));
        CK(cudaEventRecord(h->e_nbtot, s));
        if (!h->e_build) CK(cudaEventCreateWithFlags(&h->e_build, cudaEventDisableTiming));
        CK(cudaEventRecord(h->e_build, s));
        h->nb_pending = true;
        h->nb_want_csr = want_csr;
        h->nb_stream = s;
        h->nb_pos = pos;
        for (int k = 0; k < 9; ++k) h->nb_box[k] = box[k];
        h->npairs = 0;
        h->have_pairs = true;
        h->pairs_gen++;
        h->csr_from_build = want_csr;
        if (h->prof) {
            const int stf = nb_finish(h);
            if (stf) return stf;
            prof_collect(h);
        }
        return DMFFB_OK;
    }
    b.maxdeg = h->d_maxdeg;
    CK(cudaMemsetAsync(h->d_maxdeg, 0, 2 * sizeof(int), s));
    if (fine && !staged) LAUNCH(h, s, KC_NBLIST, k_pairs_warp3<0, 2><<<nblk((int64_t)n * 32, 32 * kNbWarps), 32 * kNbWarps, 0, s>>>(b));
    else if (fine && ortho) LAUNCH(h, s, KC_NBLIST, k_pairs_cell<0, 2, kNbWarps, true><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(b, chmax));
    else if (fine) LAUNCH(h, s, KC_NBLIST, k_pairs_cell<0, 2, kNbWarps, false><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(b, chmax));
    else LAUNCH(h, s, KC_NBLIST, k_pairs_warp2<0><<<nblk((int64_t)n * 32, 256), 256, 0, s>>>(b));
    CK(cudaMemsetAsync(h->d_poff, 0, sizeof(int64_t), s));
    tb = h->cub_bytes;
    LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::InclusiveSum(h->d_cub, tb, h->d_pcount, h->d_poff + 1, n, s));
    int64_t tot[2] = {0, 0};
    if (want_csr) {
        CK(cudaMemsetAsync(h->d_csr_off, 0, sizeof(int64_t), s));
        tb = h->cub_bytes;
        LAUNCH(h, s, KC_NBLIST, cub::DeviceScan::InclusiveSum(h->d_cub, tb, h->d_pcount_f, h->d_csr_off + 1, n, s));
        CK(cudaMemcpyAsync(&tot[1], h->d_csr_off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaMemcpyAsync(&tot[0], h->d_poff + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(maxdeg, h->d_maxdeg, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    // slots for the next build's single pass: the largest counts with an eighth (at least 16) of
    // headroom, for the cell-staged kernel only (the warp-per-atom kernels leave maxdeg at 0)
    if (fine && staged && maxdeg[0] > 0) {
        const int ch = maxdeg[0] + std::max(16, maxdeg[0] / 8), cf = maxdeg[1] + std::max(16, maxdeg[1] / 8);
        if (ch > h->ell_cap_h || (want_csr && cf > h->ell_cap_f)) {
            if (h->d_ell_rows) cudaFree(h->d_ell_rows);
            if (h->d_ell_ent) cudaFree(h->d_ell_ent);
            h->d_ell_rows = nullptr;
            h->d_ell_ent = nullptr;
            h->ell_cap_h = h->ell_cap_f = 0;
            if ((st = dalloc(h, &h->d_ell_rows, (size_t)h->n_cap * ch * 3 * sizeof(int32_t)))) return st;
            if (want_csr && (st = dalloc(h, &h->d_ell_ent, (size_t)h->n_cap * cf * sizeof(int32_t)))) return st;
            h->ell_cap_h = ch;
            h->ell_cap_f = want_csr ? cf : 0;
        }
    }
    if (tot[0] > h->pair_cap) {
        if (h->d_pairs) cudaFree(h->d_pairs);
        h->pair_cap = (int64_t)(tot[0] * 1.3) + 64;  // headroom as in nblist.py:37-38
        if ((st = dalloc(h, &h->d_pairs, h->pair_cap * 3 * sizeof(int32_t)))) return st;
    }
    if (want_csr && tot[1] > h->csr_cap) {
        if (h->d_csr_ent) cudaFree(h->d_csr_ent);
        h->csr_cap = (int64_t)(tot[1] * 1.3) + 1024;
        if ((st = dalloc(h, &h->d_csr_ent, h->csr_cap * sizeof(int32_t)))) return st;
    }
    b.a.pairs = h->d_pairs;
    b.a.cap = h->pair_cap;
    b.ent = want_csr ? h->d_csr_ent : nullptr;
    b.cap_f = want_csr ? h->csr_cap : 0;
    if (fine && !staged) LAUNCH(h, s, KC_NBLIST, k_pairs_warp3<1, 2><<<nblk((int64_t)n * 32, 32 * kNbWarps), 32 * kNbWarps, 0, s>>>(b));
    else if (fine && ortho) LAUNCH(h, s, KC_NBLIST, k_pairs_cell<1, 2, kNbWarps, true><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(b, chmax));
    else if (fine) LAUNCH(h, s, KC_NBLIST, k_pairs_cell<1, 2, kNbWarps, false><<<ncell, 32 * kNbWarps, stage_bytes, s>>>(b, chmax));
    else LAUNCH(h, s, KC_NBLIST, k_pairs_warp2<1><<<nblk((int64_t)n * 32, 256), 256, 0, s>>>(b));
    CK(cudaGetLastError());
    // no host wait for the fill pass: later work on this stream is ordered after it, and compute
    // calls on other streams wait for e_build before they read the engine's list
    if (h->prof) {
        CK(cudaStreamSynchronize(s));
        prof_collect(h);
    }
    if (!h->e_build) CK(cudaEventCreateWithFlags(&h->e_build, cudaEventDisableTiming));
    CK(cudaEventRecord(h->e_build, s));
    h->npairs = tot[0];
    h->have_pairs = true;
    h->pairs_gen++;
    h->csr_from_build = want_csr;
    return DMFFB_OK;
}

int dmffb_engine_pairs(dmffb_engine* h, void* stream, int32_t* pairs_out, int64_t capacity, int64_t* npairs_out) {
    if (!h || !npairs_out) return fail(h, DMFFB_BAD_ARG, "null argument");
    if (!h->have_pairs) return fail(h, DMFFB_BAD_ARG, "the engine has no neighbour list yet");
    {
        const int st = nb_finish(h);
        if (st) return st;
    }
    cudaStream_t s = (cudaStream_t)stream;
    *npairs_out = h->npairs;
    if (h->npairs > capacity || (!pairs_out && h->npairs > 0)) {
        h->err = "pair capacity too small";
        return DMFFB_NEIGHBOR_OVERFLOW;
    }
    if (h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
    if (h->npairs > 0)
        CK(cudaMemcpyAsync(pairs_out, h->d_pairs, (size_t)h->npairs * 3 * sizeof(int32_t), cudaMemcpyDeviceToDevice, s));
    return DMFFB_OK;
}

int dmffb_disp_create(const dmffb_disp_desc* d, dmffb_engine** out) {
    if (!d || !out) return DMFFB_BAD_ARG;
    *out = nullptr;
    if (d->n_atoms <= 0 || (d->pmax != 6 && d->pmax != 8 && d->pmax != 10)) return DMFFB_BAD_ARG;
    dmffb_admp_desc a;
    memset(&a, 0, sizeof(a));
    a.n_atoms = d->n_atoms;
    a.lmax = 0;
    a.lpol = 0;
    a.lpme = d->lpme;
    a.precision = d->precision;
    a.rc = d->rc;
    a.kappa = d->kappa;
    for (int k = 0; k < 3; ++k) a.K[k] = d->K[k];
    a.n_cov = d->n_cov;
    a.cov_rows = d->cov_rows;
    for (int k = 0; k < 6; ++k) a.mscales[k] = a.pscales[k] = a.dscales[k] = d->mscales[k];
    a.cg_tol = 1e-6;
    a.max_iter = 1;
    int st = dmffb_admp_create(&a, out);
    dmffb_engine* h = *out;
    if (st) return st;
    h->kind = 1;
    h->pmax = d->pmax;
    h->tt = d->tt_damping ? 1 : 0;
    const int n = h->n;
    const size_t ts = h->prec == DMFFB_FP32 ? 4 : 8;
    if ((st = dalloc(h, &h->d_c, 3 * n * ts)) || (st = dalloc(h, &h->d_tta, n * ts)) ||
        (st = dalloc(h, &h->d_ttb, n * ts)) || (st = dalloc(h, &h->d_ttq, n * ts)) || (st = dalloc(h, &h->d_glr, 3 * n * ts)) ||
        (st = dalloc(h, &h->d_gsr, 3 * n * ts)) || (st = dalloc(h, &h->d_dc, 3 * n * sizeof(double))))
        return st;
    return DMFFB_OK;
}

int dmffb_disp_set_params(dmffb_engine* h, const double* c_list, const double* a, const double* b, const double* q) {
    if (!h || h->kind != 1 || !c_list) return fail(h, DMFFB_BAD_ARG, "dispersion engine and c_list required");
    if (h->tt && (!a || !b || !q)) return fail(h, DMFFB_BAD_ARG, "TT damping needs a, b, q");
    const int n = h->n;
    // host: channel-major copy and the self energy (disp_pme.py:264-289)
    std::vector<double> cm(3 * n);
    double s6 = 0, s8 = 0, s10 = 0;
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) cm[(size_t)k * n + i] = c_list[3 * i + k];
        s6 += c_list[3 * i] * c_list[3 * i];
        s8 += c_list[3 * i + 1] * c_list[3 * i + 1];
        s10 += c_list[3 * i + 2] * c_list[3 * i + 2];
    }
    const double k2 = h->kappa * h->kappa;
    double e = -k2 * k2 * k2 / 12.0 * s6;
    if (h->pmax >= 8) e -= k2 * k2 * k2 * k2 / 48.0 * s8;
    if (h->pmax >= 10) e -= k2 * k2 * k2 * k2 * k2 / 240.0 * s10;
    h->e_self_disp = e;
    // staged through the FP64 gradient scratch ([3n], rewritten by every compute), on the engine stream
    double* tmp = h->d_grad;
    auto up = [&](const double* src, int m, void* dst) -> int {
        CK(cudaMemcpyAsync(tmp, src, m * sizeof(double), cudaMemcpyHostToDevice, h->s1));
        if (h->prec == DMFFB_FP32) k_to_t<float><<<nblk(m, 256), 256, 0, h->s1>>>(m, tmp, (float*)dst);
        else k_to_t<double><<<nblk(m, 256), 256, 0, h->s1>>>(m, tmp, (double*)dst);
        CK(cudaStreamSynchronize(h->s1));
        return DMFFB_OK;
    };
    int st = up(cm.data(), 3 * n, h->d_c);
    if (!st && h->tt) st = up(a, n, h->d_tta);
    if (!st && h->tt) st = up(b, n, h->d_ttb);
    if (!st && h->tt) st = up(q, n, h->d_ttq);
    if (st) return st;
    h->params_set = true;
    return DMFFB_OK;
}

int dmffb_disp_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                       int64_t npairs, double* forces_lr, double* forces_sr, dmffb_disp_result* result) {
    if (!h || h->kind != 1 || !pos || !box || !result) return fail(h, DMFFB_BAD_ARG, "bad arguments");
    cudaStream_t caller = (cudaStream_t)stream;
    CK(cudaEventRecord(h->e_in, caller));
    CK(cudaStreamWaitEvent(h->s1, h->e_in, 0));
    int st = h->prec == DMFFB_FP32 ? disp_compute_impl<float>(h, h->s1, pos, box, pairs, npairs, forces_lr, forces_sr, result)
                                   : disp_compute_impl<double>(h, h->s1, pos, box, pairs, npairs, forces_lr, forces_sr, result);
    cudaEventRecord(h->e_out, h->s1);
    cudaStreamWaitEvent(caller, h->e_out, 0);
    return st;
}

int dmffb_disp_set_param_grads(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 1) return fail(h, DMFFB_BAD_ARG, "dispersion engine required");
    if (enabled && h->tt && !h->d_dsr) {
        int st = dalloc(h, &h->d_dsr, 4 * (size_t)h->n_cap * sizeof(double));
        if (st) return st;
    }
    h->want_pgrad = enabled != 0;
    return DMFFB_OK;
}

int dmffb_disp_param_grads(dmffb_engine* h, void* stream, double* dE_dc, double* dEsr_dabqc) {
    if (!h || h->kind != 1) return fail(h, DMFFB_BAD_ARG, "dispersion engine required");
    if (!h->have_pgrad) return fail(h, DMFFB_BAD_ARG, "enable dmffb_disp_set_param_grads before compute");
    cudaStream_t cs = (cudaStream_t)stream;
    if (dE_dc) CK(cudaMemcpyAsync(dE_dc, h->d_dc, 3 * (size_t)h->n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (dEsr_dabqc) {
        if (h->tt) CK(cudaMemcpyAsync(dEsr_dabqc, h->d_dsr, 4 * (size_t)h->n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
        else CK(cudaMemsetAsync(dEsr_dabqc, 0, 4 * (size_t)h->n * sizeof(double), cs));
    }
    return DMFFB_OK;
}

}  // extern "C"

template <typename T>
int pairwise_compute_impl(dmffb_engine* h, cudaStream_t s, const double* pos, const double* box, const int32_t* pairs,
                          int64_t npairs, double* forces, dmffb_pairwise_result* res) {
    if (!h->params_set) return fail(h, DMFFB_BAD_ARG, "dmffb_pairwise_set_params was not called");
    if (!pos || !box || !res) return fail(h, DMFFB_BAD_ARG, "null pos/box/result");
    Box bx;
    make_box(box, bx);
    memset(res, 0, sizeof(*res));
    const int n = h->n;
    int st;
    if (!pairs) {
        if (!h->have_pairs)
            if ((st = dmffb_admp_build_neighbors(h, (void*)s, pos, box))) return st;
        if ((st = nb_finish(h))) return st;
        if (h->e_build) CK(cudaStreamWaitEvent(s, h->e_build, 0));
        pairs = h->d_pairs;
        npairs = h->npairs;
    }
    res->n_pairs = npairs;
    const bool pg = h->want_pgrad;
    const int np = sr_nparam(h->sr_kind);
    CK(cudaMemsetAsync(h->d_scal, 0, N_SCAL * sizeof(double), s));
    CK(cudaMemsetAsync(h->d_srgrad, 0, (size_t)3 * n * sizeof(T), s));
    if (pg) CK(cudaMemsetAsync(h->d_srdp, 0, (size_t)np * n * sizeof(double), s));
    if (npairs > 0) {
        SrArgs<T> a;
        a.n = n;
        a.npairs = npairs;
        a.pairs = pairs;
        a.pos = pos;
        a.p = (const T*)h->d_srp;
        for (int k = 0; k < 6; ++k) a.ms[k] = (T)h->ms[k];
        a.sign = (T)h->sr_sign;
        a.boxd = bx;
        a.grad = (T*)h->d_srgrad;
        a.dp = pg ? h->d_srdp : nullptr;
        a.scal = h->d_scal;
        const unsigned nbk = nblk(npairs, 128);
        switch (h->sr_kind) {
            case SR_TT_QQ: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_TT_QQ><<<nbk, 128, 0, s>>>(a)); break;
            case SR_SLATER_DISP: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_SLATER_DISP><<<nbk, 128, 0, s>>>(a)); break;
            case SR_SLATER: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_SLATER><<<nbk, 128, 0, s>>>(a)); break;
            case SR_QEQ_GAUSS3: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_QEQ_GAUSS3><<<nbk, 128, 0, s>>>(a)); break;
            case SR_QEQ_GAUSS2: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_QEQ_GAUSS2><<<nbk, 128, 0, s>>>(a)); break;
            default: LAUNCH(h, s, KC_PAIR_FULL, k_sr_pair<T, SR_TT_QQ_C6><<<nbk, 128, 0, s>>>(a)); break;
        }
        CK(cudaGetLastError());
    }
    if (forces) LAUNCH(h, s, KC_VEC, k_sr_finalize<T><<<nblk(3 * n, 256), 256, 0, s>>>(n, (const T*)h->d_srgrad, forces));
    CK(cudaMemcpyAsync(h->h_scal, h->d_scal, N_SCAL * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    prof_collect(h);
    res->energy = h->h_scal[0];
    for (int k = 0; k < 9; ++k) res->box_grad[k] = h->h_scal[1 + k];
    h->have_pgrad = pg;
    if (!std::isfinite(res->energy)) return fail(h, DMFFB_NONFINITE, "non-finite energy");
    return DMFFB_OK;
}

extern "C" {

int dmffb_pairwise_create(const dmffb_pairwise_desc* d, dmffb_engine** out) {
    if (!d || !out) return DMFFB_BAD_ARG;
    *out = nullptr;
    if (d->n_atoms <= 0 || d->kind < DMFFB_SR_TT_QQ || d->kind > DMFFB_SR_QEQ_GAUSS2 || !(d->rc > 0)) return DMFFB_BAD_ARG;
    dmffb_admp_desc a;
    memset(&a, 0, sizeof(a));
    a.n_atoms = d->n_atoms;
    a.precision = d->precision;
    a.rc = d->rc;
    a.n_cov = d->n_cov;
    a.cov_rows = d->cov_rows;
    for (int k = 0; k < 6; ++k) a.mscales[k] = a.pscales[k] = a.dscales[k] = d->mscales[k];
    a.cg_tol = 1e-6;
    a.max_iter = 1;
    int st = dmffb_admp_create(&a, out);
    dmffb_engine* h = *out;
    if (st) return st;
    h->kind = 3;
    h->sr_kind = d->kind;
    h->sr_sign = d->sign == 0.0 ? 1.0 : d->sign;
    const int n = h->n;
    const size_t ts = h->prec == DMFFB_FP32 ? 4 : 8;
    if ((st = dalloc(h, &h->d_srp, 4 * (size_t)n * ts)) || (st = dalloc(h, &h->d_srdp, 4 * (size_t)n * sizeof(double))) ||
        (st = dalloc(h, &h->d_srgrad, 3 * (size_t)n * ts)))
        return st;
    return DMFFB_OK;
}

int dmffb_pairwise_set_params(dmffb_engine* h, const double* params) {
    if (!h || h->kind != 3 || !params) return fail(h, DMFFB_BAD_ARG, "pairwise engine and parameters required");
    const int np = sr_nparam(h->sr_kind);
    const int64_t m = (int64_t)np * h->n;
    cudaStream_t s = h->s1;
    // staged in the gradient scratch, then converted to kernel precision
    CK(cudaMemcpyAsync(h->d_srdp, params, m * sizeof(double), cudaMemcpyHostToDevice, s));
    if (h->prec == DMFFB_FP32) k_to_t<float><<<nblk(m, 256), 256, 0, s>>>((int)m, h->d_srdp, (float*)h->d_srp);
    else k_to_t<double><<<nblk(m, 256), 256, 0, s>>>((int)m, h->d_srdp, (double*)h->d_srp);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    h->params_set = true;
    h->have_pgrad = false;
    return DMFFB_OK;
}

int dmffb_pairwise_set_param_grads(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 3) return fail(h, DMFFB_BAD_ARG, "pairwise engine required");
    h->want_pgrad = enabled != 0;
    return DMFFB_OK;
}

int dmffb_pairwise_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                           int64_t npairs, double* forces_out, dmffb_pairwise_result* result) {
    if (!h || h->kind != 3) return fail(h, DMFFB_BAD_ARG, "pairwise engine required");
    if (pairs && npairs < 0) return fail(h, DMFFB_BAD_ARG, "negative npairs");
    cudaStream_t caller = (cudaStream_t)stream;
    CK(cudaEventRecord(h->e_in, caller));
    CK(cudaStreamWaitEvent(h->s1, h->e_in, 0));
    int st = h->prec == DMFFB_FP32 ? pairwise_compute_impl<float>(h, h->s1, pos, box, pairs, npairs, forces_out, result)
                                   : pairwise_compute_impl<double>(h, h->s1, pos, box, pairs, npairs, forces_out, result);
    cudaEventRecord(h->e_out, h->s1);
    cudaStreamWaitEvent(caller, h->e_out, 0);
    return st;
}

int dmffb_pairwise_param_grads(dmffb_engine* h, void* stream, double* dE_dparams) {
    if (!h || h->kind != 3 || !dE_dparams) return fail(h, DMFFB_BAD_ARG, "pairwise engine and output required");
    if (!h->have_pgrad) return fail(h, DMFFB_BAD_ARG, "enable dmffb_pairwise_set_param_grads before compute");
    const int np = sr_nparam(h->sr_kind);
    CK(cudaMemcpyAsync(dE_dparams, h->d_srdp, (size_t)np * h->n * sizeof(double), cudaMemcpyDeviceToDevice,
                       (cudaStream_t)stream));
    return DMFFB_OK;
}

int dmffb_classical_create(const dmffb_classical_desc* d, dmffb_engine** out) {
    if (!d || !out) return DMFFB_BAD_ARG;
    *out = nullptr;
    if (d->n_atoms <= 0 || d->n_types < 0 || d->coulomb < DMFFB_COUL_NONE || d->coulomb > DMFFB_COUL_NOCUTOFF)
        return DMFFB_BAD_ARG;
    if (d->coulomb == DMFFB_COUL_RF && !(d->rc > 0)) return DMFFB_BAD_ARG;
    dmffb_admp_desc a;
    memset(&a, 0, sizeof(a));
    a.n_atoms = d->n_atoms;
    a.lmax = 0;
    a.lpol = 0;
    a.lpme = d->coulomb == DMFFB_COUL_PME ? 1 : 0;
    a.precision = d->precision;
    a.rc = d->rc;
    a.kappa = d->kappa;
    for (int k = 0; k < 3; ++k) a.K[k] = d->K[k];
    a.n_cov = d->n_cov;
    a.cov_rows = d->cov_rows;
    for (int k = 0; k < 6; ++k) a.mscales[k] = a.pscales[k] = a.dscales[k] = d->mscales_coul[k];
    a.cg_tol = 1e-6;
    a.max_iter = 1;
    int st = dmffb_admp_create(&a, out);
    dmffb_engine* h = *out;
    if (st) return st;
    h->kind = 2;
    h->ntypes = d->n_types;
    h->coul = d->coulomb;
    h->pbc = d->pbc ? 1 : 0;
    for (int k = 0; k < 6; ++k) h->mlj[k] = d->mscales_lj[k];
    if (d->coulomb == DMFFB_COUL_RF) {  // inter.py:196-203
        const double es = d->eps_solvent > 0 ? d->eps_solvent : 78.5;
        h->krf = (1.0 / (d->rc * d->rc * d->rc)) * (es - 1.0) / (2.0 * es + 1.0);
        h->crf = (1.0 / d->rc) * 3.0 * es / (2.0 * es + 1.0);
    }
    const int n = h->n;
    const size_t ts = h->prec == DMFFB_FP32 ? 4 : 8;
    const size_t tt = (size_t)std::max(1, h->ntypes) * std::max(1, h->ntypes);
    if ((st = dalloc(h, &h->d_q, n * sizeof(double))) || (st = dalloc(h, &h->d_qT, n * ts)) ||
        (st = dalloc(h, &h->d_type, n * sizeof(int32_t))) || (st = dalloc(h, &h->d_sigtt, tt * ts)) ||
        (st = dalloc(h, &h->d_epstt, tt * ts)) || (st = dalloc(h, &h->d_dq, n * sizeof(double))) ||
        (st = dalloc(h, &h->d_dsig, tt * sizeof(double))) || (st = dalloc(h, &h->d_deps, tt * sizeof(double))) ||
        (st = dalloc(h, &h->d_glr, 3 * n * ts)))
        return st;
    // covalent rows (i < j) and each atom's partner index range, for the cell pass
    {
        std::vector<int32_t> rows(3 * std::max<int64_t>(d->n_cov, 1)), lo(n, n), hi(n, -1);
        for (int64_t r = 0; r < d->n_cov; ++r) {
            const int i = d->cov_rows[3 * r], j = d->cov_rows[3 * r + 1];
            const int a0 = std::min(i, j), a1 = std::max(i, j);
            rows[3 * r] = a0;
            rows[3 * r + 1] = a1;
            rows[3 * r + 2] = d->cov_rows[3 * r + 2];
            lo[a0] = std::min(lo[a0], a1);
            hi[a0] = std::max(hi[a0], a1);
            lo[a1] = std::min(lo[a1], a0);
            hi[a1] = std::max(hi[a1], a0);
        }
        h->n_covrows = d->n_cov;
        if ((st = dalloc(h, &h->d_covrows, rows.size() * sizeof(int32_t))) ||
            (st = dalloc(h, &h->d_cov_lo, n * sizeof(int32_t))) || (st = dalloc(h, &h->d_cov_hi, n * sizeof(int32_t))))
            return st;
        CK(cudaMemcpyAsync(h->d_covrows, rows.data(), rows.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
        CK(cudaMemcpyAsync(h->d_cov_lo, lo.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
        CK(cudaMemcpyAsync(h->d_cov_hi, hi.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
        CK(cudaStreamSynchronize(h->s1));
    }
    return DMFFB_OK;
}

int dmffb_classical_set_cell_pass(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 2) return fail(h, DMFFB_BAD_ARG, "classical engine required");
    h->cell_pass = enabled != 0;
    return DMFFB_OK;
}

int dmffb_classical_set_params(dmffb_engine* h, const double* charges, const int32_t* atom_type,
                               const double* sigma_tt, const double* eps_tt) {
    if (!h || h->kind != 2) return fail(h, DMFFB_BAD_ARG, "classical engine required");
    if (h->coul != COUL_NONE && !charges) return fail(h, DMFFB_BAD_ARG, "Coulomb needs charges");
    if (h->ntypes > 0 && (!atom_type || !sigma_tt || !eps_tt)) return fail(h, DMFFB_BAD_ARG, "LJ needs types and tables");
    const int n = h->n;
    const int nt = h->ntypes;
    if (nt > 0)
        for (int i = 0; i < n; ++i)
            if (atom_type[i] < 0 || atom_type[i] >= nt) return fail(h, DMFFB_BAD_ARG, "atom type out of range");
    std::vector<double> qz(n, 0.0);
    const double* q = charges ? charges : qz.data();
    double s2 = 0.0;
    for (int i = 0; i < n; ++i) s2 += q[i] * q[i];
    h->e_self_coul = -DMFFB_DIELECTRIC * h->kappa / sqrt(M_PI) * s2;  // pme.py:1183-1222, lmax 0
    cudaStream_t s = h->s1;
    CK(cudaMemcpyAsync(h->d_q, q, n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (h->prec == DMFFB_FP32) k_to_t<float><<<nblk(n, 256), 256, 0, s>>>(n, h->d_q, (float*)h->d_qT);
    else k_to_t<double><<<nblk(n, 256), 256, 0, s>>>(n, h->d_q, (double*)h->d_qT);
    CK(cudaStreamSynchronize(s));
    if (nt > 0) {
        CK(cudaMemcpyAsync(h->d_type, atom_type, n * sizeof(int32_t), cudaMemcpyHostToDevice, s));
        const int m = nt * nt;
        double* tmp = h->d_dsig;  // [nt^2] FP64 adjoint scratch, zeroed by every compute that uses it
        for (int w = 0; w < 2; ++w) {
            CK(cudaMemcpyAsync(tmp, w == 0 ? sigma_tt : eps_tt, m * sizeof(double), cudaMemcpyHostToDevice, s));
            void* dst = w == 0 ? h->d_sigtt : h->d_epstt;
            if (h->prec == DMFFB_FP32) k_to_t<float><<<nblk(m, 256), 256, 0, s>>>(m, tmp, (float*)dst);
            else k_to_t<double><<<nblk(m, 256), 256, 0, s>>>(m, tmp, (double*)dst);
            CK(cudaStreamSynchronize(s));
        }
    }
    CK(cudaGetLastError());
    h->params_set = true;
    return DMFFB_OK;
}

int dmffb_classical_set_terms(dmffb_engine* h, int32_t kind, int64_t n_terms, const int32_t* idx, const double* prm) {
    if (!h || h->kind != 2 || kind < 0 || kind > 2 || n_terms < 0 || (n_terms > 0 && (!idx || !prm)))
        return fail(h, DMFFB_BAD_ARG, "bad term list");
    if (n_terms > 0x7fffffff) return fail(h, DMFFB_BAD_ARG, "too many terms");
    const int arity = kind + 2, np = kind == 2 ? 3 : 2;
    for (int64_t t = 0; t < n_terms * arity; ++t)
        if (idx[t] < 0 || idx[t] >= h->n) return fail(h, DMFFB_BAD_ARG, "term atom index out of range");
    if (h->d_tidx[kind]) cudaFree(h->d_tidx[kind]);
    if (h->d_tprm[kind]) cudaFree(h->d_tprm[kind]);
    if (h->d_tdprm[kind]) cudaFree(h->d_tdprm[kind]);
    h->d_tidx[kind] = nullptr;
    h->d_tprm[kind] = nullptr;
    h->d_tdprm[kind] = nullptr;
    h->nterm[kind] = 0;
    if (n_terms == 0) return DMFFB_OK;
    int st;
    if ((st = dalloc(h, &h->d_tidx[kind], n_terms * arity * sizeof(int32_t))) ||
        (st = dalloc(h, &h->d_tprm[kind], n_terms * np * sizeof(double))) ||
        (st = dalloc(h, &h->d_tdprm[kind], n_terms * 2 * sizeof(double))))
        return st;
    CK(cudaMemcpyAsync(h->d_tidx[kind], idx, n_terms * arity * sizeof(int32_t), cudaMemcpyHostToDevice, h->s1));
    CK(cudaMemcpyAsync(h->d_tprm[kind], prm, n_terms * np * sizeof(double), cudaMemcpyHostToDevice, h->s1));
    CK(cudaStreamSynchronize(h->s1));
    h->nterm[kind] = n_terms;
    return DMFFB_OK;
}

int dmffb_classical_set_param_grads(dmffb_engine* h, int32_t enabled) {
    if (!h || h->kind != 2) return fail(h, DMFFB_BAD_ARG, "classical engine required");
    h->want_pgrad = enabled != 0;
    return DMFFB_OK;
}

int dmffb_classical_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                            int64_t npairs, double* forces_out, dmffb_classical_result* result) {
    if (!h || h->kind != 2 || !pos || !box || !result) return fail(h, DMFFB_BAD_ARG, "bad arguments");
    cudaStream_t caller = (cudaStream_t)stream;
    CK(cudaEventRecord(h->e_in, caller));
    CK(cudaStreamWaitEvent(h->s1, h->e_in, 0));
    int st = h->prec == DMFFB_FP32 ? classical_compute_impl<float>(h, h->s1, pos, box, pairs, npairs, forces_out, result)
                                   : classical_compute_impl<double>(h, h->s1, pos, box, pairs, npairs, forces_out, result);
    cudaEventRecord(h->e_out, h->s1);
    cudaStreamWaitEvent(caller, h->e_out, 0);
    return st;
}

int dmffb_classical_param_grads(dmffb_engine* h, void* stream, double* dE_dq, double* dE_dsig, double* dE_deps,
                                double* dE_dbond, double* dE_dangle, double* dE_dtorsion) {
    cudaStream_t cs = (cudaStream_t)stream;
    if (!h || h->kind != 2) return fail(h, DMFFB_BAD_ARG, "classical engine required");
    if (!h->want_pgrad) return fail(h, DMFFB_BAD_ARG, "parameter gradients are not enabled");
    const size_t tt = (size_t)h->ntypes * h->ntypes;
    if (dE_dq) CK(cudaMemcpyAsync(dE_dq, h->d_dq, h->n * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (dE_dsig && tt) CK(cudaMemcpyAsync(dE_dsig, h->d_dsig, tt * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    if (dE_deps && tt) CK(cudaMemcpyAsync(dE_deps, h->d_deps, tt * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    double* dst[3] = {dE_dbond, dE_dangle, dE_dtorsion};
    for (int k = 0; k < 3; ++k)
        if (dst[k] && h->nterm[k] > 0)
            CK(cudaMemcpyAsync(dst[k], h->d_tdprm[k], h->nterm[k] * 2 * sizeof(double), cudaMemcpyDeviceToDevice, cs));
    return DMFFB_OK;
}

int dmffb_get_timings(const dmffb_engine* h, double* ms_out, int32_t n) {
    if (!h || !ms_out) return DMFFB_BAD_ARG;
    for (int k = 0; k < n && k < 6; ++k) ms_out[k] = h->t_ms[k];
    return DMFFB_OK;
}

int dmffb_set_profiling(dmffb_engine* h, int32_t enabled) {
    if (!h) return DMFFB_BAD_ARG;
    h->prof = enabled != 0;
    for (int k = 0; k < 32; ++k) { h->kstat_ms[k] = 0; h->kstat_n[k] = 0; }
    return DMFFB_OK;
}

int dmffb_get_kernel_stats(const dmffb_engine* h, double* ms_out, int64_t* launches_out, int32_t n) {
    if (!h) return DMFFB_BAD_ARG;
    for (int k = 0; k < n && k < KC_COUNT; ++k) {
        if (ms_out) ms_out[k] = h->kstat_ms[k];
        if (launches_out) launches_out[k] = h->kstat_n[k];
    }
    return DMFFB_OK;
}

int dmffb_get_counters(const dmffb_engine* h, int64_t* out, int32_t n) {
    if (!h || !out) return DMFFB_BAD_ARG;
    if (n > 0) out[0] = h->n_launch;
    if (n > 1) out[1] = h->n_fft;
    return DMFFB_OK;
}

int dmffb_set_timing(dmffb_engine* h, int32_t enabled) {
    if (!h) return DMFFB_BAD_ARG;
    h->timing = enabled != 0;
    return DMFFB_OK;
}

int dmffb_set_fused_fft(dmffb_engine* h, int32_t enabled) {
    if (!h) return DMFFB_BAD_ARG;
    h->fc_enabled = enabled != 0;
    return DMFFB_OK;
}

int dmffb_set_persistent_cg(dmffb_engine* h, int32_t mode) {
    if (!h || mode < 0 || mode > 2) return DMFFB_BAD_ARG;
    h->pcg_mode = mode;
    return DMFFB_OK;
}

int dmffb_persistent_cg_blocks(const dmffb_engine* h) {
    if (!h) return -1;
    return pcg_wanted(h) && h->pcg_max_blocks > 0 ? h->pcg_max_blocks : 0;
}

int dmffb_get_cg_phase_times(const dmffb_engine* h, double* ms_out, int32_t n) {
    if (!h || !ms_out || n < 0) return DMFFB_BAD_ARG;
    for (int k = 0; k < n && k < 8; ++k) ms_out[k] = h->pcg_phase_ms[k];
    return DMFFB_OK;
}

int dmffb_set_cg_wait_limit(dmffb_engine* h, double seconds, int32_t phantom_arrivals) {
    if (!h || !(seconds > 0) || phantom_arrivals < 0) return DMFFB_BAD_ARG;
    h->pcg_wait_s = seconds;
    h->pcg_phantom = phantom_arrivals;
    return DMFFB_OK;
}

int dmffb_fused_fft_active(const dmffb_engine* h) {
    if (!h) return -1;
    return h->fc_enabled && h->fc_ok > 0 ? 1 : 0;
}

int dmffb_set_graphs(dmffb_engine* h, int32_t enabled) {
    if (!h) return DMFFB_BAD_ARG;
    h->use_graphs = enabled != 0;
    if (!h->use_graphs && h->cg_exec) {
        cudaGraphExecDestroy(h->cg_exec);
        h->cg_exec = nullptr;
        h->cg_key.clear();
    }
    return DMFFB_OK;
}

}  // extern "C"
