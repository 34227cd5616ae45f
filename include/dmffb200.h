/*
 * dmffb200.h — C ABI of the B200 ADMP / PME energy-force engine (libdmffb200.so).
 *
 * Plain pointers and sizes only; no C++ or torch types cross this boundary.  Every call
 * returns a status (DMFFB_OK == 0); on failure `dmffb_last_error(h)` holds a message.
 * Units follow the reference backend: Angstrom, elementary charge, kJ/mol.
 *
 * The reference (deepmodeling/DMFF) has no C ABI (backend/c_api/CMakeLists.txt is empty);
 * each entry point below names the Python interface it replaces.
 */
#ifndef DMFFB200_H
#define DMFFB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DMFFB_OK = 0,
    DMFFB_BAD_ARG = 1,
    DMFFB_OOM = 2,
    DMFFB_CUDA_ERROR = 3,
    DMFFB_NOT_CONVERGED = 4,      /* warning: results written, induced dipoles not converged */
    DMFFB_NEIGHBOR_OVERFLOW = 5,  /* pair capacity too small; *npairs_out holds the count needed */
    DMFFB_NONFINITE = 6,
    DMFFB_CUFFT_ERROR = 7,
    DMFFB_SCRATCH_TOO_SMALL = 8,  /* request exceeds a fixed-size scratch limit (see the _noalloc entry) */
    DMFFB_TIMEOUT = 9             /* a bounded device-side wait ran out; the context stays usable */
};

/* local-axis types, dmff/admp/spatial.py:59-65 */
enum { DMFFB_ZTHENX = 0, DMFFB_BISECTOR = 1, DMFFB_ZBISECT = 2, DMFFB_THREEFOLD = 3,
       DMFFB_ZONLY = 4, DMFFB_NOAXISTYPE = 5 };

/* arithmetic of the pair / mesh kernels (energies, virials and CG norms are always FP64) */
enum { DMFFB_FP32 = 0, DMFFB_FP64 = 1 };

/* induced-dipole solver */
enum { DMFFB_SOLVER_CG = 0,          /* Jacobi-preconditioned CG to RMS(dE/dU) < cg_tol */
       DMFFB_SOLVER_REFERENCE = 1 }; /* U <- U - (dE/dU) pol / DIELECTRIC, dmff/admp/pme.py:342-423 */

typedef struct dmffb_engine dmffb_engine;

/* Static description of one ADMP multipolar PME system.
 * Replaces ADMPPmeForce.__init__ (dmff/admp/pme.py:43-114) plus the covalent map that
 * ADMPPmeGenerator.createPotential builds (dmff/generators/admp.py:1203-1336). */
typedef struct {
    int32_t n_atoms;
    int32_t lmax;             /* 0, 1, 2 */
    int32_t lpol;             /* induced dipoles on/off */
    int32_t lpme;             /* 0: kappa = 0 and no reciprocal part (CutoffPeriodic) */
    int32_t precision;        /* DMFFB_FP32 | DMFFB_FP64 */
    double rc;                /* cutoff, Angstrom (used by the internal neighbour build) */
    double kappa;             /* Ewald kappa, 1/Angstrom (setup_ewald_parameters, pme.py:426-466) */
    int32_t K[3];             /* PME mesh */
    const int32_t* axis_types;   /* [n_atoms] host, DMFFB_* axis type */
    const int32_t* axis_indices; /* [n_atoms*3] host, (z, x, y) atoms, -1 = unused */
    int64_t n_cov;               /* sparse covalent map rows */
    const int32_t* cov_rows;     /* [n_cov*3] host (i, j, nbond) with i < j, 1 <= nbond <= 6 */
    double mscales[6];        /* indexed nbond-1, [5] = 1.0 (trailing entry, admp.py:912-918) */
    double pscales[6];
    double dscales[6];
    int32_t solver;           /* DMFFB_SOLVER_* */
    double cg_tol;            /* CG: stop when RMS(dE/dU) <= cg_tol * RMS(dE/dU at U = 0);
                                 REFERENCE: POL_CONV, stop when max|dE/dU| < cg_tol (pme.py:394) */
    int32_t max_iter;         /* CG / reference iteration cap */
    int32_t steps_pol;        /* REFERENCE solver: >0 runs exactly this many steps (pme.py:404-422) */
} dmffb_admp_desc;

typedef struct {
    double energy;            /* total, kJ/mol */
    double e_real, e_recip, e_self, e_pol;
    double box_grad[9];       /* dE/dbox (rows = lattice vectors), kJ/mol/A, fixed Cartesian positions */
    int32_t n_iter;           /* dipole iterations used */
    int32_t converged;
    double residual_rms;      /* final RMS dE/dU */
    int64_t n_pairs;          /* pair rows processed */
} dmffb_admp_result;

/* ADMPPmeForce(...) — pme.py:43-114 */
int dmffb_admp_create(const dmffb_admp_desc* desc, dmffb_engine** out);
void dmffb_destroy(dmffb_engine* h);
const char* dmffb_last_error(const dmffb_engine* h);

/* Re-point an existing engine at another system of the same kind (same lmax, lpol, lpme and
 * precision) with n_atoms <= the n_atoms it was created with: new positions' topology, cut-off,
 * Ewald kappa / mesh K, scales and solver settings.  Device buffers are reused (grown only for a
 * larger mesh or covalent map); cuFFT plans are cached per mesh shape.  The neighbour list,
 * dipole-solve graph and parameters of the previous system are dropped: call set_params next.
 * No counterpart in the reference (its ADMPPmeForce is rebuilt per system); this is what lets a
 * serving loop keep a fixed pool of engines.  Returns DMFFB_SCRATCH_TOO_SMALL when n_atoms
 * exceeds the capacity. */
int dmffb_admp_reconfigure(dmffb_engine* h, const dmffb_admp_desc* desc);

/* Per-atom parameters, host arrays: Q_local [n*9] harmonic local-frame multipoles in the
 * reference's units (params["ADMPPmeForce"]["Q_local"][map_atomtype], admp.py:1373),
 * zero-padded to 9 components; pol [n] (A^3) and thole [n] (may be NULL when lpol == 0). */
int dmffb_admp_set_params(dmffb_engine* h, const double* Q_local, const double* pol, const double* thole);

/* Energy + forces + box gradient: ADMPPmeForce.get_energy (pme.py:186-232) with
 * jax.value_and_grad over (positions, box).  Device pointers: pos [n*3] A, U_inout [n*3]
 * (Cartesian induced dipoles e*A; read as the initial guess, overwritten with the solution;
 * may be NULL when lpol == 0), forces_out [n*3] (= -dE/dpos, may be NULL).  pairs is a
 * device array of npairs rows (i, j, nbond) with the reference's padding semantics (rows with
 * i >= j are skipped, utils.py:67-85); pairs == NULL uses the engine's own neighbour list
 * (built on the first call and by dmffb_admp_build_neighbors), while a non-NULL pairs with
 * npairs == 0 is an empty list (no real-space pairs).  box [9] is a host array.
 * stream: a cudaStream_t (NULL = legacy default stream). */
int dmffb_admp_compute(dmffb_engine* h, void* stream, const double* pos, const double* box,
                       const int32_t* pairs, int64_t npairs, double* U_inout, double* forces_out,
                       dmffb_admp_result* result);

/* Same call with HOST buffers: the engine copies pos/pairs/U in and forces/U out
 * (the path an OpenMM plugin or a ctypes caller without device memory uses). */
int dmffb_admp_compute_host(dmffb_engine* h, const double* pos, const double* box,
                            const int32_t* pairs, int64_t npairs, double* U_inout, double* forces_out,
                            dmffb_admp_result* result);

/* dE/dU at the given dipoles (the "field" of optimize_Uind, pme.py:381-392), device arrays. */
int dmffb_admp_field(dmffb_engine* h, void* stream, const double* pos, const double* box,
                     const int32_t* pairs, int64_t npairs, const double* U, double* field_out);

/* Parameter adjoints on/off for the following computes.  When on, compute() also evaluates,
 * at the converged induced dipoles (where E is stationary in U, so no adjoint solve is needed),
 * the derivatives of the energy with respect to every atom's multipoles, polarizability and
 * Thole width: the quantities jax.grad gives for params["ADMPPmeForce"] in the reference
 * (dmff/admp/pme.py:186-232 under jax.value_and_grad), before the per-type scatter. */
int dmffb_admp_set_param_grads(dmffb_engine* h, int32_t enabled);
/* Zero initial guess on/off for the following computes of a polarizable engine.  When on, the
 * dipole solve starts from U = 0 whatever U_inout holds (the solution is still written to it) and
 * skips the A U evaluation of the CG set-up.  dmffb_admp_compute_host with U_inout == NULL starts
 * from zero in the same way.  The reference's get_energy with U_init = None starts from zeros. */
int dmffb_admp_set_zero_guess(dmffb_engine* h, int32_t enabled);
/* Per-atom parameter adjoints of the last compute (device arrays, each may be NULL):
 * dE/dQ_global [n*9] and dE/dQ_local [n*9] (harmonic), dE/dpol [n] (A^-3 kJ/mol),
 * dE/dthole [n]. */
int dmffb_admp_param_grads(dmffb_engine* h, void* stream, double* dE_dQglobal, double* dE_dQlocal,
                           double* dE_dpol, double* dE_dthole);
/* The same adjoints copied to HOST arrays (dE/dQ_local [n*9], dE/dpol [n], dE/dthole [n], each may
 * be NULL): for callers of dmffb_admp_compute_host that hold no device memory. */
int dmffb_admp_param_grads_host(dmffb_engine* h, double* dE_dQlocal, double* dE_dpol, double* dE_dthole);
/* dE/dQ_global and dE/dQ_local only (same requirements as dmffb_admp_param_grads). */
int dmffb_admp_multipole_grads(dmffb_engine* h, void* stream, double* dE_dQglobal, double* dE_dQlocal);

/* Second-order pass: the vector-Jacobian product through the first derivatives of the last
 * dmffb_admp_compute, i.e. the derivatives of
 *     L = <c.pos, dE/dpos> + <c.box, dE/dbox> + <c.Q_local, dE/dQ_local> + <c.pol, dE/dpol>
 *         + <c.thole, dE/dthole>
 * with respect to positions, box and every atom's Q_local / pol / thole, with the induced dipoles
 * following their parameters and positions (total derivatives of the converged solution).  This
 * is what a loss on forces or on the virial needs for its parameter gradients (force matching,
 * dmff/optimize.py:30-84 over jax.grad of forces); the reference's jax.grad cannot give it because
 * its dipole solve is stop-gradiented (dmff/admp/pme.py:212-213, 363-371).  The dipole response
 * comes from one adjoint linear solve with the engine's CG (A dU = -d2E/dU dz c, A the dipole
 * matrix), not from unrolling the iteration; the directional derivatives of the engine's analytic
 * first derivatives along c are central differences with a step of 1e-4 (FP64 engines; 3e-3 for
 * FP32) of each quantity's own scale (1 A for positions and box), the pair list held fixed.
 * Requirements: a preceding dmffb_admp_compute whose positions, pairs and U_inout arrays still
 * hold the values of that call, converged dipoles (CG solver), the same parameters.  The pass
 * overwrites the last compute's parameter adjoints (dmffb_admp_param_grads needs a new compute).
 * Device arrays; each cotangent and each output may be NULL (zero / not wanted). */
typedef struct {
    const double* pos;      /* [n*3] cotangent of dE/dpos (= -forces) */
    double box[9];          /* cotangent of dE/dbox (host) */
    const double* Q_local;  /* [n*9] cotangent of dE/dQ_local */
    const double* pol;      /* [n] */
    const double* thole;    /* [n] */
} dmffb_admp_cotangent;

typedef struct {
    double* pos;          /* [n*3] dL/dpos */
    double box[9];        /* dL/dbox (host) */
    double* Q_local;      /* [n*9] dL/dQ_local */
    double* pol;          /* [n] dL/dpol */
    double* thole;        /* [n] dL/dthole */
    int32_t n_iter;       /* CG iterations of the adjoint solve (0 without polarization) */
    double residual_rms;  /* its final RMS residual */
    double step;          /* the finite-difference step along c */
} dmffb_admp_second;

int dmffb_admp_backward(dmffb_engine* h, void* stream, const dmffb_admp_cotangent* c, dmffb_admp_second* out);

/* Cell-list neighbour build: NeighborList.allocate (dmff/common/nblist.py:27-55) semantics —
 * all i < j with minimum-image distance < rc (FP64 test), nbond from the covalent map.
 * pos device [n*3]; box host [9]; rows written to pairs_out (device, capacity rows), sorted by i.
 * Returns DMFFB_NEIGHBOR_OVERFLOW with *npairs_out = needed count when capacity is short. */
int dmffb_build_neighbors(dmffb_engine* h, void* stream, const double* pos, const double* box, double rc,
                          int32_t* pairs_out, int64_t capacity, int64_t* npairs_out);

/* Rebuild the engine-owned pair list used when compute() gets pairs == NULL.  From an engine's
 * second build on, this returns without waiting for the device: the row count reaches the host
 * behind an event, and the list's first user (compute(), dmffb_engine_pairs) waits for it.  The
 * build reads pos on the given stream; if a slot outgrows its capacity, that first user rebuilds
 * the list from the same pos pointer, so keep the positions unchanged until then. */
int dmffb_admp_build_neighbors(dmffb_engine* h, void* stream, const double* pos, const double* box);

/* Copy of the engine's own neighbour list (the rows compute() uses when pairs == NULL), the
 * counterpart of the reference's NeighborList.pairs property (dmff/common/nblist.py:62-64) without
 * its padding rows: npairs rows (i, j, nbond), i < j, sorted by i, written to pairs_out (device,
 * capacity rows) on the given stream after the last build.  *npairs_out = the row count;
 * DMFFB_NEIGHBOR_OVERFLOW when capacity is short (nothing written). */
int dmffb_engine_pairs(dmffb_engine* h, void* stream, int32_t* pairs_out, int64_t capacity, int64_t* npairs_out);

/* Per-stage device times of the last compute() in milliseconds (CUDA events):
 * [0] frames, [1] pol solve, [2] real FULL, [3] recip FULL, [4] self+frames, [5] total. */
int dmffb_get_timings(const dmffb_engine* h, double* ms_out, int32_t n);
int dmffb_set_timing(dmffb_engine* h, int32_t enabled);

/* Per-kernel-class instrumentation: with profiling on, every launch is bracketed by CUDA events
 * on its stream and its duration is added to its class.  Classes: 0 prepare/frames, 1 pair FULL,
 * 2 pair FIELD, 3 pair MATVEC, 4 spread, 5 FFT (cuFFT), 6 convolution, 7 gather FULL,
 * 8 gather FIELD, 9 self+frame forces, 10 vector/CG ops, 11 neighbour build, 12 CG matvec
 * pair-tensor set-up, 13 pair FULL over the topologically scaled rows (FP64), 14 pair FIELD over
 * the scaled rows (FP64), 15 parameter-adjoint pair kernels, 16 bonded terms, 17 the engine-FFT
 * convolution of the dipole solve (dmffb_set_fused_fft), 18 the persistent CG solve
 * (dmffb_set_persistent_cg).  Classes 1 and 2
 * hold only the launches over the unscaled rows (kernel precision). */
int dmffb_set_profiling(dmffb_engine* h, int32_t enabled);
int dmffb_get_kernel_stats(const dmffb_engine* h, double* ms_out, int64_t* launches_out, int32_t n);
/* [0] launches of this library's kernels since create, [1] cuFFT executions. */
int dmffb_get_counters(const dmffb_engine* h, int64_t* out, int32_t n);

/* ---------------------------------------------------------------------------------------
 * Dispersion PME with optional Tang-Toennies short range.
 * dmffb_disp_create replaces ADMPDispPmeForce.__init__ (dmff/admp/disp_pme.py:21-40) plus the
 * pairwise TT set-up of ADMPDispGenerator.createPotential (dmff/generators/admp.py:150-174). */
typedef struct {
    int32_t n_atoms;
    int32_t pmax;             /* 6, 8 or 10 */
    int32_t lpme;             /* 0: kappa = 0, no reciprocal part */
    int32_t precision;        /* DMFFB_FP32 | DMFFB_FP64 */
    double rc, kappa;         /* Angstrom, 1/Angstrom */
    int32_t K[3];
    int64_t n_cov;
    const int32_t* cov_rows;  /* host [n_cov*3] (i, j, nbond), i < j */
    double mscales[6];        /* nbond-1 indexed, [5] = 1.0 */
    int32_t tt_damping;       /* 1: also evaluate ADMPDispForce's E_sr (pairwise.py:100-118) */
} dmffb_disp_desc;

typedef struct {
    double energy;            /* E_lr = real + recip + self (disp_pme.py:80-130), kJ/mol */
    double e_real, e_recip, e_self;
    double e_sr;              /* TT short range (0 unless tt_damping) */
    double box_grad[9];       /* dE_lr/dbox */
    double box_grad_sr[9];    /* dE_sr/dbox */
    int64_t n_pairs;
} dmffb_disp_result;

int dmffb_disp_create(const dmffb_disp_desc* desc, dmffb_engine** out);
/* c_list host [n*3] = sqrt(C6 1e6), sqrt(C8 1e8), sqrt(C10 1e10) (admp.py:373-378); a, b, q host [n]
 * (A/2625.5, B*0.0529177249, Q; admp.py:187-193), NULL without TT.  ADMPDispPmeForce.get_energy
 * argument c_list (disp_pme.py:45-49). */
int dmffb_disp_set_params(dmffb_engine* h, const double* c_list, const double* a, const double* b, const double* q);
/* forces_lr = -dE_lr/dpos, forces_sr = -dE_sr/dpos (device [n*3], either may be NULL);
 * pairs as in dmffb_admp_compute (NULL: the engine's own neighbour list). */
int dmffb_disp_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                       int64_t npairs, double* forces_lr, double* forces_sr, dmffb_disp_result* result);
/* Parameter adjoints on/off for the following computes (the C6/C8/C10 and TT A/B/Q entries of
 * jax.grad over params in the reference, dmff/admp/disp_pme.py:45-77, pairwise.py:47-118). */
int dmffb_disp_set_param_grads(dmffb_engine* h, int32_t enabled);
/* Adjoints of the last compute (device arrays, each may be NULL): dE_lr/dc [3n] channel-major
 * (c = sqrt(C_n 10^n) per atom: real space + reciprocal + self), dE_sr/d(a, b, q, c6) [4n]
 * channel-major (TT short range; zero without TT). */
int dmffb_disp_param_grads(dmffb_engine* h, void* stream, double* dE_dc, double* dEsr_dabqc);

/* ---------------------------------------------------------------------------------------
 * Classical terms: Lennard-Jones + point-charge Coulomb (PME real+reciprocal+self, reaction
 * field, or plain 1/r) and harmonic bonds / angles / periodic torsions.
 * dmffb_classical_create replaces the set-up of CoulombPMEForce / CoulReactionFieldForce /
 * CoulNoCutoffForce / LennardJonesForce (dmff/classical/inter.py:17-335) and of
 * HarmonicBondJaxForce / HarmonicAngleJaxForce / PeriodicTorsionJaxForce (intra.py:32-138),
 * as NonbondedGenerator, CoulombGenerator, LennardJonesGenerator and the bonded generators
 * build them (dmff/generators/classical.py:154-1394).  Units: Angstrom, e, kJ/mol, radians. */
enum { DMFFB_COUL_NONE = 0, DMFFB_COUL_PME = 1, DMFFB_COUL_RF = 2, DMFFB_COUL_NOCUTOFF = 3 };
enum { DMFFB_TERM_BOND = 0, DMFFB_TERM_ANGLE = 1, DMFFB_TERM_TORSION = 2 };

typedef struct {
    int32_t n_atoms;
    int32_t n_types;          /* LJ type count (0: no LJ) */
    int32_t precision;        /* DMFFB_FP32 | DMFFB_FP64 (pair and mesh arithmetic) */
    int32_t coulomb;          /* DMFFB_COUL_* */
    int32_t pbc;              /* minimum image on pair vectors (LJ and reaction field; PME always) */
    double rc;                /* cutoff, Angstrom: internal neighbour build and reaction field */
    double kappa;             /* Ewald kappa, 1/Angstrom (PME) */
    int32_t K[3];             /* PME mesh */
    double eps_solvent;       /* reaction field dielectric (inter.py:205, default 78.5) */
    int64_t n_cov;
    const int32_t* cov_rows;  /* host [n_cov*3] (i, j, nbond), i < j */
    double mscales_coul[6];   /* nbond-1 indexed, [5] = 1.0 (classical.py:878-881) */
    double mscales_lj[6];
} dmffb_classical_desc;

typedef struct {
    double energy;            /* sum of the terms below, kJ/mol */
    double e_coul_real, e_coul_recip, e_coul_self;
    double e_lj, e_bond, e_angle, e_torsion;
    double box_grad[9];       /* dE/dbox at fixed Cartesian positions */
    int64_t n_pairs;
} dmffb_classical_result;

int dmffb_classical_create(const dmffb_classical_desc* desc, dmffb_engine** out);
/* Per-atom charges [n] (may be NULL without Coulomb) and LJ type index [n] with type-pair tables
 * sigma_tt, eps_tt [n_types^2] (Angstrom, kJ/mol; mixing rule and NBFix already applied), host. */
int dmffb_classical_set_params(dmffb_engine* h, const double* charges, const int32_t* atom_type,
                               const double* sigma_tt, const double* eps_tt);
/* Bonded term list, host arrays: kind DMFFB_TERM_*; idx [n_terms * (2|3|4)] atom indices;
 * prm: bond (k kJ/mol/A^2, r0 A), angle (k kJ/mol/rad^2, theta0), torsion (k, psi, periodicity)
 * per term.  Replaces the index/parameter gathers of classical.py:154-787. */
int dmffb_classical_set_terms(dmffb_engine* h, int32_t kind, int64_t n_terms, const int32_t* idx,
                              const double* prm);
/* Parameter adjoints on/off for the following computes (dE/dq, dE/dsigma_tt, dE/deps_tt, dE/dprm). */
int dmffb_classical_set_param_grads(dmffb_engine* h, int32_t enabled);
/* Energy, forces (= -dE/dpos, device [n*3], may be NULL) and box gradient; pairs as in
 * dmffb_admp_compute (NULL: the engine's own neighbour list, rc from the description). */
int dmffb_classical_compute(dmffb_engine* h, void* stream, const double* pos, const double* box,
                            const int32_t* pairs, int64_t npairs, double* forces_out,
                            dmffb_classical_result* result);
/* Cell pass on/off for the following computes (off by default).  When on, a compute with pairs ==
 * NULL evaluates every pair within rc at the positions it is given straight from a cell binning of
 * those positions, without writing a pair list: the same pairs (the list build's exact FP64
 * cut-off test), scales and results as dmffb_admp_build_neighbors followed by a compute on the
 * engine's list.  Pairs with a topological scale run in FP64 from the covalent rows.  Needs
 * periodic boxes at least 5 half cut-offs wide; parameter adjoints and narrower boxes take the
 * list path.  No counterpart in the reference (its potentials always take a pair list). */
int dmffb_classical_set_cell_pass(dmffb_engine* h, int32_t enabled);
/* Parameter adjoints of the last compute (param grads enabled), device arrays, each may be NULL:
 * dE_dq [n], dE_dsig [n_types^2], dE_deps [n_types^2], dE_dbond / dE_dangle / dE_dtorsion
 * [n_terms*2] = (dE/dk, dE/d(r0 | theta0 | psi)). */
int dmffb_classical_param_grads(dmffb_engine* h, void* stream, double* dE_dq, double* dE_dsig, double* dE_deps,
                                double* dE_dbond, double* dE_dangle, double* dE_dtorsion);

/* The dipole-solve iterations' reciprocal convolution (forward FFT, influence-function multiply,
 * inverse FFT) through the engine's own three-pass FFT (x-planes, spectrum columns with the
 * multiply, x-planes) instead of cuFFT R2C + convolution + C2R, on/off (off by default; FP32
 * engines with meshes of at most 64 points per axis, else cuFFT).
 * dmffb_fused_fft_active returns 1 when the last solve used it, 0 for the cuFFT path. */
int dmffb_set_fused_fft(dmffb_engine* h, int32_t enabled);
/* The whole CG dipole solve in one persistent cooperative launch (k_cg_solve: direction update,
 * real-space matvec and dipole spread, the engine-FFT convolution, field gather and CG update per
 * iteration, separated by grid barriers; convergence decided on the device, one read-back per
 * solve).  mode 0: off (the graph-replayed per-pass solve), 1: on, 2 (default): on for systems of
 * at most 4096 atoms, where the launch chain of the per-pass solve dominates.  FP32 engines with
 * meshes of at most 64 points per axis on devices with cooperative launch only.
 * dmffb_persistent_cg_blocks returns the co-resident CTAs available to it for the current mesh
 * (0: not used).
 * dmffb_set_cg_wait_limit bounds every grid-barrier wait of the kernel (default 2 s): past it the
 * solve returns DMFFB_TIMEOUT with the context usable; phantom_arrivals > 0 makes the next solve's
 * first barrier wait for arrivals that never come (for tests of that path). */
int dmffb_set_persistent_cg(dmffb_engine* h, int32_t mode);
int dmffb_persistent_cg_blocks(const dmffb_engine* h);
int dmffb_set_cg_wait_limit(dmffb_engine* h, double seconds, int32_t phantom_arrivals);
/* Device-clock time of each pass of the persistent solve (0 direction update, 1 matvec + spread,
 * 2 forward planes, 3 spectrum columns, 4 inverse planes, 5 field gather, 6 CG update; barrier
 * waits included, measured on CTA 0), summed over the solves run while profiling was on. */
int dmffb_get_cg_phase_times(const dmffb_engine* h, double* ms_out, int32_t n);
int dmffb_fused_fft_active(const dmffb_engine* h);
/* ---------------------------------------------------------------------------------------
 * Short-range pairwise terms with per-atom parameters: the built-in kernels of
 * dmff/admp/pairwise.py evaluated in CUDA (what generate_pairwise_interaction, pairwise.py:47-95,
 * does for them in the reference), for the short-range generators of dmff/generators/admp.py
 * (QqTtDampingForce :400-526, SlaterDampingForce :529-669, SlaterExForce and the SlaterSrEs /
 * SlaterSrPol / SlaterSrDisp / SlaterDhf terms :672-863).  Per-atom parameters, host
 * [nparam * n] channel-major, in Angstrom units as the generators pass them:
 *   DMFFB_SR_TT_QQ       (b, q):           -DIELECTRIC e^-br (1 + br) q_i q_j / r, b = sqrt(b_i b_j)
 *   DMFFB_SR_SLATER_DISP (b, c6, c8, c10): Slater-ISA damped C6/C8/C10 (pairwise.py:131-156)
 *   DMFFB_SR_SLATER      (a, b):           a_i a_j ((br)^2 / 3 + br + 1) e^-br (pairwise.py:159-171)
 *   DMFFB_SR_TT_QQ_C6    (a, b, q, c):     TT_damping_qq_c6_kernel (pairwise.py:100-118)
 *   DMFFB_SR_QEQ_GAUSS3  (q, eta):         -DIELECTRIC erfc(r / s) q_i q_j / r, s = sqrt(eta_i^2 + eta_j^2),
 *                                          0 for s <= 1e-4 (ADMPQeqForce DampMod 3, dmff/admp/qeq.py:98-112)
 *   DMFFB_SR_QEQ_GAUSS2  (q, eta):         the same with s = sqrt(2 (eta_i^2 + eta_j^2)) (DampMod 2, :85-95)
 * each times mscales[nbond - 1] and the description's sign.  The parameter adjoints of the QEq
 * kinds with respect to q are the short-range part of the charge Hessian times q. */
enum { DMFFB_SR_TT_QQ = 0, DMFFB_SR_SLATER_DISP = 1, DMFFB_SR_SLATER = 2, DMFFB_SR_TT_QQ_C6 = 3,
       DMFFB_SR_QEQ_GAUSS3 = 4, DMFFB_SR_QEQ_GAUSS2 = 5 };

typedef struct {
    int32_t n_atoms;
    int32_t kind;             /* DMFFB_SR_* */
    int32_t precision;        /* DMFFB_FP32 | DMFFB_FP64 */
    double rc;                /* cutoff of the internal neighbour build, Angstrom */
    int64_t n_cov;
    const int32_t* cov_rows;  /* host [n_cov*3] (i, j, nbond), i < j */
    double mscales[6];        /* nbond-1 indexed, [5] = 1.0 */
    double sign;              /* overall factor: 1, or -1 for the SlaterSr* / SlaterDhf terms */
} dmffb_pairwise_desc;

typedef struct {
    double energy;            /* kJ/mol */
    double box_grad[9];
    int64_t n_pairs;
} dmffb_pairwise_result;

int dmffb_pairwise_create(const dmffb_pairwise_desc* desc, dmffb_engine** out);
int dmffb_pairwise_set_params(dmffb_engine* h, const double* params);
int dmffb_pairwise_set_param_grads(dmffb_engine* h, int32_t enabled);
/* forces_out = -dE/dpos (device [n*3], may be NULL); pairs as in dmffb_admp_compute. */
int dmffb_pairwise_compute(dmffb_engine* h, void* stream, const double* pos, const double* box, const int32_t* pairs,
                           int64_t npairs, double* forces_out, dmffb_pairwise_result* result);
/* dE/dparameter of the last compute (device [nparam*n], channel-major). */
int dmffb_pairwise_param_grads(dmffb_engine* h, void* stream, double* dE_dparams);

/* CUDA-graph capture of the dipole-solve loop on/off for this engine (on by default). */
int dmffb_set_graphs(dmffb_engine* h, int32_t enabled);

/* ---------------------------------------------------------------------------------------
 * Serving: continuous batching of independent ADMP evaluations (energy + forces + virial) on
 * one GPU.  No counterpart in the reference (its callers evaluate one system at a time through
 * ADMPPmeForce.get_energy, dmff/admp/pme.py:186-232).  A server owns a pool of engines ("slots",
 * each with its own streams, created at capacity_atoms and re-pointed at each request with
 * dmffb_admp_reconfigure) and one host worker thread per slot.  Requests wait in arrival order;
 * the head request is admitted when its arrival time has passed, a slot is idle and the summed
 * device footprint of the requests in flight plus its own stays within hbm_budget_bytes.
 * Admitted requests run concurrently on their slots' streams, so small requests overlap on the
 * GPU while large ones limit how many run at once.  With n_slots > 1 the slots run the per-pass
 * dipole solve (its short kernels interleave across slots); with one slot the persistent solve
 * serves small requests (dmffb_set_persistent_cg mode 2). */
typedef struct dmffb_server dmffb_server;

typedef struct {
    int32_t n_slots;          /* engines / worker threads */
    int32_t capacity_atoms;   /* largest request */
    int64_t hbm_budget_bytes; /* admission limit on summed request footprints (0: no limit) */
    int32_t lmax, lpol, precision;
    double mscales[6], pscales[6], dscales[6];
    int32_t solver;
    double cg_tol;
    int32_t max_iter;
    int32_t use_graphs;
} dmffb_server_desc;

typedef struct {
    /* inputs (host memory, alive until the request completes) */
    int32_t n_atoms;
    const double* pos;           /* [n*3] A */
    double box[9];               /* A, rows = lattice vectors */
    const int32_t* axis_types;   /* [n] */
    const int32_t* axis_indices; /* [n*3] */
    int64_t n_cov;
    const int32_t* cov_rows;     /* [n_cov*3] */
    const double* Q_local;       /* [n*9] */
    const double* pol;           /* [n] or NULL */
    const double* thole;         /* [n] or NULL */
    double rc, kappa;
    int32_t K[3];
    double t_arrival;            /* seconds on the server clock; not admitted before */
    /* outputs */
    double* forces_out;          /* [n*3] host, -dE/dpos */
    double energy;
    double box_grad[9];
    int32_t n_iter;
    int32_t status;              /* DMFFB_* of the evaluation */
    int32_t slot;
    int32_t done;                /* set to 1 last */
    double t_start, t_done;      /* server clock */
    int64_t footprint_bytes;
} dmffb_request;

int dmffb_server_create(const dmffb_server_desc* desc, dmffb_server** out);
/* Queue a request (non-blocking).  Requests must be submitted in non-decreasing t_arrival. */
int dmffb_server_submit(dmffb_server* srv, dmffb_request* req);
/* Block until every submitted request is done or timeout_s passes (DMFFB_CUDA_ERROR on timeout). */
int dmffb_server_wait(dmffb_server* srv, double timeout_s);
/* Seconds since the server was created (the clock of t_arrival / t_start / t_done). */
double dmffb_server_clock(const dmffb_server* srv);
/* Device bytes a request of this size is accounted for at admission. */
int64_t dmffb_request_footprint(int32_t n_atoms, double rc, const int32_t K[3], double box_volume, int32_t lpol);
/* Run each request once on every slot, untimed (grows buffers and caches cuFFT plans). */
int dmffb_server_prewarm(dmffb_server* srv, dmffb_request* reqs, int32_t n_reqs);
void dmffb_server_destroy(dmffb_server* srv);

/* ---------------------------------------------------------------------------------------
 * MD-platform force: the polarizable ADMP engine inside an MD engine's step, in the device
 * layout of OpenMM's CUDA platform.  Replaces the reference's OpenMM plugin kernel
 * (backend/openmm_dmff_plugin/platforms/cuda/src/CudaDMFFKernels.cpp:118-220, addForces in
 * kernels/DMFFForce.cu:1-9), which moves positions and forces through the host every step and
 * keeps the induced dipoles on the host (last_U_ind, :193-195).  Here positions are gathered
 * from the platform's posq array on the device, the neighbour list is built on the device, the
 * dipoles stay in device memory from one step to the next (each solve starts from the previous
 * step's), and the forces are added to the platform's fixed-point force buffer by an epilogue
 * kernel.  include/dmffb200_openmm.hpp holds the C++ adapter an OpenMM kernel class wraps. */
typedef struct {
    const void* posq;           /* device [padded_num_atoms] float4 (double4 if posq_double): x, y, z in nm */
    int32_t posq_double;
    long long* force_buffer;    /* device [3 * padded_num_atoms]: force (kJ/mol/nm) * 2^32 as int64, x block first */
    const int32_t* atom_index;  /* device [num_atoms]: the system atom held in each slot (NULL: identity) */
    int32_t num_atoms, padded_num_atoms;
    double box_nm[9];           /* periodic box, rows = lattice vectors, nm */
    void* stream;               /* the platform's cudaStream_t */
} dmffb_md_context;

typedef struct dmffb_md_force dmffb_md_force;

/* desc in Angstrom (as dmffb_admp_create); Q_local [n*9], pol [n], thole [n] host arrays. */
int dmffb_md_force_create(const dmffb_admp_desc* desc, const double* Q_local, const double* pol, const double* thole,
                          dmffb_md_force** out);
/* One step: energy (kJ/mol) out; with include_forces the forces are added to ctx->force_buffer.
 * Returns DMFFB_NOT_CONVERGED as a warning (results written). */
int dmffb_md_force_execute(dmffb_md_force* f, const dmffb_md_context* ctx, int32_t include_forces,
                           double* energy_kjmol);
/* The engine result of the last step (CG iterations, energy terms, box gradient in kJ/mol/A). */
int dmffb_md_force_last_result(const dmffb_md_force* f, dmffb_admp_result* out);
/* Copy of the induced dipoles kept for the next step (device [n*3], e*A, system atom order). */
int dmffb_md_force_dipoles(dmffb_md_force* f, void* stream, double* U_out);
void dmffb_md_force_destroy(dmffb_md_force* f);

/* Neighbour-list build that allocates no device memory.  No counterpart in the reference (DMFF
 * has no C ABI); same result as dmffb_build_neighbors for callers that cannot allocate on
 * demand: a host (an MD platform such as an OpenMM context, a framework with a caching
 * allocator, a process under a fixed memory budget) that owns the device heap and forbids
 * cudaMalloc after start-up.  All scratch (cell bins, per-atom counts and offsets, scan storage)
 * lives in one fixed device array inside the library; the call makes no cudaMalloc / cudaFree
 * and calls no allocating library routine.  Needs no engine handle.
 *   pos: device [n_atoms*3] FP64, Angstrom; box: host [9]; rc > 0.
 *   cov_ptr/cov_j/cov_nb: device CSR of the covalent map restricted to j > i (rows of atom i are
 *     cov_j[cov_ptr[i] .. cov_ptr[i+1]-1] with nbond cov_nb[...]); all three NULL means nbond 0.
 *   pairs_out: device [capacity*3] rows (i, j, nbond), i < j, sorted by i; *npairs_out = count.
 * Limits: n_atoms <= DMFFB_NOALLOC_MAX_ATOMS (larger -> DMFFB_SCRATCH_TOO_SMALL); the cell grid
 * is coarsened to at most DMFFB_NOALLOC_MAX_CELLS cells.  The first call on a device does a
 * one-time set-up: it looks up the array's device address (cudaGetSymbolAddress) with that device
 * current; make that first call before any stream capture begins.  Every call reads the pair
 * count back to the host and waits for its stream to finish before it returns.  Every call on a
 * device shares the one array and each call re-zeroes what it accumulates into; calls that
 * overlap on the GPU (different streams, or host threads) race on it and must be serialized by
 * the caller. */
#define DMFFB_NOALLOC_MAX_ATOMS 65536
#define DMFFB_NOALLOC_MAX_CELLS 32768
int dmffb_build_neighbors_noalloc(void* stream, const double* pos, int32_t n_atoms, const double* box, double rc,
                                  const int32_t* cov_ptr, const int32_t* cov_j, const int32_t* cov_nb,
                                  int32_t* pairs_out, int64_t capacity, int64_t* npairs_out);

#ifdef __cplusplus
}
#endif
#endif
