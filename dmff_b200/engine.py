"""Python handle over the C-ABI engine (libdmffb200.so).

``AdmpEngine`` owns one ``dmffb_engine*``: static system data goes in at construction,
per-atom parameters through ``set_params``, and ``compute`` evaluates energy, forces,
box gradient and induced dipoles for positions already on the GPU (torch tensors are used
only as device buffers; their data pointers go through the C ABI).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L

_SOLVERS = {"cg": L.DMFFB_SOLVER_CG, "reference": L.DMFFB_SOLVER_REFERENCE}
_PREC = {"fp32": L.DMFFB_FP32, "fp64": L.DMFFB_FP64}


def _i32(a, shape=None):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
    if shape is not None:
        a = a.reshape(shape)
    return a


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _dev(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


_EMPTY_ROWS = {}


def _pairs_arg(pairs, device):
    """(pointer, row count) for the C ABI.  None means "use the engine's own neighbour list"; an
    explicitly empty list must still reach the engine as a non-null pointer with 0 rows (an empty
    CUDA tensor's data pointer is null), so it points at a one-row scratch buffer."""
    if pairs is None:
        return None, 0
    if pairs.shape[0] == 0:
        key = str(device)
        if key not in _EMPTY_ROWS:
            _EMPTY_ROWS[key] = torch.zeros((1, 3), dtype=torch.int32, device=device)
        return _dev(_EMPTY_ROWS[key]), 0
    return _dev(pairs), pairs.shape[0]


class AdmpEngine:
    """One ADMP multipolar PME system on one GPU.

    Parameters mirror ``ADMPPmeForce`` (dmff/admp/pme.py:43-114): ``lmax``, ``lpol``, ``lpme``,
    ``rc`` (A), ``kappa`` (1/A) and mesh ``K``; ``axis_types``/``axis_indices`` as built by the
    generator; ``cov_rows`` the sparse covalent map (i, j, nbond); scales of length 6 with the
    trailing 1.0.  ``precision`` 'fp32' (FP32 pair/mesh arithmetic, FP64 accumulation) or 'fp64'.
    ``solver`` 'cg' (converged to ``cg_tol`` RMS dE/dU) or 'reference' (the reference's fixed step
    iteration, ``steps_pol`` steps or until max|dE/dU| < ``cg_tol``)."""

    def __init__(self, n_atoms, lmax, lpol, lpme, rc, kappa, K, axis_types, axis_indices, cov_rows,
                 mscales, pscales=None, dscales=None, precision="fp32", solver="cg", cg_tol=1e-6, max_iter=500,
                 steps_pol=None, device=None):
        self.lib = L.load()
        self.n = self.n_cap = int(n_atoms)
        self.lmax, self.lpol, self.lpme, self.precision = int(lmax), bool(lpol), bool(lpme), precision
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        d = self._desc(n_atoms, rc, kappa, K, axis_types, axis_indices, cov_rows, mscales, pscales, dscales,
                       solver, cg_tol, max_iter, steps_pol)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_admp_create(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if st != L.DMFFB_OK:
            msg = self.lib.dmffb_last_error(h).decode() if h.value else "invalid description"
            if h.value:
                self.lib.dmffb_destroy(h)
            self.h = None
            raise L.EngineError(st, msg)
        self._U_buf = torch.zeros((self.n_cap, 3), dtype=torch.float64, device=self.device)
        self._F_buf = torch.zeros((self.n_cap, 3), dtype=torch.float64, device=self.device)
        self.U, self.forces = self._U_buf, self._F_buf

    def _desc(self, n_atoms, rc, kappa, K, axis_types, axis_indices, cov_rows, mscales, pscales, dscales, solver,
              cg_tol, max_iter, steps_pol):
        n = int(n_atoms)
        d = L.AdmpDesc()
        d.n_atoms = n
        d.lmax = self.lmax
        d.lpol = int(self.lpol)
        d.lpme = int(self.lpme)
        d.precision = _PREC[self.precision]
        d.rc = float(rc)
        d.kappa = float(kappa) if self.lpme else 0.0
        for k in range(3):
            d.K[k] = int(K[k]) if self.lpme else 0
        at = _i32(axis_types if axis_types is not None else np.full(n, 5), (n,))
        ai = _i32(axis_indices if axis_indices is not None else np.full((n, 3), -1), (n * 3,))
        cov = _i32(cov_rows if cov_rows is not None else np.zeros((0, 3)), (-1,))
        self._keep = (at, ai, cov)
        d.axis_types = _ptr(at)
        d.axis_indices = _ptr(ai)
        d.n_cov = cov.size // 3
        d.cov_rows = _ptr(cov)
        one6 = [0.0, 0.0, 1.0, 1.0, 1.0, 1.0]
        for k in range(6):
            d.mscales[k] = float(mscales[k])
            d.pscales[k] = float((pscales if pscales is not None else one6)[k])
            d.dscales[k] = float((dscales if dscales is not None else one6)[k])
        d.solver = _SOLVERS[solver]
        d.cg_tol = float(cg_tol)
        d.max_iter = int(max_iter)
        d.steps_pol = int(steps_pol) if steps_pol else 0
        return d

    def reconfigure(self, n_atoms, rc, kappa, K, axis_types, axis_indices, cov_rows, mscales, pscales=None,
                    dscales=None, solver="cg", cg_tol=1e-6, max_iter=500, steps_pol=None):
        """Point this engine at another system of the same kind with n_atoms <= the capacity it was
        created with (buffers and cuFFT plans are reused); set_params must follow."""
        d = self._desc(n_atoms, rc, kappa, K, axis_types, axis_indices, cov_rows, mscales, pscales, dscales,
                       solver, cg_tol, max_iter, steps_pol)
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_admp_reconfigure(self.h, ctypes.byref(d)))
        self.n = int(n_atoms)
        self.U, self.forces = self._U_buf[: self.n], self._F_buf[: self.n]

    def __del__(self):
        if getattr(self, "h", None) is not None and self.h.value:
            try:
                self.lib.dmffb_destroy(self.h)
            except Exception:
                pass
            self.h = None

    def _check(self, st, allow=()):
        if st != L.DMFFB_OK and st not in allow:
            raise L.EngineError(st, self.lib.dmffb_last_error(self.h).decode())
        return st

    def set_params(self, Q_local, pol=None, thole=None):
        Q = np.zeros((self.n, 9), dtype=np.float64)
        Qi = np.asarray(Q_local.detach().cpu() if torch.is_tensor(Q_local) else Q_local, dtype=np.float64)
        Q[:, : Qi.shape[1]] = Qi
        Q = np.ascontiguousarray(Q)
        p = t = None
        if pol is not None:
            p = np.ascontiguousarray(np.asarray(pol.detach().cpu() if torch.is_tensor(pol) else pol, np.float64))
            t = np.ascontiguousarray(np.asarray(thole.detach().cpu() if torch.is_tensor(thole) else thole, np.float64))
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_admp_set_params(
                self.h, Q.ctypes.data_as(ctypes.c_void_p), None if p is None else p.ctypes.data_as(ctypes.c_void_p),
                None if t is None else t.ctypes.data_as(ctypes.c_void_p)))

    @staticmethod
    def _box(box):
        b = np.ascontiguousarray(np.asarray(box.detach().cpu() if torch.is_tensor(box) else box, np.float64).reshape(9))
        return b

    def compute(self, pos, box, pairs=None, U=None, forces=None, stream=None):
        """pos: cuda float64 [n,3] (A); box: 3x3 (A); pairs: cuda int32 [np,3] or None (internal list);
        U: cuda float64 [n,3] initial / output induced dipoles (defaults to the engine's buffer).
        Returns (result struct, forces tensor, U tensor); forces = -dE/dpos."""
        assert pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous()
        b = self._box(box)
        if pairs is not None:
            assert pairs.is_cuda and pairs.dtype == torch.int32 and pairs.is_contiguous()
        if U is None:
            U = self.U
        if forces is None:
            forces = self.forces
        res = L.AdmpResult()
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        st = self.lib.dmffb_admp_compute(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos), b.ctypes.data_as(ctypes.c_void_p),
            *_pairs_arg(pairs, self.device), _dev(U) if self.lpol else None, _dev(forces),
            ctypes.byref(res))
        self._check(st, allow=(L.DMFFB_NOT_CONVERGED,))
        return res, forces, U

    def compute_host(self, pos, box, pairs=None, U=None, forces_out=None, U_out=None):
        """Host-buffer entry point: numpy in, numpy out (copies inside the engine).  forces_out /
        U_out: optional caller-owned float64 [n, 3] C-contiguous arrays (pinned memory copies
        fastest) that receive the forces and the dipoles; U, when given, is the initial guess."""
        pos = np.ascontiguousarray(np.asarray(pos, np.float64))
        b = self._box(box)
        pr = None if pairs is None else np.ascontiguousarray(np.asarray(pairs, np.int32))

        def out_array(a):
            if a is None:
                return np.zeros((self.n, 3))
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.shape == (self.n, 3)
                    and a.flags["C_CONTIGUOUS"] and a.flags["WRITEABLE"]):
                raise ValueError("output arrays must be writeable C-contiguous float64 [n, 3]")
            return a

        Uh = out_array(U_out)
        if U is not None:
            Uh[...] = np.asarray(U, np.float64)
        elif U_out is not None and not getattr(self, "_zero_guess", False):
            Uh[...] = 0.0  # the default initial guess (ignored by the engine under set_zero_guess)
        F = out_array(forces_out)
        res = L.AdmpResult()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_admp_compute_host(
                self.h, pos.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p),
                None if pr is None else pr.ctypes.data_as(ctypes.c_void_p), 0 if pr is None else pr.shape[0],
                Uh.ctypes.data_as(ctypes.c_void_p), F.ctypes.data_as(ctypes.c_void_p), ctypes.byref(res))
        self._check(st, allow=(L.DMFFB_NOT_CONVERGED,))
        return res, F, Uh

    def field(self, pos, box, pairs, U):
        out = torch.empty((self.n, 3), dtype=torch.float64, device=self.device)
        b = self._box(box)
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_admp_field(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos), b.ctypes.data_as(ctypes.c_void_p),
            *_pairs_arg(pairs, self.device), _dev(U), _dev(out)))
        return out

    def set_param_grads(self, on=True):
        """Parameter adjoints (dE/dQ, dE/dpol, dE/dthole) on/off for the following computes."""
        self._check(self.lib.dmffb_admp_set_param_grads(self.h, int(bool(on))))

    def set_zero_guess(self, on=True):
        """Dipole solves of the following computes start from U = 0 (the U buffer's content is
        ignored on input and receives the solution); the CG set-up then skips its A U pass."""
        self._check(self.lib.dmffb_admp_set_zero_guess(self.h, int(bool(on))))
        self._zero_guess = bool(on)

    def param_grads(self):
        """{'Q_global', 'Q_local': [n, 9], 'pol', 'thole': [n]} of the last compute."""
        dev = self.device
        out = {"Q_global": torch.empty((self.n, 9), dtype=torch.float64, device=dev),
               "Q_local": torch.empty((self.n, 9), dtype=torch.float64, device=dev),
               "pol": torch.empty(self.n, dtype=torch.float64, device=dev),
               "thole": torch.empty(self.n, dtype=torch.float64, device=dev)}
        s = torch.cuda.current_stream(dev)
        self._check(self.lib.dmffb_admp_param_grads(self.h, ctypes.c_void_p(s.cuda_stream), _dev(out["Q_global"]),
                                                    _dev(out["Q_local"]), _dev(out["pol"]), _dev(out["thole"])))
        return out

    def multipole_grads(self):
        return self.param_grads()["Q_global"]

    def backward(self, c_pos=None, c_box=None, c_Q=None, c_pol=None, c_thole=None):
        """Second-order pass at the last compute (dmffb_admp_backward): the derivatives of
        <c_pos, dE/dpos> + <c_box, dE/dbox> + <c_Q, dE/dQ_local> + <c_pol, dE/dpol> + <c_thole, dE/dthole>
        with respect to positions, box, Q_local [n, 9], pol and thole, the induced dipoles following
        (one adjoint CG solve).  Cotangents: cuda float64 tensors (or None); returns a dict of
        tensors (box: [3, 3] host) plus the adjoint solve's iteration count and the step used."""
        dev = self.device
        n = self.n

        def dv(t, shape):
            if t is None:
                return None
            return t.detach().to(device=dev, dtype=torch.float64).reshape(shape).contiguous()

        cp, cq = dv(c_pos, (n, 3)), dv(c_Q, (n, 9))
        cpo, cth = dv(c_pol, (n,)), dv(c_thole, (n,))
        c = L.AdmpCotangent()
        c.pos = cp.data_ptr() if cp is not None else None
        c.Q_local = cq.data_ptr() if cq is not None else None
        c.pol = cpo.data_ptr() if cpo is not None else None
        c.thole = cth.data_ptr() if cth is not None else None
        if c_box is not None:
            b = np.asarray(c_box.detach().cpu() if torch.is_tensor(c_box) else c_box, np.float64).reshape(9)
            for k in range(9):
                c.box[k] = float(b[k])
        out = {"pos": torch.empty((n, 3), dtype=torch.float64, device=dev),
               "Q_local": torch.empty((n, 9), dtype=torch.float64, device=dev),
               "pol": torch.empty(n, dtype=torch.float64, device=dev),
               "thole": torch.empty(n, dtype=torch.float64, device=dev)}
        o = L.AdmpSecond()
        o.pos, o.Q_local = out["pos"].data_ptr(), out["Q_local"].data_ptr()
        o.pol, o.thole = out["pol"].data_ptr(), out["thole"].data_ptr()
        s = torch.cuda.current_stream(dev)
        self._check(self.lib.dmffb_admp_backward(self.h, ctypes.c_void_p(s.cuda_stream), ctypes.byref(c),
                                                 ctypes.byref(o)))
        out["box"] = torch.tensor(list(o.box), dtype=torch.float64).reshape(3, 3)
        out["n_iter"], out["residual_rms"], out["step"] = int(o.n_iter), float(o.residual_rms), float(o.step)
        return out

    def build_neighbors(self, pos, box, rc, capacity=None):
        """All i<j within rc (FP64 minimum-image test) as a cuda int32 [np,3] tensor sorted by i."""
        b = self._box(box)
        s = torch.cuda.current_stream(self.device)
        need = ctypes.c_int64(0)
        cap = int(capacity) if capacity else 0
        buf = torch.empty((max(cap, 1), 3), dtype=torch.int32, device=self.device)
        st = self.lib.dmffb_build_neighbors(self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos),
                                            b.ctypes.data_as(ctypes.c_void_p), float(rc), _dev(buf), cap,
                                            ctypes.byref(need))
        if st == L.DMFFB_NEIGHBOR_OVERFLOW:
            cap = int(need.value)
            buf = torch.empty((max(cap, 1), 3), dtype=torch.int32, device=self.device)
            st = self.lib.dmffb_build_neighbors(self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos),
                                                b.ctypes.data_as(ctypes.c_void_p), float(rc), _dev(buf), cap,
                                                ctypes.byref(need))
        self._check(st)
        return buf[: need.value]

    def rebuild_internal_pairs(self, pos, box):
        b = self._box(box)
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_admp_build_neighbors(self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos),
                                                        b.ctypes.data_as(ctypes.c_void_p)))

    def internal_pairs(self):
        """The engine's own neighbour list (built by ``rebuild_internal_pairs`` or the first
        compute without pairs) as a cuda int32 [np, 3] tensor, rows sorted by i."""
        s = torch.cuda.current_stream(self.device)
        need = ctypes.c_int64(0)
        self._check(self.lib.dmffb_engine_pairs(self.h, ctypes.c_void_p(s.cuda_stream), None, 0, ctypes.byref(need)),
                    allow=(L.DMFFB_NEIGHBOR_OVERFLOW,))
        buf = torch.empty((max(need.value, 1), 3), dtype=torch.int32, device=self.device)
        self._check(self.lib.dmffb_engine_pairs(self.h, ctypes.c_void_p(s.cuda_stream), _dev(buf), buf.shape[0],
                                                ctypes.byref(need)))
        return buf[: need.value]

    def set_fused_fft(self, on=True):
        """The dipole solve's reciprocal convolution through the engine's own FFT kernels (FP32,
        meshes up to 64 per axis) or through cuFFT (dmffb_set_fused_fft)."""
        self._check(self.lib.dmffb_set_fused_fft(self.h, int(bool(on))))

    def set_persistent_cg(self, mode=True):
        """The whole CG dipole solve in one persistent cooperative launch (FP32, meshes up to 64
        per axis; dmffb_set_persistent_cg): True / 1 always, False / 0 never (the graph-replayed
        per-pass solve), "auto" / 2 (the default) for systems of at most 4096 atoms."""
        m = 2 if mode == "auto" else int(mode)
        self._check(self.lib.dmffb_set_persistent_cg(self.h, m))

    def persistent_cg_blocks(self):
        """Co-resident CTAs of the persistent solve for the current mesh (0: not used)."""
        return int(self.lib.dmffb_persistent_cg_blocks(self.h))

    def set_cg_wait_limit(self, seconds, phantom_arrivals=0):
        """Bound of each grid-barrier wait of the persistent solve; phantom_arrivals > 0 makes the
        next solve's barrier wait for arrivals that never come (it returns DMFFB_TIMEOUT)."""
        self._check(self.lib.dmffb_set_cg_wait_limit(self.h, float(seconds), int(phantom_arrivals)))

    CG_PHASES = ["direction", "matvec_spread", "fft_planes_fwd", "fft_columns", "fft_planes_inv", "gather",
                 "update"]

    def cg_phase_times(self):
        """{pass: ms} of the persistent solves run while profiling was on (device clock, CTA 0)."""
        arr = (ctypes.c_double * 8)()
        self.lib.dmffb_get_cg_phase_times(self.h, arr, 8)
        return {k: arr[i] for i, k in enumerate(self.CG_PHASES)}

    def fused_fft_active(self):
        """Whether the last solve's convolution ran through the engine's FFT (else cuFFT)."""
        return bool(self.lib.dmffb_fused_fft_active(self.h))

    def set_timing(self, on=True):
        self.lib.dmffb_set_timing(self.h, int(on))

    def set_profiling(self, on=True):
        self.lib.dmffb_set_profiling(self.h, int(on))

    def kernel_stats(self):
        """{class: (total ms, launches)} accumulated while profiling was on."""
        n = len(L.KERNEL_CLASSES)
        ms = (ctypes.c_double * n)()
        cnt = (ctypes.c_int64 * n)()
        self.lib.dmffb_get_kernel_stats(self.h, ms, cnt, n)
        return {k: (ms[i], cnt[i]) for i, k in enumerate(L.KERNEL_CLASSES)}

    def counters(self):
        out = (ctypes.c_int64 * 2)()
        self.lib.dmffb_get_counters(self.h, out, 2)
        return {"launches": out[0], "fft_execs": out[1]}

    def timings(self):
        arr = (ctypes.c_double * 6)()
        self.lib.dmffb_get_timings(self.h, arr, 6)
        return list(arr)


class DispEngine:
    """Dispersion PME (C6/C8/C10, dmff/admp/disp_pme.py) with optional Tang-Toennies short range
    (ADMPDispForce, dmff/admp/pairwise.py:100-118) on one GPU."""

    def __init__(self, n_atoms, pmax, lpme, rc, kappa, K, cov_rows, mscales, tt=False, precision="fp32",
                 device=None):
        self.lib = L.load()
        self.n = int(n_atoms)
        self.tt = bool(tt)
        self.mscales = tuple(float(x) for x in mscales)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        d = L.DispDesc()
        d.n_atoms = self.n
        d.pmax = int(pmax)
        d.lpme = int(bool(lpme))
        d.precision = _PREC[precision]
        d.rc = float(rc)
        d.kappa = float(kappa) if lpme else 0.0
        for k in range(3):
            d.K[k] = int(K[k]) if lpme else 0
        cov = _i32(cov_rows if cov_rows is not None else np.zeros((0, 3)), (-1,))
        self._keep = cov
        d.n_cov = cov.size // 3
        d.cov_rows = _ptr(cov)
        for k in range(6):
            d.mscales[k] = self.mscales[k]
        d.tt_damping = int(self.tt)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_disp_create(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if st != L.DMFFB_OK:
            msg = self.lib.dmffb_last_error(h).decode() if h.value else "invalid description"
            if h.value:
                self.lib.dmffb_destroy(h)
            self.h = None
            raise L.EngineError(st, msg)
        self.f_lr = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)
        self.f_sr = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)

    __del__ = AdmpEngine.__del__
    _check = AdmpEngine._check
    _box = staticmethod(AdmpEngine._box)
    rebuild_internal_pairs = AdmpEngine.rebuild_internal_pairs
    build_neighbors = AdmpEngine.build_neighbors
    internal_pairs = AdmpEngine.internal_pairs
    set_profiling = AdmpEngine.set_profiling
    kernel_stats = AdmpEngine.kernel_stats

    def set_params(self, c_list, a=None, b=None, q=None):
        host = lambda x: None if x is None else np.ascontiguousarray(
            np.asarray(x.detach().cpu() if torch.is_tensor(x) else x, np.float64))
        c, a, b, q = host(c_list), host(a), host(b), host(q)
        ptr = lambda x: None if x is None else x.ctypes.data_as(ctypes.c_void_p)
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_disp_set_params(self.h, ptr(c), ptr(a), ptr(b), ptr(q)))

    def compute(self, pos, box, pairs=None):
        """Returns (result, (forces_lr, forces_sr)); forces = -dE/dpos of E_lr and E_sr."""
        assert pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous()
        b = self._box(box)
        res = L.DispResult()
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_disp_compute(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos), b.ctypes.data_as(ctypes.c_void_p),
            *_pairs_arg(pairs, self.device), _dev(self.f_lr), _dev(self.f_sr), ctypes.byref(res)))
        return res, (self.f_lr, self.f_sr)

    def set_param_grads(self, on=True):
        self._check(self.lib.dmffb_disp_set_param_grads(self.h, int(bool(on))))

    def param_grads(self):
        """{'c': dE_lr/dc [n, 3], 'a', 'b', 'q', 'c6': dE_sr/d. [n]} of the last compute."""
        dc = torch.empty(3 * self.n, dtype=torch.float64, device=self.device)
        dsr = torch.empty(4 * self.n, dtype=torch.float64, device=self.device)
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_disp_param_grads(self.h, ctypes.c_void_p(s.cuda_stream), _dev(dc), _dev(dsr)))
        dsr = dsr.reshape(4, self.n)
        return {"c": dc.reshape(3, self.n).T, "a": dsr[0], "b": dsr[1], "q": dsr[2], "c6": dsr[3]}


_COUL = {"none": L.DMFFB_COUL_NONE, "pme": L.DMFFB_COUL_PME, "rf": L.DMFFB_COUL_RF,
         "nocutoff": L.DMFFB_COUL_NOCUTOFF}
_TERM = {"bond": (L.DMFFB_TERM_BOND, 2, 2), "angle": (L.DMFFB_TERM_ANGLE, 3, 2),
         "torsion": (L.DMFFB_TERM_TORSION, 4, 3)}


class ClassicalEngine:
    """Classical terms on one GPU: LJ + point-charge Coulomb (``coulomb`` 'pme' | 'rf' |
    'nocutoff' | 'none'; dmff/classical/inter.py) and harmonic bond / angle / periodic torsion
    term lists (dmff/classical/intra.py).  Units: Angstrom, e, kJ/mol, radians.

    ``n_types`` > 0 enables LJ; ``set_params`` takes per-atom charges and LJ type indices plus
    the type-pair tables sigma_tt / eps_tt (mixing and NBFix applied by the caller)."""

    def __init__(self, n_atoms, n_types=0, coulomb="none", pbc=True, rc=10.0, kappa=0.0, K=(0, 0, 0),
                 cov_rows=None, mscales_coul=(0, 0, 0, 1, 1, 1), mscales_lj=(0, 0, 0, 1, 1, 1),
                 eps_solvent=78.5, precision="fp32", device=None):
        self.lib = L.load()
        self.n = int(n_atoms)
        self.n_types = int(n_types)
        self.coulomb = coulomb
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        d = L.ClassicalDesc()
        d.n_atoms = self.n
        d.n_types = self.n_types
        d.precision = _PREC[precision]
        d.coulomb = _COUL[coulomb]
        d.pbc = int(bool(pbc))
        d.rc = float(rc)
        d.kappa = float(kappa) if coulomb == "pme" else 0.0
        for k in range(3):
            d.K[k] = int(K[k]) if coulomb == "pme" else 0
        d.eps_solvent = float(eps_solvent)
        cov = _i32(cov_rows if cov_rows is not None else np.zeros((0, 3)), (-1,))
        self._keep = cov
        d.n_cov = cov.size // 3
        d.cov_rows = _ptr(cov)
        for k in range(6):
            d.mscales_coul[k] = float(mscales_coul[k])
            d.mscales_lj[k] = float(mscales_lj[k])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_classical_create(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if st != L.DMFFB_OK:
            msg = self.lib.dmffb_last_error(h).decode() if h.value else "invalid description"
            if h.value:
                self.lib.dmffb_destroy(h)
            self.h = None
            raise L.EngineError(st, msg)
        self.forces = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)
        self.n_terms = {"bond": 0, "angle": 0, "torsion": 0}
        self._pgrad = False

    __del__ = AdmpEngine.__del__
    _check = AdmpEngine._check
    _box = staticmethod(AdmpEngine._box)
    rebuild_internal_pairs = AdmpEngine.rebuild_internal_pairs
    build_neighbors = AdmpEngine.build_neighbors
    internal_pairs = AdmpEngine.internal_pairs
    set_profiling = AdmpEngine.set_profiling
    kernel_stats = AdmpEngine.kernel_stats
    counters = AdmpEngine.counters

    @staticmethod
    def _host(x, dtype=np.float64):
        if x is None:
            return None
        x = x.detach().cpu().numpy() if torch.is_tensor(x) else x
        return np.ascontiguousarray(np.asarray(x, dtype=dtype))

    def set_params(self, charges=None, atom_type=None, sigma_tt=None, eps_tt=None):
        q, t = self._host(charges), self._host(atom_type, np.int32)
        sg, ep = self._host(sigma_tt), self._host(eps_tt)
        ptr = lambda x: None if x is None else x.ctypes.data_as(ctypes.c_void_p)
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_classical_set_params(self.h, ptr(q), ptr(t), ptr(sg), ptr(ep)))

    def set_terms(self, kind, idx, prm):
        code, arity, npar = _TERM[kind]
        idx = self._host(idx, np.int32).reshape(-1, arity)
        prm = self._host(prm).reshape(-1, npar)
        assert idx.shape[0] == prm.shape[0]
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_classical_set_terms(self.h, code, idx.shape[0],
                                                           idx.ctypes.data_as(ctypes.c_void_p),
                                                           prm.ctypes.data_as(ctypes.c_void_p)))
        self.n_terms[kind] = idx.shape[0]

    def set_param_grads(self, on=True):
        if bool(on) != self._pgrad:
            self._check(self.lib.dmffb_classical_set_param_grads(self.h, int(bool(on))))
            self._pgrad = bool(on)

    def set_cell_pass(self, on=True):
        """Computes without pairs evaluate every pair within rc straight from the cell grid of the
        positions given (no pair list written); see dmffb_classical_set_cell_pass."""
        self._check(self.lib.dmffb_classical_set_cell_pass(self.h, int(bool(on))))

    def compute(self, pos, box, pairs=None):
        """Returns (result, forces); forces = -dE/dpos (kJ/mol/A), device [n, 3] FP64."""
        assert pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous()
        if pairs is not None:
            assert pairs.is_cuda and pairs.dtype == torch.int32 and pairs.is_contiguous()
        b = self._box(box)
        res = L.ClassicalResult()
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_classical_compute(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos), b.ctypes.data_as(ctypes.c_void_p),
            *_pairs_arg(pairs, self.device), _dev(self.forces), ctypes.byref(res)))
        return res, self.forces

    def param_grads(self):
        """{'q': [n], 'sigma_tt': [T, T], 'eps_tt': [T, T], 'bond'|'angle'|'torsion': [m, 2]} of the last compute."""
        dev = self.device
        T = max(self.n_types, 0)
        out = {"q": torch.empty(self.n, dtype=torch.float64, device=dev),
               "sigma_tt": torch.empty((T, T), dtype=torch.float64, device=dev),
               "eps_tt": torch.empty((T, T), dtype=torch.float64, device=dev)}
        for k in ("bond", "angle", "torsion"):
            out[k] = torch.empty((self.n_terms[k], 2), dtype=torch.float64, device=dev)
        s = torch.cuda.current_stream(dev)
        self._check(self.lib.dmffb_classical_param_grads(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(out["q"]), _dev(out["sigma_tt"]) if T else None,
            _dev(out["eps_tt"]) if T else None, _dev(out["bond"]) if self.n_terms["bond"] else None,
            _dev(out["angle"]) if self.n_terms["angle"] else None,
            _dev(out["torsion"]) if self.n_terms["torsion"] else None))
        return out


class PairwiseEngine:
    """Short-range pairwise term with per-atom parameters on one GPU (dmffb_pairwise_*): the
    built-in kernels of dmff/admp/pairwise.py (``kind`` one of L.DMFFB_SR_*), Angstrom units,
    parameters [nparam, n] in the order of the C header, ``sign`` -1 for the SlaterSr* terms."""

    def __init__(self, n_atoms, kind, rc, cov_rows=None, mscales=(0, 0, 0, 1, 1, 1), sign=1.0, precision="fp32",
                 device=None):
        self.lib = L.load()
        self.n = int(n_atoms)
        self.kind = int(kind)
        self.nparam = L.SR_NPARAM[self.kind]
        self.mscales = tuple(float(x) for x in mscales)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        d = L.PairwiseDesc()
        d.n_atoms, d.kind, d.precision, d.rc = self.n, self.kind, _PREC[precision], float(rc)
        cov = _i32(cov_rows if cov_rows is not None else np.zeros((0, 3)), (-1,))
        self._keep = cov
        d.n_cov = cov.size // 3
        d.cov_rows = _ptr(cov)
        for k in range(6):
            d.mscales[k] = self.mscales[k]
        d.sign = float(sign)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_pairwise_create(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if st != L.DMFFB_OK:
            msg = self.lib.dmffb_last_error(h).decode() if h.value else "invalid description"
            if h.value:
                self.lib.dmffb_destroy(h)
            self.h = None
            raise L.EngineError(st, msg)
        self.forces = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)
        self._pgrad = False

    __del__ = AdmpEngine.__del__
    _check = AdmpEngine._check
    _box = staticmethod(AdmpEngine._box)
    rebuild_internal_pairs = AdmpEngine.rebuild_internal_pairs
    internal_pairs = AdmpEngine.internal_pairs
    set_profiling = AdmpEngine.set_profiling
    kernel_stats = AdmpEngine.kernel_stats

    def set_params(self, params):
        """params: [nparam, n] (array or tensor), Angstrom units."""
        p = params.detach().cpu().numpy() if torch.is_tensor(params) else np.asarray(params)
        p = np.ascontiguousarray(np.asarray(p, dtype=np.float64).reshape(self.nparam, self.n))
        with torch.cuda.device(self.device):
            self._check(self.lib.dmffb_pairwise_set_params(self.h, p.ctypes.data_as(ctypes.c_void_p)))

    def set_param_grads(self, on=True):
        self._check(self.lib.dmffb_pairwise_set_param_grads(self.h, int(bool(on))))
        self._pgrad = bool(on)

    def compute(self, pos, box, pairs=None):
        """Returns (result, forces); forces = -dE/dpos, device [n, 3] FP64."""
        assert pos.is_cuda and pos.dtype == torch.float64 and pos.is_contiguous()
        b = self._box(box)
        res = L.PairwiseResult()
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_pairwise_compute(
            self.h, ctypes.c_void_p(s.cuda_stream), _dev(pos), b.ctypes.data_as(ctypes.c_void_p),
            *_pairs_arg(pairs, self.device), _dev(self.forces), ctypes.byref(res)))
        return res, self.forces

    def param_grads(self):
        """dE/dparameter [nparam, n] of the last compute."""
        out = torch.empty((self.nparam, self.n), dtype=torch.float64, device=self.device)
        s = torch.cuda.current_stream(self.device)
        self._check(self.lib.dmffb_pairwise_param_grads(self.h, ctypes.c_void_p(s.cuda_stream), _dev(out)))
        return out
