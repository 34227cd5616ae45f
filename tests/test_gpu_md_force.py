"""The MD-platform force (dmffb_md_force_*) on the GPU, in OpenMM's CUDA layout: positions gathered
from a posq array in a permuted atom order (nm), forces added to a fixed-point force buffer
(kJ/mol/nm * 2^32, [3][padded]), the induced dipoles kept on the device across steps.  Checked
against dmffb_admp_compute_host on the same positions (the path the reference's plugin takes
through the host, backend/openmm_dmff_plugin/platforms/cuda/src/CudaDMFFKernels.cpp:118-220)."""
import ctypes

import numpy as np
import pytest
import torch

from dmff_b200 import _lib as L
from dmff_b200.synthetic import water_box
from tests.helpers import make_engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("posq_double", [True, False])
def test_md_force_matches_host_entry(posq_double):
    lib = L.load()
    dev = torch.device("cuda", 0)
    s = water_box(216, 18.6, seed=51, lmax=2, pol=True, rc=6.0)
    n, padded = s["n_atoms"], s["n_atoms"] + 29
    ref_eng = make_engine(s, precision="fp32", cg_tol=1e-8)
    d, keep = _desc(s)
    Q = np.ascontiguousarray(s["Q_local"], dtype=np.float64)
    pol = np.ascontiguousarray(s["pol"], dtype=np.float64)
    th = np.ascontiguousarray(s["thole"], dtype=np.float64)
    h = ctypes.c_void_p()
    with torch.cuda.device(dev):
        assert lib.dmffb_md_force_create(ctypes.byref(d), Q.ctypes.data, pol.ctypes.data, th.ctypes.data,
                                         ctypes.byref(h)) == 0
    rng = np.random.default_rng(3)
    perm = rng.permutation(n).astype(np.int32)  # slot -> system atom
    stream = torch.cuda.current_stream(dev)
    try:
        pos = s["pos"].copy()
        iters = []
        for step in range(3):
            dt = torch.float64 if posq_double else torch.float32
            posq = torch.zeros((padded, 4), dtype=dt, device=dev)
            posq[:n, :3] = torch.tensor(pos[perm] / 10.0, dtype=dt, device=dev)  # nm, platform order
            fbuf = torch.zeros(3 * padded, dtype=torch.int64, device=dev)
            idx = torch.tensor(perm, device=dev)
            c = L.MdContext()
            c.posq, c.posq_double = posq.data_ptr(), int(posq_double)
            c.force_buffer, c.atom_index = fbuf.data_ptr(), idx.data_ptr()
            c.num_atoms, c.padded_num_atoms = n, padded
            for k, v in enumerate((s["box"] / 10.0).reshape(9)):
                c.box_nm[k] = float(v)
            c.stream = stream.cuda_stream
            e = ctypes.c_double(0.0)
            st = lib.dmffb_md_force_execute(h, ctypes.byref(c), 1, ctypes.byref(e))
            assert st == 0
            torch.cuda.synchronize()
            res = L.AdmpResult()
            assert lib.dmffb_md_force_last_result(h, ctypes.byref(res)) == 0
            iters.append(res.n_iter)
            # decode the fixed-point buffer (slot order, kJ/mol/nm) back to system order in kJ/mol/A
            fb = fbuf.cpu().numpy().reshape(3, padded)[:, :n].T / 2.0 ** 32
            F = np.zeros((n, 3))
            F[perm] = fb / 10.0
            assert np.all(fbuf.cpu().numpy().reshape(3, padded)[:, n:] == 0)
            # the host-buffer entry on the positions the platform held
            p_used = posq[:n, :3].double().cpu().numpy() * 10.0
            p_sys = np.zeros_like(p_used)
            p_sys[perm] = p_used
            r2, F2, _ = ref_eng.compute_host(p_sys, s["box"])
            assert abs(e.value - r2.energy) <= 1e-6 * abs(r2.energy)
            rms = np.sqrt(np.mean((F - F2) ** 2)) / np.sqrt(np.mean(F2 ** 2))
            assert rms < 1e-5
            pos = pos + rng.normal(0.0, 0.01, size=pos.shape)  # a small MD-like move
        # the dipoles carried over: later steps start from the previous solution
        assert min(iters[1:]) < iters[0]
        U = torch.empty((n, 3), dtype=torch.float64, device=dev)
        assert lib.dmffb_md_force_dipoles(h, ctypes.c_void_p(stream.cuda_stream), ctypes.c_void_p(U.data_ptr())) == 0
        torch.cuda.synchronize()
        assert float(U.abs().max()) > 0
    finally:
        lib.dmffb_md_force_destroy(h)


def _desc(s):
    """dmffb_admp_desc of a polarizable FP32 water box (the arrays it points at are returned too)."""
    d = L.AdmpDesc()
    d.n_atoms = s["n_atoms"]
    d.lmax, d.lpol, d.lpme, d.precision = 2, 1, 1, L.DMFFB_FP32
    d.rc, d.kappa = float(s["rc"]), float(s["kappa"])
    for k in range(3):
        d.K[k] = int(s["K"][k])
    at = np.ascontiguousarray(s["axis_types"], dtype=np.int32)
    ai = np.ascontiguousarray(s["axis_indices"], dtype=np.int32).reshape(-1)
    cov = np.ascontiguousarray(s["cov_rows"], dtype=np.int32).reshape(-1)
    d.axis_types = at.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    d.axis_indices = ai.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    d.n_cov = cov.size // 3
    d.cov_rows = cov.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    for k in range(6):
        d.mscales[k], d.pscales[k], d.dscales[k] = s["mscales"][k], s["pscales"][k], s["dscales"][k]
    d.solver, d.cg_tol, d.max_iter, d.steps_pol = L.DMFFB_SOLVER_CG, 1e-8, 500, 0
    return d, (at, ai, cov)
