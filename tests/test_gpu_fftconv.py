"""The dipole solve's reciprocal convolution through the engine's own FFT kernels (x-plane
forward pass, spectrum columns with the influence multiply, x-plane inverse pass) against the
cuFFT path of the same engine, on 7-smooth meshes (engine FFT) and prime ones (which keep cuFFT),
and on a small box against the oracle."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import serving_system, water_box
from tests.helpers import make_engine, oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu


def _solve(eng, s, fused):
    eng.set_persistent_cg(False)  # the per-pass solve: cuFFT or the engine FFT kernels
    eng.set_fused_fft(fused)
    eng.set_zero_guess(True)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.rebuild_internal_pairs(pos, s["box"])
    res, F, U = eng.compute(pos, s["box"])
    torch.cuda.synchronize()
    return res, F.cpu().numpy().copy(), U.cpu().numpy().copy(), eng.fused_fft_active()


@pytest.mark.parametrize("n_waters", [150, 300, 700, 2300, 3900, 9000])
def test_fused_convolution_matches_cufft(n_waters):
    """Serving-stream boxes: meshes 17^3 (prime), 21^3, 28^3, 41^3 (prime), 50^3 and beyond."""
    s = serving_system(n_waters, 500 + n_waters)
    eng = make_engine(s, precision="fp32", cg_tol=1e-7)
    r0, F0, U0, cl0 = _solve(eng, s, False)
    r1, F1, U1, cl1 = _solve(eng, s, True)
    assert not cl0
    assert cl1 == (max(s["K"]) <= 64), (s["K"], cl1)
    assert abs(r1.energy - r0.energy) <= 2e-6 * abs(r0.energy), (s["K"], r1.energy, r0.energy)
    assert rel_force_rms(F1, F0) < 1e-5
    assert np.abs(U1 - U0).max() <= 1e-5 * np.abs(U0).max()
    assert abs(r1.n_iter - r0.n_iter) <= 4


def test_fused_convolution_small_box_matches_oracle():
    """A 64-water box (mesh 18^3 at rc 6 A) through the fused path against the float64 oracle."""
    s = water_box(64, 13.0, seed=61, lmax=2, pol=True, rc=6.0)
    assert s["K"] == (18, 18, 18)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr, solver="cg", tol=1e-9)
    eng = make_engine(s, precision="fp32", cg_tol=1e-7)
    res, F, U, cl = _solve(eng, s, True)
    assert cl
    assert abs(res.energy - ref["E"]) <= 1e-5 * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= 1e-4
    assert np.abs(U - ref["U"]).max() <= 1e-4 * np.abs(ref["U"]).max()
