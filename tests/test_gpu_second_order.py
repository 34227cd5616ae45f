"""Second-order derivatives on the GPU: gradients of losses on forces and on the virial with respect
to parameters and positions, the induced dipoles following their parameters through one adjoint
CG solve (dmffb_admp_backward).  The reference's jax.grad stops gradients at the dipole solve
(dmff/admp/pme.py:212-213, 363-371), so it cannot serve as the oracle here: the exact reference is
the float64 oracle differentiated implicitly (tests/helpers.py:oracle_force_loss_grads, itself
pinned against finite differences on the CPU), and central finite differences of the loss with the
dipoles re-solved.  The consumer pattern is a force-matching fit (dmff/optimize.py:30-84)."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import disp_params, water_box, workload
from tests.helpers import make_engine, oracle_force_loss_grads, oracle_pairs

pytestmark = pytest.mark.gpu


def _relmax(got, want):
    got, want = np.asarray(got), np.asarray(want)
    return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


@pytest.fixture(scope="module")
def small():
    s = water_box(27, 9.3, seed=24, lmax=2, pol=True, rc=4.6)
    pr = oracle_pairs(s)
    w = np.random.default_rng(5).normal(size=(s["n_atoms"], 3))
    return s, pr, w, oracle_force_loss_grads(s, pr, w)


def test_engine_backward_matches_exact_oracle(small):
    """The C-ABI pass (FP64 engine) against the oracle's implicit second derivatives."""
    s, pr, w, ex = small
    eng = make_engine(s, precision="fp64", cg_tol=1e-12)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    pairs = torch.tensor(pr, dtype=torch.int32, device="cuda")
    res, F, U = eng.compute(pos, s["box"], pairs=pairs)
    assert res.converged == 1
    out = eng.backward(c_pos=torch.tensor(w, device="cuda"))
    assert out["n_iter"] > 0 and out["step"] > 0
    assert _relmax(out["pos"].cpu().numpy(), ex["pos"]) < 1e-6
    assert _relmax(out["Q_local"].cpu().numpy(), ex["Q"]) < 1e-6
    assert _relmax(out["pol"].cpu().numpy(), ex["pol"]) < 1e-6
    assert _relmax(out["thole"].cpu().numpy(), ex["thole"]) < 1e-5
    # the pass leaves the engine's state as it found it: the same compute gives the same result
    res2, F2, _ = eng.compute(pos, s["box"], pairs=pairs, U=U.clone())
    assert abs(res2.energy - res.energy) <= 1e-12 * abs(res.energy)


def _dropin(s, precision):
    from dmff_b200.admp.pme import ADMPPmeForce
    return ADMPPmeForce(s["box"], s["types"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], 2, True, True,
                        cov_rows=s["cov_rows"], precision=precision, cg_tol=1e-12 if precision == "fp64" else 1e-6,
                        max_iter=2000)


def _force_loss_grads(f, s, pr, w, wbox, Qt, pt, tt, create_graph=True):
    """L = <w, forces> + <wbox, dE/dbox> through autograd (double backward through the engine)."""
    types = torch.as_tensor(s["types"])
    ms, ps, ds = (torch.tensor(s[k]) for k in ("mscales", "pscales", "dscales"))
    pos = torch.tensor(s["pos"], requires_grad=True)
    box = torch.tensor(s["box"], requires_grad=True)
    E = f.get_energy(pos, box, pr, Qt[types], pt[types], tt[types], ms, ps, ds, U_init=torch.zeros((s["n_atoms"], 3)))
    gpos, gbox = torch.autograd.grad(E, (pos, box), create_graph=create_graph)
    L = (torch.as_tensor(w) * -gpos).sum() + (torch.as_tensor(wbox) * gbox).sum()
    return L, pos


def _fd_check(s, pr, w, wbox, grads, cases, rtol):
    """central differences (h = 1e-5) of the same loss on the FP64 drop-in path, dipoles re-solved"""
    f64 = _dropin(s, "fp64")
    h = 1e-5
    for k, idx in cases:
        vals = []
        for sgn in (1.0, -1.0):
            args = [torch.tensor(s["Q_type"]), torch.tensor([1.0, 0.5], dtype=torch.float64),
                    torch.tensor([0.33, 0.33], dtype=torch.float64)]
            args[k][idx] += sgn * h
            with torch.enable_grad():
                L, _ = _force_loss_grads(f64, s, pr, w, wbox, *args, create_graph=False)
            vals.append(float(L))
        fd = (vals[0] - vals[1]) / (2 * h)
        got = float(grads[k][idx])
        assert abs(got - fd) <= rtol * max(abs(fd), 1e-3 * np.abs(grads[k]).max()), (k, idx, got, fd)


@pytest.mark.parametrize("precision,rtol", [("fp64", 1e-5), ("fp32", 1e-4)])
def test_force_matching_gradients_vs_finite_differences(precision, rtol):
    """Per-type gradients of a loss on forces and on the box gradient through the drop-in API with
    create_graph=True, against central differences of the same loss."""
    s = water_box(27, 9.3, seed=24, lmax=2, pol=True, rc=4.6)
    pr = oracle_pairs(s)
    rng = np.random.default_rng(7)
    w, wbox = rng.normal(size=(s["n_atoms"], 3)), rng.normal(size=(3, 3)) * 0.1
    f = _dropin(s, precision)
    Qt = torch.tensor(s["Q_type"], requires_grad=True)
    pt = torch.tensor([1.0, 0.5], dtype=torch.float64, requires_grad=True)
    tt = torch.tensor([0.33, 0.33], dtype=torch.float64, requires_grad=True)
    L, _ = _force_loss_grads(f, s, pr, w, wbox, Qt, pt, tt)
    grads = [g.detach().numpy() for g in torch.autograd.grad(L, (Qt, pt, tt))]
    assert f.last_second_order["n_iter"] > 0
    _fd_check(s, pr, w, wbox, grads, [(0, (0, 0)), (0, (0, 1)), (0, (1, 4)), (1, (0,)), (1, (1,)), (2, (0,))], rtol)


def test_position_hessian_vector_product_vs_finite_differences(small):
    """d/dpos of <w, forces>: the Hessian of the reduced energy along w, against central
    differences of the forces with the dipoles re-solved."""
    s, pr, w, ex = small
    f = _dropin(s, "fp64")
    Qt = torch.tensor(s["Q_type"])
    pt, tt = torch.tensor([1.0, 0.5], dtype=torch.float64), torch.tensor([0.33, 0.33], dtype=torch.float64)
    L, pos = _force_loss_grads(f, s, pr, w, np.zeros((3, 3)), Qt, pt, tt)
    (gpos,) = torch.autograd.grad(L, pos)
    # the exact oracle gives d<w, dE/dpos>/dpos = -d<w, forces>/dpos
    assert _relmax(-gpos.numpy(), ex["pos"]) < 1e-6


def test_fp32_second_order_at_c2_size():
    """The differentiation workload's size (6144 atoms): gradient of a force-matching loss with
    respect to per-type multipoles and polarizabilities through the FP32 drop-in path (second order
    on an FP64 engine of the same system) against central differences of the FP64 loss."""
    s = workload("c2")
    pr = oracle_pairs(s)
    rng = np.random.default_rng(8)
    w = rng.normal(size=(s["n_atoms"], 3))
    f = _dropin(s, "fp32")
    Qt = torch.tensor(s["Q_type"], requires_grad=True)
    pt = torch.tensor([1.0, 0.5], dtype=torch.float64, requires_grad=True)
    tt = torch.tensor([0.33, 0.33], dtype=torch.float64, requires_grad=True)
    L, _ = _force_loss_grads(f, s, pr, w, np.zeros((3, 3)), Qt, pt, tt)
    grads = [g.detach().numpy() for g in torch.autograd.grad(L, (Qt, pt, tt))]
    _fd_check(s, pr, w, np.zeros((3, 3)), grads, [(0, (0, 0)), (0, (1, 1)), (1, (0,)), (1, (1,))], 1e-4)


def test_dispersion_force_loss_gradients_vs_finite_differences():
    """Dispersion PME + Tang-Toennies (ADMPDispPmeForce with the fused TT term): the gradient of a
    loss on forces with respect to the per-atom C6/C8/C10 (through c = sqrt(C 10^n)) and the TT A
    parameters, against central differences of the FP64 loss."""
    from dmff_b200.admp.disp_pme import ADMPDispPmeForce
    s = water_box(64, 12.4, seed=21, lmax=2, pol=False, rc=6.0)
    d = disp_params(64, seed=2)
    pr = oracle_pairs(s)
    w = np.random.default_rng(9).normal(size=(s["n_atoms"], 3))

    def loss(precision, c, a, create_graph):
        f = ADMPDispPmeForce(s["box"], s["rc"], s["ethresh"], 10, cov_rows=s["cov_rows"], tt_damping=True,
                             precision=precision)
        pos = torch.tensor(s["pos"], requires_grad=True)
        E = f.get_energy(pos, torch.tensor(s["box"]), pr, c, torch.tensor(d["mscales"]),
                         tt=(a, torch.tensor(d["b"]), torch.tensor(d["q"])))
        (g,) = torch.autograd.grad(E, pos, create_graph=create_graph)
        return (torch.as_tensor(w) * -g).sum()

    for precision, rtol in (("fp64", 1e-5), ("fp32", 1e-4)):
        c = torch.tensor(d["c_list"], requires_grad=True)
        a = torch.tensor(d["a"], requires_grad=True)
        gc, ga = (t.detach().numpy() for t in torch.autograd.grad(loss(precision, c, a, True), (c, a)))
        h = 1e-5
        for grad, idx, which in ((gc, (0, 0), 0), (gc, (4, 2), 0), (ga, (3,), 1)):
            vals = []
            for sgn in (1.0, -1.0):
                cc, aa = torch.tensor(d["c_list"]), torch.tensor(d["a"])
                (cc if which == 0 else aa)[idx] += sgn * h
                vals.append(float(loss("fp64", cc, aa, False)))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(grad[idx] - fd) <= rtol * max(abs(fd), 1e-3 * np.abs(grad).max()), (precision, idx, grad[idx], fd)
