"""The host utilities with the reference's names (``dmff_b200.admp.multipole``, ``.admp.spatial``,
``.utils``) against the reference's own known-answer vectors: the parametrised cases of
tests/test_admp/test_multipole.py, test_sptial.py, test_noaxistype.py and tests/test_utils.py,
extracted into tests/golden/kats.json by tests/golden/make_golden.py.  Tolerances as the
reference's tests state them."""
import json
import os

import numpy as np
import torch

from dmff_b200 import utils as U
from dmff_b200.admp import multipole as M
from dmff_b200.admp import spatial as S

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kats.json")))


def test_convert_cart2harm_known_answers():
    for case in KATS["multipole"]["cases"]["test_convert_cart2harm"]:
        Q = M.convert_cart2harm(torch.tensor(case["theta"]), 2)
        np.testing.assert_allclose(Q.numpy(), np.array(case["expected"]), rtol=1e-6)


def test_rotations_known_answers():
    for case in KATS["multipole"]["cases"]["test_rot_global_local"]:
        F = torch.tensor(case["local_frames"], dtype=torch.float64)
        Qg = torch.tensor(case["Q_global"], dtype=torch.float64)
        Ql = torch.tensor(case["Q_local"], dtype=torch.float64)
        np.testing.assert_allclose(M.rot_global2local(Qg, F, 2).numpy(), Ql.numpy(), rtol=1e-4, atol=1e-6)
        np.testing.assert_allclose(M.rot_local2global(Ql, F, 2).numpy(), Qg.numpy(), rtol=1e-4, atol=1e-6)


def test_pair_frames_and_pbc_known_answers():
    for case in KATS["spatial"]["cases"]["test_build_quasi_internal"]:
        out = S.build_quasi_internal(*(torch.tensor(case[k], dtype=torch.float64) for k in ("r1", "r2", "dr", "norm_dr")))
        np.testing.assert_allclose(out.numpy(), np.array(case["expected"]), rtol=1e-5, atol=1e-6)
    for case in KATS["spatial"]["cases"]["test_pbc_shift"]:
        out = S.pbc_shift(*(torch.tensor(case[k], dtype=torch.float64) for k in ("drvecs", "box", "box_inv")))
        np.testing.assert_allclose(out.numpy(), np.array(case["expected"]))


def test_local_frames_known_answers():
    cases = (KATS["spatial"]["cases"]["test_generate_construct_local_frames"]
             + KATS["noaxistype"]["cases"]["test_generate_construct_local_frames"])
    assert cases
    for case in cases:
        f = S.generate_construct_local_frames(np.array(case["axis_types"]), np.array(case["axis_indices"]))
        F = f(np.array(case["positions"]), np.array(case["box"]))
        np.testing.assert_allclose(F.numpy(), np.array(case["expected_local_frames"]), rtol=1e-4, atol=1e-5)


def test_pair_helpers_known_answers():
    k = KATS["utils"]
    np.testing.assert_array_equal(U.regularize_pairs(k["pairs"]).numpy(), np.array(k["regularized"]))
    np.testing.assert_array_equal(U.pair_buffer_scales(k["pairs"]).numpy(), np.array(k["buffer_scales"]))
