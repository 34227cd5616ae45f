"""The float64 oracle gives the same energy whatever the host's thread count, and the recorded value
of the fixture the GPU parity tests pin it with."""
import torch

from dmff_b200.synthetic import water_box
from tests.helpers import oracle_pairs, oracle_reference

C0_SMALL_ORACLE_E = -398.00509400279407


def test_oracle_energy_is_independent_of_thread_count():
    s = water_box(64, 12.4, seed=10, lmax=2, pol=False, rc=6.0)
    pr = oracle_pairs(s)
    n0 = torch.get_num_threads()
    try:
        vals = []
        for nt in (1, 3, max(n0, 2)):
            torch.set_num_threads(nt)
            vals.append(oracle_reference(s, pr, want_box=False)["E"])
    finally:
        torch.set_num_threads(n0)
    assert vals[0] == vals[1] == vals[2]
    assert abs(vals[0] - C0_SMALL_ORACLE_E) <= 1e-12 * abs(C0_SMALL_ORACLE_E)
