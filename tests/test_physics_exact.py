"""The exact 2D Ising anchors (Kaufman's finite-torus partition function)
checked against brute-force enumeration, so the GPU physics tests compare
against numbers that are themselves verified."""
import math

import pytest

from tests.exact_ising import brute_force, energy_per_site, log_z


@pytest.mark.parametrize("m,n", [(4, 4), (4, 2), (2, 4)])
@pytest.mark.parametrize("beta", [0.1, 0.3, 0.4406868, 0.6, 1.0])
def test_kaufman_equals_enumeration(m, n, beta):
    lz, e = brute_force(beta, m, n)
    assert abs(log_z(beta, m, n) - lz) < 1e-9 * max(1.0, abs(lz))
    assert abs(energy_per_site(beta, m, n) - e) < 1e-7


def test_infinite_lattice_limit_at_criticality():
    # E/N -> -sqrt(2) at beta_c as L grows (Onsager)
    bc = 0.5 * math.log(1 + math.sqrt(2))
    assert abs(energy_per_site(bc, 512, 512) + math.sqrt(2)) < 2e-3
