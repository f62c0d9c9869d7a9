"""The seeded synthetic workloads on the CPU: the generator's stated
distributions and symmetry, irrep consistency of the 8-irrep systems, the
64-system batch's ranges, and reproducibility (the benchmark's inputs are a
function of the seed alone)."""
import numpy as np

from acesb200.workloads import WORKLOADS, batch_systems, synthetic_df


def test_generator_distributions_and_symmetry():
    eps, B, irr = synthetic_df(6, 30, 40, seed=5)
    o = 6
    assert np.all((eps[:o] >= -1.5) & (eps[:o] <= -0.3)) and np.all(np.diff(eps[:o]) >= 0)
    assert np.all((eps[o:] >= 0.2) & (eps[o:] <= 3.0)) and np.all(np.diff(eps[o:]) >= 0)
    np.testing.assert_array_equal(B, B.transpose(0, 2, 1))
    # B = (X + X^T)/2 with X ~ N(0, 0.02^2): off-diagonal std 0.02/sqrt(2)
    off = B[:, ~np.eye(36, dtype=bool)]
    assert abs(off.std() / (0.02 / np.sqrt(2)) - 1) < 0.05
    assert np.all(irr == 0)
    eps2, B2, _ = synthetic_df(6, 30, 40, seed=5, bscale=0.25)
    np.testing.assert_array_equal(eps2, eps)
    np.testing.assert_allclose(B2, 0.25 * B, rtol=0, atol=0)


def test_irrep_blocked_integrals_are_symmetry_consistent():
    eps, B, irr = synthetic_df(8, 40, 60, seed=1004, irreps=8)
    o = 8
    # DPD order: occupied, then virtual, each sorted by irrep
    assert np.all(np.diff(irr[:o]) >= 0) and np.all(np.diff(irr[o:]) >= 0)
    # (pq|rs) vanishes unless irrep(p)^irrep(q)^irrep(r)^irrep(s) == 0
    g = np.einsum("Lpq,Lrs->pqrs", B, B)
    sym = (irr[:, None, None, None] ^ irr[None, :, None, None] ^ irr[None, None, :, None]
           ^ irr[None, None, None, :]) != 0
    assert np.abs(g[sym]).max() == 0.0
    assert np.abs(g[~sym]).max() > 0.0


def test_batch_systems_ranges_and_reproducibility():
    systems = batch_systems()
    assert len(systems) == 64
    for k, s in enumerate(systems):
        assert 4 <= s["nocc"] <= 24 and 30 <= s["nvir"] <= 220
        assert s["irreps"] == 8 and s["seed"] == 1000 + k
    assert batch_systems() == systems
    # the named workloads keep their published shapes
    assert (WORKLOADS["c2"]["nocc"], WORKLOADS["c2"]["nvir"], WORKLOADS["c2"]["naux"]) == (20, 180, 600)
    assert (WORKLOADS["c3"]["nocc"], WORKLOADS["c3"]["nvir"], WORKLOADS["c3"]["naux"]) == (30, 270, 900)
    a = synthetic_df(**WORKLOADS["c2conv"])
    b = synthetic_df(**WORKLOADS["c2conv"])
    np.testing.assert_array_equal(a[1][:5, :10, :10], b[1][:5, :10, :10])
