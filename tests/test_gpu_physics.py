"""Physics checks of the move kernel that bit-parity with the oracle cannot
give: without a field (chiN = kappaN = 0) a chain with harmonic bonds
k |r_i - r_j|^2 is an ideal Gaussian chain, so every bond vector component has
variance 1 / (2k), <|b|^2> = 3 / (2k) and <R_e^2> = (N - 1) <|b|^2>.  Started
far from that (a bond length of a third of the equilibrium one), the smart-MC
moves with their Metropolis correction must relax to it and stay there; a
wrong acceptance formula breaks detailed balance and shifts the averages."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import new_arch_b200
    return new_arch_b200


@pytest.mark.parametrize("smc_a", [0.02, 0.1])
def test_ideal_chain_bond_statistics(nb, smc_a):
    from new_arch_b200.spec import diblock_melt
    n = 16
    spec = diblock_melt(8000, n, 0.5, (16, 16, 16), 0.0, 0.0, seed=123, smc_a=smc_a)
    spec.archs[0].init_sigma = 0.7 / np.sqrt(3.0) / 3.0      # start far from equilibrium
    k = spec.harmonic_normb
    b2_eq = 3.0 / (2.0 * k)
    with nb.System(spec) as s:
        s.init_coords()
        start = s.analyze()[0]["bond2"][3]
        assert start < 0.3 * b2_eq
        s.step(1500)                                          # relax
        samples = []
        for _ in range(40):
            s.step(25)
            o = s.analyze()[0]
            samples.append((o["bond2"][:3], o["re2"][3]))
        st = s.stats()
    bond2 = np.array([x[0] for x in samples])                 # per-component means, per sample
    re2 = np.array([x[1] for x in samples])
    acc = st["total_accepts"] / st["total_moves"]
    assert 0.05 < acc < 0.999
    # 8000 chains x 15 bonds per sample: per-sample noise of a mean is ~0.5 %
    np.testing.assert_allclose(bond2.mean(axis=0), [b2_eq / 3] * 3, rtol=0.01)
    np.testing.assert_allclose(re2.mean(), (n - 1) * b2_eq, rtol=0.03)
