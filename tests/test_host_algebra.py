"""Host-side FP64 algebra of the product against the sympy-based oracle."""
import numpy as np
import pytest

from cosmonpc_b200 import angular as A
from oracle import angular as O


def test_wigner3j_matches_sympy():
    for j1, j2, j3 in [(0, 0, 0), (2, 0, 2), (1, 1, 0), (2, 2, 0), (1, 1, 2), (2, 2, 4), (4, 2, 2), (3, 3, 2)]:
        for m1 in range(-j1, j1 + 1):
            for m2 in range(-j2, j2 + 1):
                m3 = -m1 - m2
                if abs(m3) > j3:
                    continue
                assert A.wigner3j(j1, j2, j3, m1, m2, m3) == pytest.approx(
                    O.wigner3j(j1, j2, j3, m1, m2, m3), abs=1e-15)


def test_magnetic_configs_match():
    for cfg in [(0, 0, 0), (2, 0, 2), (1, 1, 0), (2, 2, 0), (1, 1, 2), (2, 2, 4)]:
        a, av = A.magnetic_configs_box(*cfg)
        b, bv = O.magnetic_configs_box(*cfg)
        assert a == b and np.allclose(av, bv, atol=1e-15)
        a, av = A.magnetic_configs_survey(*cfg)
        b, bv = O.magnetic_configs_survey(*cfg)
        assert a == b and np.allclose(av, bv, atol=1e-15)


@pytest.mark.parametrize("racah", [True, False])
def test_harmonics_match_reference_polynomials(racah):
    rng = np.random.default_rng(0)
    v = rng.normal(size=(3, 200))
    v /= np.linalg.norm(v, axis=0)
    z = np.zeros(1)
    for l in range(0, 9):
        for m in range(-l, l + 1):
            got = A.ylm_numpy(l, m, *v, racah=racah)
            ref = O.ylm_function(l, m, racah)(*v)
            assert np.max(np.abs(got - ref)) < 1e-12
            assert A.ylm_origin_value(l, m, racah) == pytest.approx(
                complex(O.ylm_function(l, m, racah)(z, z, z)[0]).real, abs=1e-15)


def test_assoc_legendre_and_q_ells():
    for l in range(0, 5):
        for m in range(-l, l + 1):
            for mu in np.linspace(-0.99, 0.99, 5):
                assert A.assoc_legendre(l, m, mu) == pytest.approx(O.assoc_legendre(l, m, mu), abs=1e-13)
    k_eff = np.array([0.012, 0.021, 0.033, 0.041])
    k3 = np.linspace(0.02, 0.09, 7)
    for cfg in [(0, 0, 0), (2, 0, 2), (1, 1, 2), (2, 2, 0)]:
        for i in range(4):
            for j in range(4):
                np.testing.assert_allclose(A.q_ells_eff(i, j, k_eff, *cfg, k3),
                                           O.q_ells_eff(i, j, k_eff, *cfg, k3), atol=1e-13)


def test_pair_assembly_matches_complex_brute_force():
    """S_ij from real component Grams equals sum G F1 F2 on complex fields."""
    from cosmonpc_b200 import engine

    rng = np.random.default_rng(1)
    nb, ncell = 3, 50
    G = rng.normal(size=ncell)
    F1 = rng.normal(size=(nb, ncell)) + 1j * rng.normal(size=(nb, ncell))
    F2 = rng.normal(size=(nb, ncell)) + 1j * rng.normal(size=(nb, ncell))

    class SF:
        def key(self, leg, b, c):
            return (tuple(leg), b, c)

    sf = SF()
    legs = {(1, 1, 0, False): F1, (2, -1, 0, False): F2}
    comp = {0: np.real, 1: np.imag}
    for mode in ("leg", "eq", "conj"):
        ps = engine.PairSpec((1, 1, 0, False), mode, (2, -1, 0, False) if mode == "leg" else None, sign=-1.0)
        rows = ps.row_keys(sf, range(nb))
        cols = ps.col_keys(sf, range(nb))
        val = lambda k: comp[k[2]](legs[k[0]][k[1]])
        T = np.array([[np.sum(G * val(r) * val(c)) for c in cols] for r in rows])
        S = engine.assemble(ps, T, rows, cols, list(range(nb)), list(range(nb)))
        F2m = {"leg": F2, "eq": F1, "conj": -np.conj(F1)}[mode]
        ref = np.array([[np.sum(G * F1[i] * F2m[j]) for j in range(nb)] for i in range(nb)])
        np.testing.assert_allclose(S, ref, atol=1e-12)


def test_vectorised_q_matches_oracle():
    k_eff = np.array([0.012, 0.021, 0.033, 0.041, np.nan])
    k3 = np.linspace(0.02, 0.09, 9)
    for cfg in [(0, 0, 0), (2, 0, 2), (1, 1, 2), (2, 2, 0), (1, 1, 0)]:
        Q = A.q_ells_matrix(k_eff, *cfg, k3)
        for i in range(4):
            for j in range(4):
                np.testing.assert_allclose(Q[i, j], O.q_ells_eff(i, j, k_eff, *cfg, k3), atol=1e-13)
        assert np.all(Q[4] == 0) and np.all(Q[:, 4] == 0)


@pytest.mark.parametrize("mode,leg1,leg2,sign", [("leg", (2, 1, 0, False), (0, 0, 1, False), 1.0),
                                                 ("eq", (2, -2, 0, False), None, 1.0),
                                                 ("conj", (1, 1, 0, True), None, -1.0),
                                                 ("conj", (2, 0, 0, False), None, 1.0)])
def test_gram_block_assembly_matches_entrywise(mode, leg1, leg2, sign):
    """The index-array assembly of a Gram block equals the per-entry rule,
    with components missing from the block reading as zero."""
    from cosmonpc_b200 import engine

    class SF:
        def key(self, leg, b, comp):
            return (tuple(leg), int(b), int(comp))

    sf = SF()
    ps = engine.PairSpec(leg1, mode, leg2, sign)
    rbins, cbins = [1, 2, 4], [0, 2, 3, 5]
    rows = list(dict.fromkeys(ps.row_keys(sf, rbins)))[:-1]  # one row component absent
    cols = list(dict.fromkeys(ps.col_keys(sf, cbins)))
    rng = np.random.default_rng(5)
    T = rng.standard_normal((len(rows), len(cols)))
    S = engine.assemble(ps, T, rows, cols, rbins, cbins)
    ri = {k: i for i, k in enumerate(rows)}
    ci = {k: j for j, k in enumerate(cols)}
    t = lambda k1, k2: T[ri[k1], ci[k2]] if k1 in ri and k2 in ci else 0.0
    ref = np.array([[engine._assemble_entry(ps, t, a, c) for c in cbins] for a in rbins])
    np.testing.assert_array_equal(S, ref)


def test_launch_groups_merge_same_columns_within_staging_limit():
    """FP32 weight groups with identical columns share a launch while the
    staged rows (weights + padded rows + padded columns unless shared) fit."""
    from cosmonpc_b200 import engine

    class SF:
        precision = "f32"

        def __init__(self):
            self.slot = {}

        def key(self, leg, b, comp):
            k = (tuple(leg), int(b), int(comp))
            self.slot.setdefault(k, len(self.slot))
            return k

    sf = SF()
    u0 = [sf.key((0, 0, 2, True), b, 0) for b in range(20)]
    u2 = [sf.key((2, 0, 2, True), b, 0) for b in range(20)]
    other = [sf.key((4, 0, 2, True), b, 0) for b in range(20)]
    # (000) rows u0, (202) rows u2, both against columns u0: merged, columns shared
    assert engine._launch_groups(sf, [u0, u2], [u0, u0]) == [[0, 1]]
    # different columns: separate launches
    assert engine._launch_groups(sf, [u0, u2], [u0, u2]) == [[0], [1]]
    # 2 weights + 40 rows + 20 unshared columns > 48 staged rows: separate
    assert engine._launch_groups(sf, [u2, other], [u0, u0]) == [[0], [1]]
    sf.precision = "f64"
    assert engine._launch_groups(sf, [u0, u2], [u0, u0]) == [[0], [1]]


def test_lognormal_box_exact_count():
    from cosmonpc_b200.mocks import lognormal_box_exact

    for n in (1000, 4321):
        pos = lognormal_box_exact(n, 500.0, 3)
        assert pos.shape == (n, 3)
        assert pos.min() >= 0.0 and pos.max() < 500.0
