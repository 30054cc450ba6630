"""TBTK's JSON serialization of the path's results (tbtk_b200/export.py).

Pinned three ways: against the reference's own serialize() text committed in
tests/golden/export.npz (made by tests/golden/make_golden.py from the
compiled reference), with the oracle's results in place of the reference's
(the oracle equals the reference bit for bit, so the text must too), and,
where the reference subset is built, by TBTK's deserializing constructors
reading the exported text and writing it back unchanged.

The reference leaves defaultValue of LDOS and Density uninitialised, so its
text carries arbitrary bits there; comparisons set that one field to the
"0" this library writes.
"""
import re

import numpy as np
import pytest
from conftest import golden

from tbtk_b200 import export as X
from tbtk_b200 import lattice as L

DEFAULT = re.compile(r'"defaultValue":"[^"]*"')


def _ref_text(t):
    return DEFAULT.sub('"defaultValue":"0"', str(t))


def _tuples(a):
    return [tuple(int(v) for v in row) for row in a]


def _window(g, key="window"):
    lo, hi, res = g[key]
    return float(lo), float(hi), int(res)


def test_ldos_text_equals_reference():
    g = golden("export")
    lo, hi, _ = _window(g)
    assert X.ldos_json(_tuples(g["ldos_sites"]), g["ldos"], lo, hi) == _ref_text(g["ldos_text"])
    lo, hi, _ = _window(g, "hc_window")
    assert X.ldos_json(_tuples(g["hc_sites"]), g["hc_ldos"], lo, hi) == _ref_text(g["hc_text"])


def test_greens_function_text_equals_reference():
    g = golden("export")
    lo, hi, _ = _window(g)
    for ty in (1, 3):
        got = X.greens_function_json(_tuples(g["gf_to"]), tuple(g["gf_from"]), g[f"gf_{ty}"],
                                     lo, hi)
        assert got == str(g[f"gf_text_{ty}"])


def test_density_text_equals_reference():
    g = golden("export")
    got = X.density_json(_tuples(g["density_sites"]), g["density"])
    assert got == _ref_text(g["density_text"])


def test_oracle_results_export_as_reference(oracle):
    """The LDOS and Green's functions of the oracle (the restatement the CUDA
    path is checked against bit for bit) give the reference's text."""
    g = golden("export")
    lo, hi, res = _window(g)
    lat = L.square(6, 5, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    rowptr, col, val = lat.csr()
    s, M, bro = 8.0, 256, 1e-3
    table = oracle.lookup_table(M, oracle.range(lo, hi, res), s)

    def damped(frm, to):
        return oracle.damp(oracle.moments(rowptr, col, val, s, M, frm, to), bro)

    sites = _tuples(g["ldos_sites"])
    ldos = np.array([oracle.ldos_table(table, damped(lat.basis(x), [lat.basis(x)])[0])
                     for x in sites])
    assert X.ldos_json(sites, ldos, lo, hi) == _ref_text(g["ldos_text"])
    to, frm = _tuples(g["gf_to"]), tuple(int(v) for v in g["gf_from"])
    mu = damped(lat.basis(frm), [lat.basis(t) for t in to])
    gf = np.array([oracle.greens_table(table, 1, mu[k]) for k in range(len(to))])
    assert X.greens_function_json(to, frm, gf, lo, hi) == str(g["gf_text_1"])


def _every_index(shape):
    return [tuple(int(v) for v in np.unravel_index(b, shape)) for b in range(int(np.prod(shape)))]


def test_pattern_ldos_text_equals_reference():
    """calculateLDOS(patterns) with IDX_ALL and IDX_SUM_ALL: the entries, the
    wildcard nodes of the index tree and the sums over IDX_SUM_ALL give the
    reference's text."""
    g = golden("export")
    lo, hi, _ = _window(g, "pat_window")
    shape = (6, 5, 2)
    every = _every_index(shape)
    table = {idx: g["pat_ldos_all"][b] for b, idx in enumerate(every)}
    for k in range(int(g["pat_count"])):
        pats = _tuples(g[f"pat_patterns_{k}"])
        got = X.ldos_json_patterns(pats, every, table, lo, hi)
        assert got == _ref_text(g[f"pat_text_{k}"]), pats


def test_pattern_ldos_from_oracle(oracle):
    """The same texts from the oracle's LDOS at the expanded indices."""
    g = golden("export")
    lo, hi, res = _window(g, "pat_window")
    lat = L.square(6, 5, t=1.0, J=0.5, W=2.0, alpha=0.3, periodic=True, seed=11)
    rowptr, col, val = lat.csr()
    s, M, bro = 8.0, 128, 1e-3
    table = oracle.lookup_table(M, oracle.range(lo, hi, res), s)
    every = _every_index(lat.shape)
    for k in (0, 2, 3):
        pats = _tuples(g[f"pat_patterns_{k}"])
        ldos = {}
        for idx in X.expand_patterns(pats, every):
            b = lat.basis(idx)
            mu = oracle.damp(oracle.moments(rowptr, col, val, s, M, b, [b]), bro)
            ldos[idx] = oracle.ldos_table(table, mu[0])
        assert X.ldos_json_patterns(pats, every, ldos, lo, hi) == _ref_text(g[f"pat_text_{k}"])


def test_pattern_expansion_and_errors():
    every = _every_index((3, 2, 2))
    S, A = X.IDX_SUM_ALL, X.IDX_ALL
    assert X.expand_patterns([(1, S, 0)], every) == [(1, 0, 0), (1, 1, 0)]
    assert X.expand_patterns([(A, 1, 1), (0, 1, 1)], every) == [(0, 1, 1), (1, 1, 1), (2, 1, 1)]
    tree = X.IndexTree()
    tree.add((1, S, 0), wildcards=True)
    tree.generate_linear_map()
    assert tree.linear_index_of((1, 1, 0)) == 0 and tree.indices() == [(1, S, 0)]
    with pytest.raises(ValueError, match="wildcard"):
        X.expand_patterns([(1, -1610612739, 0)], every)  # IDX_SPIN
    with pytest.raises(ValueError, match="match no index"):
        X.ldos_json_patterns([(5, 0, 0)], every, {}, -1.0, 1.0)
    t = X.IndexTree()
    t.add((1, 0, 0))
    with pytest.raises(ValueError, match="wildcard"):
        t.add((1, S, 0), wildcards=True)
    # a summed and a concrete entry under the same subindex: TBTK's
    # IndexTree::add rejects the pair (and exits)
    with pytest.raises(ValueError, match="wildcard"):
        X.ldos_json_patterns([(2, S, S), (A, 0, 1)], every,
                             {i: np.zeros(3) for i in every}, -1.0, 1.0)


def test_reference_reads_exported_text(reference):
    """TBTK's Property::LDOS, EnergyResolvedProperty<complex<double>> and
    Property::Density constructors read the exported text and serialize
    the same text again, with the data in the tree's order."""
    rng = np.random.default_rng(4)
    sites = [(3, 1, 0), (0, 2, 1), (3, 0, 1), (7, 7, 0)]
    ldos = rng.random((4, 9)) * 10.0 ** rng.integers(-8, 3, (4, 9))
    text = X.ldos_json(sites, ldos, -2.5, 3.0)
    back, values = reference.reserialize(0, text, ldos.size)
    assert back == text
    got = X.loads(text)
    np.testing.assert_allclose(values.reshape(4, 9), got["data"], rtol=0)
    gf = rng.standard_normal((3, 5)) + 1j * rng.standard_normal((3, 5))
    text = X.greens_function_json(sites[:3], (1, 1, 1), gf, -1.0, 1.0)
    back, values = reference.reserialize(1, text, 2 * gf.size)
    assert back == text
    dens = rng.random(4)
    text = X.density_json(sites, dens)
    back, values = reference.reserialize(2, text, 4)
    assert back == text
    every = _every_index((4, 3, 2))
    table = {idx: rng.random(6) for idx in every}
    text = X.ldos_json_patterns([(2, X.IDX_SUM_ALL, X.IDX_SUM_ALL), (1, X.IDX_ALL, 1)], every,
                                table, -1.0, 1.0)
    back, values = reference.reserialize(0, text, 4 * 6)
    assert back == text


def test_loads_round_trip():
    rng = np.random.default_rng(1)
    sites = [(2, 0, 1), (0, 3, 0), (2, 0, 0)]
    ldos = rng.random((3, 6))
    r = X.loads(X.ldos_json(sites, ldos, -1.0, 2.0))
    assert r["kind"] == "LDOS"
    order = sorted(range(3), key=lambda k: sites[k])
    assert r["indices"] == [sites[k] for k in order]
    np.testing.assert_allclose(r["data"], ldos[order], rtol=6e-6)
    np.testing.assert_allclose(r["energies"], [-1.0 + k * 0.6 for k in range(6)])
    gf = rng.standard_normal((2, 4)) + 1j * rng.standard_normal((2, 4))
    r = X.loads(X.greens_function_json(sites[:2], (1, 1, 1), gf, 0.0, 3.0))
    assert r["kind"] == "GreensFunction"
    assert r["indices"] == [(0, 3, 0, None, 1, 1, 1), (2, 0, 1, None, 1, 1, 1)]
    np.testing.assert_allclose(r["data"], gf[[1, 0]], rtol=2e-5)
    every = _every_index((3, 2, 2))
    table = {idx: np.full(4, 0.125 * (1 + sum(idx))) for idx in every}
    r = X.loads(X.ldos_json_patterns([(1, X.IDX_SUM_ALL, 0), (2, 1, 1)], every, table,
                                     -1.0, 1.0))
    assert r["indices"] == [(1, X.IDX_SUM_ALL, 0), (2, 1, 1)]
    np.testing.assert_allclose(r["data"][:, 0], [0.25 + 0.375, 0.625])
    r = X.loads(X.density_json(sites, [0.25, 0.5, 0.75]))
    assert r["kind"] == "Density" and r["energies"] is None
    np.testing.assert_allclose(r["data"][:, 0], [0.5, 0.75, 0.25])


def test_json_number_format():
    """Doubles as nlohmann::json 2.1.1 writes them; data as std::ostream."""
    assert X.dumps({"b": 1.0, "a": -0.0, "c": 0.0}) == '{"a":-0.0,"b":1.0,"c":0.0}'
    assert X.dumps([1e20, 0.1, 1 / 3, float("nan"), float("inf")]) == \
        "[1e+20,0.1,0.333333333333333,null,null]"
    assert X.dumps([True, 3, "x"]) == '[true,3,"x"]'
    assert X._datum_real(1e-5) == "1e-05" and X._datum_real(123456789.0) == "1.23457e+08"
    assert X._datum_complex(0.5 - 2j) == "(0.5,-2)"


def test_export_rejects_bad_input():
    with pytest.raises(ValueError, match="wildcard"):
        X.ldos_json([(0, -1)], np.zeros((1, 3)), -1.0, 1.0)
    with pytest.raises(ValueError, match="more than once"):
        X.ldos_json([(0, 1), (0, 1)], np.zeros((2, 3)), -1.0, 1.0)
    with pytest.raises(ValueError, match="incompatible"):
        X.ldos_json([(0, 1), (0, 1, 2)], np.zeros((2, 3)), -1.0, 1.0)
    with pytest.raises(ValueError, match="data blocks"):
        X.ldos_json([(0, 1), (0, 2)], np.zeros((3, 3)), -1.0, 1.0)
    with pytest.raises(ValueError, match="resolution"):
        X.ldos_json([(0, 1)], np.zeros((1, 1)), -1.0, 1.0)
    with pytest.raises(ValueError, match="not an LDOS"):
        X.loads('{"id":"Magnetization"}')
