"""CPU: the GAS restriction normalisation (csf_fci.gas) against the
reference's own canonical block sets (fixtures made by
pyscf/mcscf/addons_gas.normalize_gas_spec, tests/golden/make_golden.py) and
the expectations of the reference's tests (pyscf/mcscf/test/test_gasci.py:
120-161)."""
import numpy as np
import pytest

from conftest import load_golden

GAS_CASES = ["gas_ras_norb6_3e3e", "gas_cumocc_norb7_4e3e", "gas_supergroup_norb6_3e3e", "gas_spinsg_norb6_2e2e"]


def _gas():
    import pyscf_forge_b200.csf_fci.gas as G
    return G


def _restr(g):
    t = str(g["gas_restr_type"])
    if t == "ras":
        return {"max_holes": int(g["ras_max_holes"]), "max_particles": int(g["ras_max_particles"])}, t
    return g["gas_restr"].tolist(), t


@pytest.mark.parametrize("tag", GAS_CASES)
def test_canonical_blocks_match_reference(tag):
    G = _gas()
    g = load_golden(tag)
    nelec = (int(g["neleca"]), int(g["nelecb"]))
    restr, t = _restr(g)
    korbs, blocks = G.normalize_gas_spec(tuple(g["gas_orbs"].tolist()), nelec, restr, t)
    assert korbs == tuple(g["kernel_gas_orbs"].tolist())
    np.testing.assert_array_equal(blocks, g["blocks"])
    assert G.gas_ndet(korbs, nelec, blocks) == int(np.count_nonzero(g["allowed_dets"]))
    assert G.is_spin_complete(korbs, nelec, blocks)


def test_equivalent_restriction_types():
    """test_gasci.py:120-147: one space, three spellings."""
    G = _gas()
    expected = np.asarray([[0, 2, 2, 0], [1, 1, 1, 1], [2, 0, 0, 2]], dtype=np.int32)
    explicit = [[2, 0, 0, 2], [1, 1, 1, 1], [0, 2, 2, 0], [1, 1, 1, 1]]
    for t, r in (("spin-supergroup", explicit), ("supergroup", [[2, 2]]), ("cumulative-occ", [[2, 2], [4, 4]])):
        np.testing.assert_array_equal(G.normalize_gas_spec((2, 2), (2, 2), r, t)[1], expected)
    assert G.is_spin_complete((2, 2), (2, 2), expected)


def test_ras_matches_cumulative_bounds():
    """test_gasci.py:149-161."""
    G = _gas()
    korbs, ras = G.normalize_gas_spec((1, 2, 1), (2, 2), {"max_holes": 1, "max_particles": 1}, "ras")
    _, cum = G.normalize_gas_spec((1, 2, 1), (2, 2), [[1, 2], [3, 4], [4, 4]], "cumulative-occ")
    assert korbs == (1, 2, 1)
    np.testing.assert_array_equal(ras, cum)


def test_ras_drops_empty_spaces():
    G = _gas()
    korbs, blocks = G.normalize_gas_spec((0, 4, 2), (2, 2), {"max_holes": 0, "max_particles": 1}, "ras")
    assert korbs == (4, 2)
    assert np.all(blocks[:, 1] + blocks[:, 3] <= 1)


def test_spin_incomplete_set_is_rejected():
    """A spin-supergroup set missing alpha/beta splits spans no whole
    configurations; the CSF basis cannot represent it."""
    G = _gas()
    assert not G.is_spin_complete((2, 2), (2, 2), [[1, 1, 1, 1]])
    with pytest.raises(ValueError):
        G.spin_free_supergroups((2, 2), (2, 2), [[1, 1, 1, 1]], "spin-supergroup")
    korbs, sg = G.spin_free_supergroups((2, 2), (2, 2), [[2, 2]], "supergroup")
    assert korbs == (2, 2) and sg.tolist() == [[2, 2]]


def test_validation_errors():
    G = _gas()
    with pytest.raises(TypeError):
        G.normalize_gas_spec((2, 2), (2, 2), [[2.0, 2.0]], "supergroup")
    with pytest.raises(TypeError):
        G.normalize_gas_spec((2, 2), (2, 2), [[True, 3]], "supergroup")
    with pytest.raises(ValueError):
        G.normalize_gas_spec((2, 2), (2, 2), None, "spin-supergroup")
    with pytest.raises(NotImplementedError):
        G.normalize_gas_spec((2, 2), (2, 2), [[2, 2]], "no-such-type")
    with pytest.raises(ValueError):
        G.normalize_gas_spec((2, 2), (2, 2), [[3, 2]], "supergroup")  # wrong electron count
    with pytest.raises(ValueError):
        G.normalize_gas_spec((2, 2), (2, 2), [[3, 2], [4, 4]], "cumulative-occ")  # min > max
    with pytest.raises(ValueError):
        G.normalize_gas_spec((1, 2, 1), (2, 2), {"max_holes": 1}, "ras")
    korbs, loose = G.normalize_gas_spec((2, 2), (2, 2), [[0, 4], [4, 4]], "cumulative-occ")
    assert G.is_spin_complete(korbs, (2, 2), loose) and loose.shape[0] == 9  # every split of 4 electrons
    korbs, single = G.normalize_gas_spec((4,), (2, 1))
    assert korbs == (4,) and single.tolist() == [[2, 1]]


def test_solver_checks_subspace_sizes():
    import pyscf_forge_b200 as P
    sol = P.csf_solver(None, smult=1, gas_orbs=(2, 3), gas_restr=[[2, 2]], gas_restr_type="supergroup")
    with pytest.raises(ValueError):
        sol.gas_spec(6, (2, 2))
