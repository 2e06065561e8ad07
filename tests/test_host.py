"""CPU: host-side logic of the package (shape bookkeeping, genealogical
addressing, argument validation, integral layouts)."""
import numpy as np
import pytest

import restate as R


def test_csfvec_shape_matches_restatement():
    from pyscf_forge_b200.csf_fci import csfstring as C
    from pyscf_forge_b200.csf_fci import csdstring as D
    for norb in range(1, 9):
        for na in range(0, norb + 1):
            for nb in range(0, norb + 1):
                a = D.get_csdaddrs_shape(norb, na, nb)
                b = R.get_csdaddrs_shape(norb, na, nb)
                for x, y in zip(a[1:], b[1:]):
                    assert np.array_equal(x, y)
                for smult in range(abs(na - nb) + 1, na + nb + 3, 2):
                    try:
                        ref = R.get_csfvec_shape(norb, na, nb, smult)
                    except R.ImpossibleCIvecError:
                        with pytest.raises(C.ImpossibleCIvecError):
                            C.get_csfvec_shape(norb, na, nb, smult)
                        continue
                    got = C.get_csfvec_shape(norb, na, nb, smult)
                    assert got[0] == ref[0]
                    for x, y in zip(got[1:], ref[1:]):
                        assert np.array_equal(x, y)


def test_impossible_spin_raises():
    from pyscf_forge_b200.csf_fci import csfstring as C
    with pytest.raises(C.ImpossibleSpinError):
        C.get_csfvec_shape(4, 3, 1, 1)
    with pytest.raises(C.ImpossibleSpinError):
        C.get_csfvec_shape(4, 2, 2, 7)
    with pytest.raises(C.ImpossibleCIvecError):
        C.get_csfvec_shape(4, 5, 2, 4)


def test_genealogical_round_trip():
    """test_csfstring.py:41-51: addrs2str <-> strs2addr for nspin 0..20."""
    from pyscf_forge_b200.csf_fci import csfstring as C
    rng = np.random.default_rng(0)
    for nspin in range(21):
        for s2 in range(nspin % 2, nspin + 1, 2):
            smult = s2 + 1
            ncsf = C.count_csfs(nspin, smult)
            assert ncsf == R.count_csfs(nspin, smult)
            addrs = rng.integers(0, ncsf, size=min(ncsf, 5))
            strs = C.addrs2str(nspin, smult, addrs)
            assert np.array_equal(C.strs2addr(nspin, smult, strs), addrs)
            assert np.array_equal(strs, R.gen_addrs2str(nspin, smult, addrs))
            assert np.array_equal(C.csf_gentable(nspin, smult), R.csf_gentable(nspin, smult))


def test_no_overflow_26_spins():
    """test_csfstring.py:64-69 counterpart for the counting path."""
    from pyscf_forge_b200.csf_fci import csfstring as C
    assert C.count_csfs(26, 27) == 1
    assert C.count_csfs(26, 1) == R.count_csfs(26, 1)


def test_eri_layouts():
    from pyscf_forge_b200._runtime import eri_pair_matrix
    from conftest import seeded_integrals
    h1, eri = seeded_integrals(5, 6)
    e4 = eri_pair_matrix(eri, 5)
    assert e4.shape == (15, 15)
    np.testing.assert_allclose(e4, R.restore4(eri, 5))
    e8 = e4[np.tril_indices(15)]
    np.testing.assert_allclose(eri_pair_matrix(e8, 5), e4)
    np.testing.assert_allclose(eri_pair_matrix(e4, 5), e4)


def test_state_weights_validation():
    """State weights: non-empty, finite, non-negative, summing to one
    (the checks of pyscf/mcscf/addons_gas.py:103-114)."""
    import pytest
    from pyscf_forge_b200.state_average import validate_state_weights
    assert list(validate_state_weights([0.25, 0.75])) == [0.25, 0.75]
    for bad in ([], [[0.5, 0.5]], [0.5, float("nan")], [1.5, -0.5], [0.5, 0.4]):
        with pytest.raises(ValueError):
            validate_state_weights(bad)


def _max_rank_worker(rank, world, port, q):
    import os
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        q.put((rank, bench.max_over_ranks(1.5 + rank, world, device="cpu")))
    finally:
        dist.destroy_process_group()


def test_bench_max_over_ranks_gloo():
    """The multi-replica timing reduction of bench.py (max over ranks) on
    two gloo ranks: every rank sees the slowest rank's time."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_max_rank_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}
