"""Batched tensor-core rescoring (tcgen05 kind::i8) against the int64 oracle.

Integer work, so the bar is bit-exact: every statistic and every Gram entry
equals the oracle's int64 recompute (xwo_rescore, the restatement of the
reference's rebuild_gram / verify_weighing).  At the benchmark's size (65536
matrices per order) the tensor-core results are compared with the
independent SIMT kernel for every matrix and with the oracle on a sample.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
import xtax_b200 as X

pytestmark = pytest.mark.gpu


def random_fixed_degree(count, n, w, seed):
    """Row-only fixed-degree ternary matrices: w nonzeros per row at uniform
    positions with uniform signs (row-major)."""
    rng = np.random.default_rng(seed)
    W = np.zeros((count, n, n), dtype=np.int8)
    for m in range(count):
        idx = np.argsort(rng.random((n, n)), axis=1)[:, :w]
        signs = rng.integers(0, 2, size=(n, w)) * 2 - 1
        np.put_along_axis(W[m], idx, signs.astype(np.int8), axis=1)
    return W


def oracle_stats(M, n, w):
    st, G, _ = O.rescore(n, w, M.T.reshape(-1))   # oracle takes column-major W
    exact = O.verify(n, w, M.T.reshape(-1)) == 3
    return [int(st[0]), int(st[1]), int(st[2]), 1 if (st[1] == 0 and (np.diag(G) == w).all()) else 0], G, exact


@pytest.mark.parametrize("n", [32, 64, 96, 128])
@pytest.mark.parametrize("count", [1, 3, 37, 301])
def test_tensor_core_rescore_matches_oracle(n, count):
    w = n // 2
    W = random_fixed_degree(count, n, w, seed=n * 1000 + count)
    # plant exact weighing matrices: direct sums of Sylvester blocks of order 32
    syl = O.sylvester(n, 32).reshape(n, n).T.astype(np.int8)   # row-major
    for m in range(0, count, 7):
        W[m] = syl
    stats, G = X.rescore(W, n, w, gram=True)
    for m in range(count):
        ww = 32 if m % 7 == 0 else w
        ref, Gref, _ = oracle_stats(W[m], n, ww)
        if ww != w:
            # the diagonal check uses the call's w: Sylvester rows have weight 32
            ref[3] = 1 if (ref[1] == 0 and (np.diag(Gref) == w).all()) else 0
        assert stats[m].tolist() == ref, (m, stats[m], ref)
        assert (G[m] == Gref).all(), m


@pytest.mark.parametrize("n", [32, 64, 96, 128])
def test_rescore_at_benchmark_size(n):
    torch = pytest.importorskip("torch")
    count, w = 65536, n // 2
    gen = torch.Generator(device="cuda").manual_seed(n)
    # fixed-degree rows on the device: random permutation keys pick w columns
    W = torch.zeros((count, n, n), dtype=torch.int8, device="cuda")
    for c0 in range(0, count, 4096):
        keys = torch.rand((4096, n, n), device="cuda", generator=gen)
        idx = keys.argsort(dim=2)[:, :, :w]
        signs = (torch.randint(0, 2, (4096, n, w), device="cuda", generator=gen) * 2 - 1).to(torch.int8)
        W[c0:c0 + 4096].scatter_(2, idx, signs)
        del keys, idx, signs
    s_tc = torch.zeros((count, 4), dtype=torch.int32, device="cuda")
    s_simt = torch.zeros((count, 4), dtype=torch.int32, device="cuda")
    rc = X.lib().xw_rescore_device(C.c_void_p(W.data_ptr()), count, n, w, C.c_void_p(s_tc.data_ptr()), None, 0, None)
    assert rc == X.XW_OK
    rc = X.lib().xw_rescore_device(C.c_void_p(W.data_ptr()), count, n, w, C.c_void_p(s_simt.data_ptr()), None, 1,
                                   None)
    assert rc == X.XW_OK
    torch.cuda.synchronize()
    assert X.lib().xw_rescore_status() == X.XW_OK
    assert torch.equal(s_tc, s_simt)
    Wh = W.cpu().numpy()
    sh = s_tc.cpu().numpy()
    rng = np.random.default_rng(n)
    for m in rng.choice(count, 64, replace=False):
        ref, _, _ = oracle_stats(Wh[m], n, w)
        assert sh[m].tolist() == ref, m


@pytest.mark.parametrize("n", [1, 5, 12, 26, 63, 100, 127, 160, 256])
def test_simt_rescore_for_orders_off_the_tensor_core_grid(n):
    # orders that are not multiples of 32 take the SIMT kernel
    count, w = 17, max(1, n // 3)
    W = random_fixed_degree(count, n, w, seed=500 + n)
    stats, G = X.rescore(W, n, w, gram=True)
    for m in range(count):
        ref, Gref, _ = oracle_stats(W[m], n, w)
        assert stats[m].tolist() == ref, (m, stats[m], ref)
        assert (G[m] == Gref).all(), m


def test_rescore_empty_batch_and_bad_arguments():
    import ctypes as C
    stats = np.zeros((1, 4), dtype=np.int32)
    W = np.zeros((1, 32, 32), dtype=np.int8)
    assert X.lib().xw_rescore(W.ctypes.data_as(C.POINTER(C.c_int8)), 0, 32, 16,
                              stats.ctypes.data_as(C.POINTER(C.c_int32)), None) == X.XW_OK
    assert X.lib().xw_rescore(W.ctypes.data_as(C.POINTER(C.c_int8)), 1, 257, 16,
                              stats.ctypes.data_as(C.POINTER(C.c_int32)), None) == X.XW_ERR_INVALID
