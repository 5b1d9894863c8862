"""Two-index classes of the reference's example script (overlap_2idx,
nuclear_2idx; examples/example_input.py:83-107): the C restatement pinned to
the reference's emitted C99 (tests/golden/twoidx.npz), and the CUDA drop-ins
and batch entry point against both."""
import os

import numpy as np
import pytest

from conftest import GOLDEN


def _golden():
    z = np.load(os.path.join(GOLDEN, 'twoidx.npz'))
    pairs = {k: z[k] for k in ('xa', 'ca', 'la', 'xb', 'cb', 'lb', 'cc', 'off', 'size')}
    return pairs, z['overlap'], z['nuclear'], z['work_array_size']


def _blocks(pairs):
    la, lb = pairs['la'], pairs['lb']
    n = ((la + 1) * (la + 2) // 2) * ((lb + 1) * (lb + 2) // 2)
    return [(int(o), int(o + k)) for o, k in zip(pairs['off'], n)]


def _assert_blocks(got, ref, pairs, rel):
    """Per pair: |got - ref| <= rel * max(1, max |ref block|) (primitive,
    unnormalised integrals span many decades across pairs)."""
    worst = 0.0
    for i, (b, e) in enumerate(_blocks(pairs)):
        scale = max(1.0, float(np.abs(ref[b:e]).max()))
        err = float(np.abs(got[b:e] - ref[b:e]).max()) / scale
        worst = max(worst, err)
        assert err <= rel, 'pair %d (la=%d lb=%d): %.3e' % (i, pairs['la'][i], pairs['lb'][i], err)
    return worst


def _subset(pairs, keep):
    idx = np.nonzero(keep)[0]
    la, lb = pairs['la'][idx], pairs['lb'][idx]
    sizes = ((la + 1) * (la + 2) // 2) * ((lb + 1) * (lb + 2) // 2)
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    sub = dict(xa=pairs['xa'][idx], ca=pairs['ca'].reshape(-1, 3)[idx].ravel(), la=la, xb=pairs['xb'][idx],
               cb=pairs['cb'].reshape(-1, 3)[idx].ravel(), lb=lb, cc=pairs['cc'].reshape(-1, 3)[idx].ravel(),
               off=off, size=np.int64(sizes.sum()))
    return sub, idx


def _gather(full, pairs, idx):
    blocks = _blocks(pairs)
    return np.concatenate([full[blocks[i][0]:blocks[i][1]] for i in idx])


# ---------------------------------------------------------------- CPU: oracle
@pytest.mark.parametrize('kind', [0, 1])
def test_oracle_matches_reference_fixture(kind):
    from oracle import loader
    pairs, ov, nu, _ = _golden()
    got = loader.twoidx_batch(kind, pairs)
    _assert_blocks(got, ov if kind == 0 else nu, pairs, 1e-13)


def test_oracle_work_array_size_matches_reference():
    from oracle import loader
    lib = loader.load_oracle()
    for kind, la, lb, want in _golden()[3]:
        assert lib.oracle_2idx_work_array_size(int(kind), int(la), int(lb)) == want


def test_oracle_dropin_strides():
    """The emitted calling convention: only output_array[ia*iskipa + ib*iskipb] written."""
    import ctypes as C
    from oracle import loader
    lib = loader.load_oracle()
    dp = C.POINTER(C.c_double)
    pairs, ov, nu, _ = _golden()
    blocks = _blocks(pairs)
    for i in (3, 77, 200):
        la, lb = int(pairs['la'][i]), int(pairs['lb'][i])
        na, nb = (la + 1) * (la + 2) // 2, (lb + 1) * (lb + 2) // 2
        iskipa, iskipb = nb + 2, 1  # b fastest, padded rows
        for kind, ref in ((0, ov), (1, nu)):
            out = np.full(na * iskipa + 4, -7.0)
            A = np.ascontiguousarray(pairs['ca'][3 * i:3 * i + 3])
            B = np.ascontiguousarray(pairs['cb'][3 * i:3 * i + 3])
            Cc = np.ascontiguousarray(pairs['cc'][3 * i:3 * i + 3])
            work = np.zeros(4)
            args = [float(pairs['xa'][i]), A.ctypes.data_as(dp), la, na, iskipa, float(pairs['xb'][i]),
                    B.ctypes.data_as(dp), lb, nb, iskipb]
            if kind == 0:
                lib.oracle_overlap_2idx_ab_prim_cart_main(*args, work.ctypes.data_as(dp), out.ctypes.data_as(dp))
            else:
                lib.oracle_nuclear_2idx_ab_m_cC_prim_cart_main(*args, Cc.ctypes.data_as(dp),
                                                               work.ctypes.data_as(dp), out.ctypes.data_as(dp))
            blk = ref[blocks[i][0]:blocks[i][1]].reshape(nb, na).T
            written = np.zeros(out.shape, bool)
            for ia in range(na):
                for ib in range(nb):
                    written[ia * iskipa + ib * iskipb] = True
                    assert abs(out[ia * iskipa + ib * iskipb] - blk[ia, ib]) <= 1e-13 * max(1, abs(blk).max())
            assert np.all(out[~written] == -7.0)


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize('kind', [0, 1])
def test_batch_matches_reference_fixture(kind):
    import torch
    from intception_b200 import twoidx
    pairs, ov, nu, _ = _golden()
    batch = twoidx.TwoIndexBatch(pairs)
    got = batch.compute(kind).cpu().numpy()
    torch.cuda.synchronize()
    assert batch.device_status() == 0
    _assert_blocks(got, ov if kind == 0 else nu, pairs, 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize('kind', [0, 1])
@pytest.mark.parametrize('lmax', [0, 1, 2, 3, 4, 5, 6])
def test_batch_every_group_size(kind, lmax):
    """Each lmax selects its lane-group size and shared-memory plan."""
    from intception_b200 import twoidx
    pairs, ov, nu, _ = _golden()
    sub, idx = _subset(pairs, (pairs['la'] <= lmax) & (pairs['lb'] <= lmax))
    ref = _gather(ov if kind == 0 else nu, pairs, idx)
    batch = twoidx.TwoIndexBatch(sub)
    assert batch.lmax == lmax
    got = batch.compute(kind).cpu().numpy()
    assert batch.device_status() == 0
    _assert_blocks(got, ref, sub, 1e-12)


@pytest.mark.gpu
def test_batch_refuses_pairs_above_lmax():
    """Pairs above the declared lmax are skipped (blocks untouched) and
    flagged; every other pair is still evaluated."""
    import torch
    from intception_b200 import twoidx
    pairs, ov, nu, _ = _golden()
    sub, idx = _subset(pairs, (pairs['la'] <= 3) & (pairs['lb'] <= 3))
    ref = _gather(nu, pairs, idx)
    batch = twoidx.TwoIndexBatch(sub)
    out = torch.full((int(sub['size']),), -7.0, dtype=torch.float64, device='cuda')
    batch.compute(twoidx.NUCLEAR, out=out, lmax=2)
    assert batch.device_status() == twoidx._eri.IB_ERR_ARG
    got = out.cpu().numpy()
    high = (sub['la'] > 2) | (sub['lb'] > 2)
    assert high.any() and (~high).any()
    for i, (b, e) in enumerate(_blocks(sub)):
        if high[i]:
            assert np.all(got[b:e] == -7.0)
        else:
            assert np.abs(got[b:e] - ref[b:e]).max() <= 1e-12 * max(1.0, float(np.abs(ref[b:e]).max()))


@pytest.mark.gpu
def test_dropins_match_reference_fixture_with_strides():
    from intception_b200 import twoidx
    pairs, ov, nu, _ = _golden()
    blocks = _blocks(pairs)
    rng = np.random.default_rng(5)
    for i in list(rng.choice(len(pairs['la']), 40, replace=False)) + [len(pairs['la']) - 1]:
        la, lb = int(pairs['la'][i]), int(pairs['lb'][i])
        na, nb = twoidx.ncart(la), twoidx.ncart(lb)
        iskipa, iskipb = 1, na + 3
        A, B, Cc = (pairs[k][3 * i:3 * i + 3] for k in ('ca', 'cb', 'cc'))
        for kind, ref in ((0, ov), (1, nu)):
            out = np.full(nb * iskipb + 2, -7.0)
            if kind == 0:
                twoidx.overlap_main(pairs['xa'][i], A, la, na, iskipa, pairs['xb'][i], B, lb, nb, iskipb, out)
            else:
                twoidx.nuclear_main(pairs['xa'][i], A, la, na, iskipa, pairs['xb'][i], B, lb, nb, iskipb, Cc, out)
            blk = ref[blocks[i][0]:blocks[i][1]].reshape(nb, na)
            view = np.stack([out[ib * iskipb:ib * iskipb + na] for ib in range(nb)])
            assert np.abs(view - blk).max() <= 1e-12 * max(1.0, np.abs(blk).max())
            mask = np.ones(out.shape, bool)
            for ib in range(nb):
                mask[ib * iskipb:ib * iskipb + na] = False
            assert np.all(out[mask] == -7.0)


@pytest.mark.gpu
def test_dropin_argument_errors():
    from intception_b200 import twoidx
    out = np.zeros(64)
    A = np.zeros(3)
    with pytest.raises(twoidx._eri.IntceptionError):
        twoidx.overlap_main(1.0, A, 1, 2, 1, 1.0, A, 0, 1, 3, out)  # na != 3
    with pytest.raises(twoidx._eri.IntceptionError):
        twoidx.nuclear_main(1.0, A, 7, 36, 1, 1.0, A, 0, 1, 36, A, np.zeros(64))  # l = 7
    twoidx.overlap_main(1.0, A, 0, 1, 1, 1.0, A, 0, 1, 1, out)  # still usable afterwards
    assert abs(out[0] - (np.pi / 2.0) ** 1.5) < 1e-14


@pytest.mark.gpu
def test_work_array_sizes_match_reference():
    from intception_b200 import twoidx
    for kind, la, lb, want in _golden()[3]:
        f = twoidx.overlap_work_array_size if kind == 0 else twoidx.nuclear_work_array_size
        assert f(int(la), int(lb)) == want


@pytest.mark.gpu
@pytest.mark.parametrize('kind', [0, 1])
def test_large_batch_symmetry_and_translation(kind):
    """Full-size properties: swapping a and b transposes every block, and a
    rigid shift of all centres leaves every block unchanged."""
    import torch
    from intception_b200 import twoidx
    rng = np.random.default_rng(9)
    n = 200000
    la = rng.integers(0, 4, n).astype(np.int32)
    lb = rng.integers(0, 4, n).astype(np.int32)
    xa = np.exp(rng.uniform(np.log(0.1), np.log(30.0), n))
    xb = np.exp(rng.uniform(np.log(0.1), np.log(30.0), n))
    ca, cb, cc = (rng.uniform(0, 3, (n, 3)) for _ in range(3))
    p = dict(xa=xa, ca=ca, la=la, xb=xb, cb=cb, lb=lb, cc=cc)
    q = dict(xa=xb, ca=cb, la=lb, xb=xa, cb=ca, lb=la, cc=cc)
    s = dict(p, ca=ca + 1.7, cb=cb + 1.7, cc=cc + 1.7)
    g = [twoidx.TwoIndexBatch(d).compute(kind) for d in (p, q, s)]
    torch.cuda.synchronize()
    g = [x.cpu().numpy() for x in g]
    off_p, _ = twoidx.block_offsets(la, lb)
    off_q, _ = twoidx.block_offsets(lb, la)
    for i in rng.choice(n, 3000, replace=False):
        na, nb = twoidx.ncart(la[i]), twoidx.ncart(lb[i])
        bp = g[0][off_p[i]:off_p[i] + na * nb].reshape(nb, na)
        bq = g[1][off_q[i]:off_q[i] + na * nb].reshape(na, nb)
        scale = max(1.0, np.abs(bp).max())
        assert np.abs(bp - bq.T).max() <= 1e-12 * scale
    scale = np.maximum(1.0, np.abs(g[0]))
    assert np.max(np.abs(g[2] - g[0]) / scale) <= 1e-9  # shifted centres round differently


@pytest.mark.gpu
@pytest.mark.parametrize('kind', [0, 1])
def test_batch_bulk_copied_chunks_vs_oracle(kind):
    """Five complete 512-pair chunks (their inputs fetched by bulk copies into
    alternating shared-memory buffers) and a partial one (plain loads), against
    the C restatement; then the same pairs with one input array 8 bytes off a
    16-byte boundary, which sends every chunk through plain loads."""
    import torch
    from intception_b200 import twoidx
    from oracle import loader
    pairs = twoidx.make_pairs(5 * 512 + 77, lmax=2, seed=12)
    pairs['off'], pairs['size'] = twoidx.block_offsets(pairs['la'], pairs['lb'])
    ref = loader.twoidx_batch(kind, pairs)
    batch = twoidx.TwoIndexBatch(pairs)
    got = batch.compute(kind).cpu().numpy()
    assert batch.device_status() == 0
    _assert_blocks(got, ref, pairs, 1e-12)
    shifted = torch.empty(batch.n + 1, dtype=torch.float64, device=batch.xa.device)
    shifted[1:] = batch.xa
    batch.xa = shifted[1:]
    assert batch.xa.data_ptr() % 16 == 8
    got2 = batch.compute(kind).cpu().numpy()
    assert batch.device_status() == 0
    assert np.array_equal(got, got2)


@pytest.mark.gpu
@pytest.mark.parametrize('kind', [0, 1])
def test_bounded_wait_gives_up_and_reports_timeout(kind):
    """The thread kernel's wait for a chunk's bulk copies is bounded: with the
    testing knob, chunk 0's bytes are announced on its barrier but never
    copied, the block gives up after 2^14 polls, stores IB_ERR_TIMEOUT, drains
    its other copies and returns.  Chunk 0's pairs stay untouched, every other
    chunk is correct, and the knob is one-shot."""
    import torch
    from intception_b200 import twoidx
    from oracle import loader
    pairs = twoidx.make_pairs(8 * 512, 2, seed=5, box=6.0)
    pairs['off'], pairs['size'] = twoidx.block_offsets(pairs['la'], pairs['lb'])
    ref = loader.twoidx_batch(kind, {k: np.asarray(v).reshape(-1) if k in ('ca', 'cb', 'cc') else v
                                     for k, v in pairs.items()})
    batch = twoidx.TwoIndexBatch(pairs)
    out = torch.full((batch.size,), -7.0, dtype=torch.float64, device='cuda')
    assert twoidx._lib().intception_b200_twoidx_test_stall(0, 1 << 14) == 0
    batch.compute(kind, out=out)
    torch.cuda.synchronize()
    assert batch.device_status() == twoidx._eri.IB_ERR_TIMEOUT
    got = out.cpu().numpy()
    blocks = _blocks(pairs)
    for i, (b, e) in enumerate(blocks):
        if i < 512:
            assert np.all(got[b:e] == -7.0)
        else:
            assert np.abs(got[b:e] - ref[b:e]).max() <= 1e-12 * max(1.0, float(np.abs(ref[b:e]).max()))
    batch.status.zero_()
    batch.compute(kind, out=out)
    torch.cuda.synchronize()
    assert batch.device_status() == 0
    _assert_blocks(out.cpu().numpy(), ref, pairs, 1e-12)
