"""Per-block format selection on the GPU: candidate encoders and sizes against
the oracle, the blockwise container, features, MLP gradients against a
float64 CPU restatement, training, and what the trained selector gains over
the methods without it."""
import numpy as np
import pytest

import oracle as O
from oracle import selector_ref as R

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sel(ms):
    import engine_b200.selector as S
    return S


@pytest.fixture(scope="module")
def mixed(ms, arena, orc, sel):
    """96 blocks, segments of 4 blocks cycling through the four families."""
    nblk = 96
    z = orc.zipf_table(1.2, 1 << 20)
    d = sel.gen(arena, 11, nblk, 4, z)
    return d, nblk, sel.to_host(d, nblk * sel.BLOCK, np.uint64).reshape(nblk, sel.BLOCK)


def test_generator_is_deterministic(ms, arena, orc, sel, mixed):
    d, nblk, x = mixed
    d2 = sel.gen(arena, 11, nblk, 4, orc.zipf_table(1.2, 1 << 20))
    assert np.array_equal(sel.to_host(d2, nblk * sel.BLOCK, np.uint64).reshape(nblk, -1), x)
    # family of block b: (segment + seed) % 4 -> 0 uniform, 1 sorted, 2 runs, 3 Zipf
    fam = [((b // 4) + 11) % 4 for b in range(nblk)]
    assert all(np.all(np.diff(x[b].astype(np.float64)) > 0) for b in range(nblk) if fam[b] == 1)
    assert all(len(np.unique(x[b])) < 200 for b in range(nblk) if fam[b] == 2)


@pytest.mark.parametrize("cand", [0, 1, 2, 3, 4])
def test_candidate_payloads_and_sizes(ms, arena, orc, sel, mixed, cand):
    d, nblk, x = mixed
    st, sz = sel.analyze(arena, d, nblk)
    sizes = sel.to_host(sz, nblk * 5, np.uint32).reshape(nblk, 5)
    choice = sel.to_device(arena, np.full(nblk, cand, dtype=np.uint8))
    cont = sel.Container(arena, d, nblk, st, choice)
    raw = cont.host_bytes()
    psz = sel.to_host(cont.psz, nblk, np.uint32)
    code_off, pay_off, total = R.container_positions(psz.astype(np.int64))
    assert cont.nbytes == total
    for b in range(nblk):
        code, payload = R.candidate_payload(orc, x[b], cand)
        assert sizes[b, cand] == len(payload), b
        assert psz[b] == len(payload)
        assert raw[code_off[b]] == code
        got = raw[pay_off[b]: pay_off[b] + len(payload)]
        assert np.array_equal(R.mask_for_header(got, cand), R.mask_for_header(payload, cand)), b


def test_compress_all_matches_size_pass(ms, arena, sel, mixed):
    d, nblk, x = mixed
    _, sz1 = sel.analyze(arena, d, nblk)
    _, sz2 = sel.compress_all(arena, d, nblk)
    assert np.array_equal(sel.to_host(sz1, nblk * 5, np.uint32), sel.to_host(sz2, nblk * 5, np.uint32))


def test_container_select_sum(ms, arena, orc, sel, mixed):
    d, nblk, x = mixed
    st, sz = sel.analyze(arena, d, nblk)
    rng = np.random.default_rng(3)
    choice = rng.integers(0, 5, nblk).astype(np.uint8)
    cont = sel.Container(arena, d, nblk, st, sel.to_device(arena, choice))
    for cmp, val in ((O.CMP_LT, 1 << 19), (O.CMP_GE, 1000), (O.CMP_EQ, int(x[9, 5]))):
        s, c, err = cont.select_sum(cmp, val)
        flat = x.ravel()
        es, ec = orc.select_project_sum(cmp, val, flat, flat, len(flat))
        assert (s, c, err) == (es, ec, 0), cmp


def test_features_match_restatement(ms, arena, sel, mixed):
    d, nblk, x = mixed
    f = sel.to_host(sel.features(arena, d, nblk), nblk * 32, np.float32).reshape(nblk, 32)
    for b in range(nblk):
        np.testing.assert_allclose(f[b], R.features(x[b]), rtol=1e-6, atol=1e-7)


def test_mlp_gradients_match_cpu(ms, arena, sel, mixed):
    d, nblk, x = mixed
    _, sz = sel.analyze(arena, d, nblk)
    fd = sel.features(arena, d, nblk)
    m = sel.Mlp(seed=5, max_batch=256)
    try:
        idx = np.arange(nblk, dtype=np.uint32)
        g, loss = m.grads(arena, fd, sz, nblk, idx)
        feats = sel.to_host(fd, nblk * 32, np.float32).reshape(nblk, 32)
        sizes = sel.to_host(sz, nblk * 5, np.uint32).reshape(nblk, 5)
        eloss, eg = R.loss_and_grads(m.params(), feats, sizes)
        assert abs(loss - eloss) <= 1e-4 * max(1.0, eloss)
        np.testing.assert_allclose(g, eg, rtol=2e-3, atol=1e-5 * np.abs(eg).max())
    finally:
        m.close()


def test_mlp_predictions_match_cpu(ms, arena, sel, mixed):
    """The tensor-core forward pass (k_mlp_choose) against the float64
    restatement with the same BF16 rounding points, after a few training
    steps so that every layer carries signal; also the choice and the
    fallback decision derived from the predictions."""
    d, nblk, x = mixed
    _, sz = sel.analyze(arena, d, nblk)
    fd = sel.features(arena, d, nblk)
    m = sel.Mlp(seed=9, max_batch=256)
    try:
        m.train(arena, fd, sz, nblk, steps=30, batch=96)
        margin = 0.05
        ch, nf, pr = m.choose(arena, fd, nblk, margin, want_pred=True)
        got = sel.to_host(pr, nblk * 5, np.float32).reshape(nblk, 5)
        feats = sel.to_host(fd, nblk * 32, np.float32).reshape(nblk, 32)
        want = R.forward(m.params(), feats)
        np.testing.assert_allclose(got, want, rtol=1e-3, atol=2e-2)
        choice = sel.to_host(ch, nblk, np.uint8)
        srt = np.sort(got, axis=1)
        unsure = srt[:, 1] - srt[:, 0] < margin
        assert np.array_equal(choice == 255, unsure)
        assert np.array_equal(choice[~unsure], np.argmin(got, axis=1)[~unsure])
        assert int(sel.to_host(nf, 1, np.uint64)[0]) == int(unsure.sum())
    finally:
        m.close()


def _dataset(ms, arena, orc, sel, seed, nblk):
    d = sel.gen(arena, seed, nblk, 32, orc.zipf_table(1.2, 1 << 20))
    st, sz = sel.analyze(arena, d, nblk)
    return d, st, sz, sel.features(arena, d, nblk)


def test_training_and_what_the_network_gains(ms, arena, orc, sel):
    """Train on 2^14 labelled blocks, evaluate on 2^12 held-out blocks: the
    network's picks (with the 2% fallback) stay within 3% of the exhaustive
    footprint while deciding most blocks without the exhaustive pass, and
    beat the best single format for the whole column."""
    ntr, nte = 1 << 14, 1 << 12
    dtr, _, sztr, ftr = _dataset(ms, arena, orc, sel, 21, ntr)
    dte, _, szte, fte = _dataset(ms, arena, orc, sel, 99, nte)
    m = sel.Mlp(seed=1, max_batch=4096)
    try:
        curve = m.train(arena, ftr, sztr, ntr, steps=600, batch=1024, lr=3e-3)
        assert curve[-20:].mean() < 0.25 * curve[:5].mean()
        ch, nf, _ = m.choose(arena, fte, nte, margin_log2=float(np.log2(1.02)))
        n_fallback = int(sel.to_host(nf, 1, np.uint64)[0])
        sel.resolve(dte, nte, ch)
        learned = sel.footprint(arena, szte, ch, nte)
        best, _ = sel.argmin(arena, szte, nte)
        exhaustive = sel.footprint(arena, szte, best, nte)
        sizes = sel.to_host(szte, nte * 5, np.uint32).reshape(nte, 5).astype(np.int64)
        single = sizes.sum(0).min()
        assert learned <= 1.03 * exhaustive, (learned, exhaustive)
        assert learned < single
        assert n_fallback < nte // 2
    finally:
        m.close()


def test_checkpoint_roundtrip(ms, arena, orc, sel, mixed):
    d, nblk, x = mixed
    _, sz = sel.analyze(arena, d, nblk)
    fd = sel.features(arena, d, nblk)
    a = sel.Mlp(seed=2, max_batch=256)
    b = sel.Mlp(seed=3, max_batch=256)
    try:
        a.train(arena, fd, sz, nblk, steps=20, batch=96)
        b.load_state(a.state())
        _, _, pa = a.choose(arena, fd, nblk, 0.0, want_pred=True)
        _, _, pb = b.choose(arena, fd, nblk, 0.0, want_pred=True)
        assert np.array_equal(sel.to_host(pa, nblk * 5, np.float32), sel.to_host(pb, nblk * 5, np.float32))
    finally:
        a.close()
        b.close()


# ---------------------------------------------------------------------------
# blockwise_individual_f and the exhaustive selector against the reference
# ---------------------------------------------------------------------------
def _gpu_container(sel, arena, x, choice):
    nblk = len(choice)
    d = sel.to_device(arena, np.ascontiguousarray(x, dtype=np.uint64))
    st, sz = sel.analyze(arena, d, nblk)
    cont = sel.Container(arena, d, nblk, st, sel.to_device(arena, np.asarray(choice, dtype=np.uint8)))
    codes = sel.to_host(cont.codes, nblk, np.uint8)
    return R.mask_container(cont.host_bytes(), choice), codes, sel.to_host(sz, nblk * 5, np.uint32).reshape(nblk, 5), \
        (d, st)


def _restricted_codes(sel, arena, nblk, sizes, d_st):
    """The GPU's exhaustive pick over the candidates the reference's container
    shares (static_vbp, dynamic_vbp, delta+dvbp, for+dvbp; first on ties), as
    format codes."""
    best = np.argmin(sizes[:, :4], axis=1).astype(np.uint8)
    d, st = d_st
    cont = sel.Container(arena, d, nblk, st, sel.to_device(arena, best))
    return sel.to_host(cont.codes, nblk, np.uint8)


def test_blockwise_container_matches_reference_golden(ms, arena, sel):
    from golden_util import load
    fx = load()
    if fx is None or "bwi/bytes" not in fx:
        pytest.skip("golden fixtures missing")
    got, codes, sizes, d_st = _gpu_container(sel, arena, fx["bwi/in"], fx["bwi/choice"])
    assert np.array_equal(codes, fx["bwi/codes"])
    assert np.array_equal(got, fx["bwi/bytes"])
    want = np.array([R.shared_code(int(c)) for c in fx["bwi/exhaustive"]])
    mine = _restricted_codes(sel, arena, len(want), sizes, d_st)
    shared = want >= 0
    assert shared.sum() >= 40
    assert np.array_equal(mine[shared], want[shared])


def test_blockwise_container_and_exhaustive_vs_reference_live(ms, arena, orc, ref, sel):
    """4096 device-generated blocks of the four families: the GPU container
    for random shared picks equals the reference's container byte for byte,
    and the GPU's exhaustive choice agrees with the reference's selector
    wherever the latter picks a shared format."""
    if ref.isa != 512:
        pytest.skip("the reference's AVX2 layouts differ from the device's")
    nblk = 4096
    d = sel.gen(arena, 29, nblk, 8, orc.zipf_table(1.2, 1 << 20))
    x = sel.to_host(d, nblk * sel.BLOCK, np.uint64)
    choice = np.random.default_rng(5).integers(0, 4, nblk).astype(np.uint8)
    got, codes, sizes, d_st = _gpu_container(sel, arena, x, choice)
    assert np.array_equal(got, R.mask_container(ref.bwi_compress(x, codes), choice))
    want = np.array([R.shared_code(int(c)) for c in ref.exhaustive_choose(x)])
    mine = _restricted_codes(sel, arena, nblk, sizes, d_st)
    shared = want >= 0
    assert shared.sum() >= nblk // 4
    assert np.array_equal(mine[shared], want[shared])
