"""Staged leaf screen (mb_screen) against the binary128 oracle's sums at the 7 offsets."""
import numpy as np
import pytest

from mertens_bound_b200 import hit_polish, k2, synth
from mertens_bound_b200._lib import K2Error

pytestmark = pytest.mark.gpu

SCORE_TOL = 2e-5    # |GPU score - exact score|: MUFU, FP32 products and sums over <= 256 terms


@pytest.fixture(scope="module")
def table(gpu, small_table):
    t = k2.ZeroTable.from_data(small_table)
    yield t
    t.close()


def oracle_scores(oracle, small_table, pts, k, ends, step):
    """max_m |S_m| after each stage, S_m = K2 over the stage's zeros at v + m step (exact 64.64)."""
    st = hit_polish._fixed(step)
    P = pts.shape[0]
    out = np.zeros((P, len(ends)))
    vals = np.zeros((7, len(ends), P))
    for mi, m in enumerate(range(-3, 4)):
        v = [(int(a) << 64 | int(b)) + m * st for a, b in pts]
        c = synth.Candidates(np.array([x >> 64 for x in v], dtype=np.uint64),
                             np.array([x & ((1 << 64) - 1) for x in v], dtype=np.uint64), np.zeros(P))
        for s, e in enumerate(ends):
            hi, _ = oracle.k2(c, small_table, k, e)
            vals[mi, s] = hi[:, 0]
    for s in range(len(ends)):
        out[:, s] = np.max(np.abs(vals[:, s, :]), axis=0)
    return out


def points(P, seed):
    c = synth.make_candidates(P, seed=seed)
    return np.stack([c.v_int, c.v_frac], axis=1).astype(np.uint64)


@pytest.mark.parametrize("stages", [hit_polish.SCREEN_GPU, hit_polish.SCREEN_CPU])
def test_screen_scores_vs_oracle(table, small_table, oracle, stages):
    pts = points(384, seed=21)
    k, step = 3e-9, hit_polish.SCREEN_STEP
    ends, _ = stages
    want = oracle_scores(oracle, small_table, pts, k, ends, step)
    # thresholds that pass about half the leaves at each stage, so every stage is reached
    thr = tuple(float(np.quantile(want[:, s], 0.35)) for s in range(len(ends)))
    r = hit_polish.screen_leaves(table, pts, k, (ends, thr), step, all_scores=True)
    got = r.scores
    reached = got >= 0
    assert reached[:, 0].all()
    assert np.max(np.abs(got[reached] - want[reached])) <= SCORE_TOL
    # stage s is reached exactly when every earlier stage passed (on the GPU's scores)
    for s in range(1, len(ends)):
        passed = np.all(got[:, :s] >= np.array(thr[:s], dtype=np.float32), axis=1)
        assert np.array_equal(reached[:, s], passed)
    # hits: the leaves that passed every stage, ascending, with their scores
    allpass = np.all(got >= np.array(thr, dtype=np.float32), axis=1)
    assert np.array_equal(r.hits, np.flatnonzero(allpass))
    assert np.array_equal(r.hit_scores, got[r.hits])
    # decisions agree with the exact sums away from the thresholds
    exact_pass = np.all(want >= np.array(thr), axis=1)
    margin = np.min(np.abs(want - np.array(thr)), axis=1)
    clear = margin > SCORE_TOL
    assert np.array_equal(allpass[clear], exact_pass[clear])
    assert 0 < allpass.sum() < len(pts)


def test_screen_capacity_and_args(table):
    pts = points(2048, seed=22)
    r = hit_polish.screen_leaves(table, pts, stages=((64,), (0.0,)))
    assert len(r.hits) == 2048 and r.scores is None
    with pytest.raises(K2Error, match="MB_ERR_CAPACITY"):
        hit_polish.screen_leaves(table, pts, stages=((64,), (0.0,)), max_hits=100)
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        hit_polish.screen_leaves(table, pts, stages=((128, 64), (0.1, 0.2)))
    with pytest.raises(K2Error, match="MB_ERR_ARG"):
        hit_polish.screen_leaves(table, pts, stages=((2048,), (0.1,)))
    e = hit_polish.screen_leaves(table, pts[:0])
    assert len(e.hits) == 0


def test_screen_ragged_batch(table):
    """A leaf count that is not a multiple of the CTA size: the tail CTA's idle lanes."""
    pts = points(1000, seed=23)
    a = hit_polish.screen_leaves(table, pts, stages=((64, 128), (0.2, 0.3)), all_scores=True)
    b = hit_polish.screen_leaves(table, pts[:999], stages=((64, 128), (0.2, 0.3)), all_scores=True)
    assert np.array_equal(a.scores[:999], b.scores)


def test_screen_device_pointers(table):
    """mb_screen_dev on device leaves gives the host call's scores, hit set and per-hit scores
    (hits in arbitrary order on the device), twice in a row on the same buffers."""
    import torch
    pts = points(3000, seed=29)
    stages = ((64, 128, 256), (0.2, 0.3, 0.35))
    host = hit_polish.screen_leaves(table, pts, stages=stages, all_scores=True)
    assert 0 < len(host.hits) < len(pts)
    dev = torch.device("cuda", 0)
    vi = torch.from_numpy(pts[:, 0].view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(pts[:, 1].view(np.int64).copy()).to(dev)
    cap = len(pts)
    hits = torch.empty(cap, dtype=torch.int64, device=dev)
    hsc = torch.empty(cap, 3, dtype=torch.float32, device=dev)
    cnt = torch.empty(1, dtype=torch.int64, device=dev)
    sc = torch.empty(len(pts), 3, dtype=torch.float32, device=dev)
    for _ in range(2):
        hit_polish.screen_leaves_dev(table, vi.data_ptr(), vf.data_ptr(), len(pts), hits.data_ptr(),
                                     hsc.data_ptr(), cnt.data_ptr(), cap, stages=stages, d_scores=sc.data_ptr())
        torch.cuda.synchronize(dev)
        n = int(cnt.item())
        assert n == len(host.hits)
        order = np.argsort(hits[:n].cpu().numpy())
        assert np.array_equal(hits[:n].cpu().numpy()[order], host.hits)
        assert np.array_equal(hsc[:n].cpu().numpy()[order], host.hit_scores)
        assert np.array_equal(sc.cpu().numpy(), host.scores)


def test_screen_device_edges(table):
    """mb_screen_dev: no leaves gives a zero count; a hit buffer smaller than the hits keeps that
    many (a subset of the host call's hits) and reports the full count; argument errors raise."""
    import torch
    dev = torch.device("cuda", 0)
    pts = points(2000, seed=31)
    stages = ((64, 128, 256), (0.2, 0.3, 0.35))
    host = hit_polish.screen_leaves(table, pts, stages=stages)
    assert len(host.hits) > 3
    vi = torch.from_numpy(pts[:, 0].view(np.int64).copy()).to(dev)
    vf = torch.from_numpy(pts[:, 1].view(np.int64).copy()).to(dev)
    hits = torch.empty(2, dtype=torch.int64, device=dev)
    hsc = torch.empty(2, 3, dtype=torch.float32, device=dev)
    cnt = torch.full((1,), 7, dtype=torch.int64, device=dev)
    hit_polish.screen_leaves_dev(table, vi.data_ptr(), vf.data_ptr(), 0, hits.data_ptr(), hsc.data_ptr(),
                                 cnt.data_ptr(), 2, stages=stages)
    torch.cuda.synchronize(dev)
    assert int(cnt.item()) == 0
    hit_polish.screen_leaves_dev(table, vi.data_ptr(), vf.data_ptr(), len(pts), hits.data_ptr(), hsc.data_ptr(),
                                 cnt.data_ptr(), 2, stages=stages)
    torch.cuda.synchronize(dev)
    assert int(cnt.item()) == len(host.hits)
    assert set(hits.cpu().numpy().tolist()) <= set(host.hits.tolist())
    with pytest.raises(K2Error):
        hit_polish.screen_leaves_dev(table, vi.data_ptr(), vf.data_ptr(), len(pts), hits.data_ptr(),
                                     hsc.data_ptr(), cnt.data_ptr(), 2, stages=((128, 64), (0.1, 0.2)))
    with pytest.raises(K2Error):
        hit_polish.screen_leaves_dev(table, vi.data_ptr(), vf.data_ptr(), len(pts), 0, 0, cnt.data_ptr(), 2,
                                     stages=stages)
