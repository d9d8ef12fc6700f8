"""GPU checks of the learned orientation proposal against its CPU oracle:
input builders, forward pass, loss and every parameter gradient; the gated
packing loop against the plain one.  Run on a B200 with `pytest -m gpu`."""
import numpy as np
import pytest

from oracle import psb_proposal_oracle as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prop_mod(gpu_core):
    from psacking_b200 import proposal
    return proposal


def test_item_grids_match_oracle(prop_mod):
    from psacking_b200 import workloads
    from psacking_b200.rotations import orientation_maps
    maps = orientation_maps(24)
    items = workloads.config2_items(7)[:5] + [np.ones((40, 3, 33), np.int32), np.ones((1, 1, 1), np.int32)]
    got = prop_mod.item_grids(items, maps).cpu().numpy().reshape(len(items), 24, 32, 32, 32)
    for k, it in enumerate(items):
        want = P.oriented_grids(it, maps)
        assert np.array_equal(got[k], want), k


def test_height_map_matches_oracle(prop_mod):
    import torch
    rng = np.random.default_rng(1)
    for shape in [(128, 128, 128), (240, 123, 100), (40, 17, 9)]:
        t = np.zeros(shape, np.int32)
        for _ in range(12):
            lo = [int(rng.integers(0, s)) for s in shape]
            hi = [min(s, l + int(rng.integers(1, max(2, s // 3)))) for s, l in zip(shape, lo)]
            t[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] = int(rng.integers(1, 9))
        dt = torch.from_numpy(t).cuda()
        out = torch.empty(1024, dtype=torch.float32, device="cuda")
        prop_mod.check(prop_mod.lib().psb_height_map(
            prop_mod.ctypes.c_void_p(dt.data_ptr()), *shape, prop_mod.ctypes.c_void_p(out.data_ptr())))
        assert np.allclose(out.cpu().numpy(), P.height_map(t).ravel(), rtol=0, atol=2e-7)


def _batch(rng, B):
    grids = (rng.random((B, 24, 32, 32, 32)) < 0.06).astype(np.float32)
    grids[:, :, 16:] = 0.0
    hm = rng.random((B, 32, 32)).astype(np.float32)
    mask = np.ones((B, 24), np.float32)
    mask[1, 10:] = 0
    target = np.zeros((B, 24), np.float32)
    target[0, [2, 5, 9]] = [0.5, 0.25, 0.25]
    target[1, 3] = 1.0
    if B > 2:
        target[2] = 0.0  # an item without a target is left out of the mean
    return grids, hm, mask, target


def test_forward_backward_match_oracle(prop_mod):
    import torch
    rng = np.random.default_rng(11)
    B = 3
    flat = P.init_params(2)
    d = P.unpack(flat.astype(np.float64))
    for name, shape in P.LAYERS:
        if name.endswith(".b"):
            d[name] = rng.normal(0.0, 0.05, shape)
    flat = P.pack(d).astype(np.float32)
    grids, hm, mask, target = _batch(rng, B)
    prop = prop_mod.Proposal(flat)
    tg = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in
          (grids.reshape(B * 24, -1), hm.reshape(B, -1), mask, target)]
    logits, loss = prop.run(*tg)
    g = prop.grads()
    want_loss, want_logit, want_g = P.loss_and_grads(flat, grids, hm, target.astype(np.float64),
                                                      mask.astype(np.float64))
    lg = logits.cpu().numpy()
    assert np.allclose(lg, want_logit, rtol=1e-4, atol=1e-4 * np.abs(want_logit).max())
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    off = 0
    gmax = np.abs(want_g).max()
    for name, shape in P.LAYERS:
        n = int(np.prod(shape))
        a, b = g[off:off + n], want_g[off:off + n]
        # per layer, relative to its largest gradient; the head bias has an
        # exact gradient of 0 (softmax is shift invariant), hence the floor
        scale = max(np.abs(b).max(), 1e-3 * gmax)
        assert np.abs(a - b).max() <= 2e-3 * scale, (name, np.abs(a - b).max(), scale)
        off += n
    prop.close()


def test_adam_reduces_loss(prop_mod):
    import torch
    rng = np.random.default_rng(5)
    B = 4
    grids, hm, mask, target = _batch(rng, B)
    target[3, 7] = 1.0
    prop = prop_mod.Proposal(prop_mod.init_params(3))
    tg = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in
          (grids.reshape(B * 24, -1), hm.reshape(B, -1), mask, target)]
    losses = []
    for _ in range(30):
        _, loss = prop.run(*tg, want_logits=False)
        losses.append(loss)
        prop.adam(1e-3)
    assert losses[-1] < 0.5 * losses[0], losses[::5]
    prop.close()


def test_gated_loop_without_gating_equals_plain(prop_mod):
    """top-k = 24 (every orientation kept) and a margin above 1 (always the
    full sweep) must reproduce the plain run exactly."""
    from psacking_b200 import workloads
    from psacking_b200.rotations import orientation_maps
    maps = orientation_maps(24)
    seq = prop_mod.sorted_by_volume(workloads.config2_items(3)[:12])
    tray = prop_mod.Tray((96, 96, 96))
    prop = prop_mod.Proposal(prop_mod.init_params(1))
    plain, ptray, _ = tray.pack(seq, maps)
    key = [(r.found, r.x, r.y, r.z, r.orientation, r.score) for r in plain]
    for topk, margin in [(24, 0.0), (4, 1.01)]:
        res, t2, stats = tray.pack(seq, maps, prop=prop, topk=topk, margin=margin)
        assert [(r.found, r.x, r.y, r.z, r.orientation, r.score) for r in res] == key
        assert np.array_equal(t2, ptray)
        assert stats[0] == len(seq)
        assert stats[1] == (len(seq) if margin > 1 else 0)
    # a real gate: every placement is still a valid, non-overlapping one
    res, t3, stats = tray.pack(seq, maps, prop=prop, topk=2, margin=0.0)
    assert stats[1] == 0
    assert sum(r.found for r in res) >= 1
    assert int((t3 > 0).sum()) == sum(int((s > 0).sum()) for s, r in zip(seq, res) if r.found)
    prop.close()
    tray.close()


def test_trained_proposal_gains_over_untrained(prop_mod):
    """What the trained network buys, on the held-out config-2 seeds 0..9
    (training used seeds 10000+): a best orientation lands in its top-k far
    more often than with the untrained network, and the gated loop keeps the
    final density within 1 percentage point of the plain method while
    searching a fraction of the orientations."""
    import json
    from psacking_b200 import train_proposal as TP
    if not prop_mod.WEIGHTS.exists():
        pytest.fail("psacking_b200/proposal_weights.npz is missing (python -m psacking_b200.train_proposal)")
    with np.load(prop_mod.WEIGHTS) as z:
        topk, margin = int(z["topk"]), float(z["margin"])
    trained = prop_mod.load()
    untrained = prop_mod.Proposal(prop_mod.init_params(0))
    recs = prop_mod.generate(range(3))
    r_t = prop_mod.topk_recall(trained, recs, k=topk)
    r_u = prop_mod.topk_recall(untrained, recs, k=topk)
    assert r_t >= r_u + 0.15, (r_t, r_u)
    ev = TP.evaluate(trained, seeds=tuple(range(10)), topk=topk, margin=margin)
    print(json.dumps({k: v for k, v in ev.items() if k != "per_seed"}))
    assert ev["density_gap_pp"] <= 1.0, ev["density_gap_pp"]
    assert ev["fallback_rate"] < 0.2, ev["fallback_rate"]
    trained.close()
    untrained.close()
