"""CPU checks of the proposal network's oracle: analytic gradients against
central finite differences, and the input builders' definitions."""
import numpy as np

from oracle import psb_proposal_oracle as P


def test_param_count():
    assert P.n_params() == 287073


def test_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    B = 2
    flat = P.init_params(5)
    # non-zero biases keep pre-activations off the ReLU kink (with zero
    # biases, empty regions of the grid sit exactly at it)
    d = P.unpack(flat.astype(np.float64))
    for name, shape in P.LAYERS:
        if name.endswith(".b"):
            d[name] = rng.normal(0.0, 0.05, shape)
    flat = P.pack(d).astype(np.float32)
    grids = (rng.random((B, 24, 32, 32, 32)) < 0.08).astype(np.float64)
    hm = rng.random((B, 32, 32))
    mask = np.ones((B, 24))
    mask[1, 6:] = 0
    target = np.zeros((B, 24))
    target[0, [1, 4]] = [0.75, 0.25]
    target[1, 2] = 1.0
    loss, _, g = P.loss_and_grads(flat, grids, hm, target, mask)
    assert np.isfinite(loss) and loss > 0
    used = P.pack(P.weights_as_used(flat))

    def L(v):
        logit, _ = P.forward(P.unpack(v), grids, hm)
        return P.loss_and_dlogit(logit, target, mask)[0]

    # one weight of every layer plus a few random ones
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in P.LAYERS])
    idx = list(offs[:-1] + 1) + list(rng.choice(len(used), 4, replace=False))
    idx = [i for i in idx if i < len(used)]
    for i in idx:
        # a small step: with binary inputs many pre-activations sit near the
        # ReLU kink, and a large step would cross some of them
        e = 1e-7
        vp, vm = used.copy(), used.copy()
        vp[i] += e
        vm[i] -= e
        num = (L(vp) - L(vm)) / (2 * e)
        assert abs(num - g[i]) <= 1e-7 + 1e-4 * abs(num), (i, num, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.0000001, 65504.0], np.float32)
    r = P.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0078125 and r[3] == -3.0


def test_item_grid_and_orientations():
    item = np.zeros((40, 7, 3), np.int32)
    item[0:40, 0, 0] = 1
    item[5, 6, 2] = 1
    g = P.item_grid(item)          # s = 2
    assert g[0, 0, 0] == 2 / 8 and g[2, 3, 1] == 1 / 8 and g.sum() == 41 / 8
    maps = np.array([[0, 1, 2, 0, 0, 0], [2, 1, 0, 1, 0, 0]], np.int32)
    og = P.oriented_grids(item, maps)
    assert np.array_equal(og[0], g)
    # map 1: oriented axis 0 <- base axis 2 flipped (G = 2), axis 2 <- base axis 0
    assert og[1][1, 0, 0] == g[0, 0, 0] and og[1][0, 3, 2] == g[2, 3, 1]


def test_height_map():
    t = np.zeros((64, 40, 10), np.int32)
    t[0:2, 0:2, 0:5] = 1
    h = P.height_map(t)
    # blocks of 2 x 2 columns (ceil(64/32), ceil(40/32))
    assert h[0, 0] == 0.5 and h[0, 1] == 0.0
