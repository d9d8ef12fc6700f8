"""CPU oracle of the learned orientation proposal network (test infrastructure).

A float64 NumPy restatement of the network that psacking_b200's CUDA kernels
(psb_proposal.cuh) run in FP32 with BF16 weights: forward pass, masked softmax
cross-entropy against soft targets, and the analytic gradient of every
parameter.  The tests compare the GPU's logits, loss and gradients with this
module (the weights are rounded to BF16 here too, so both sides compute with
the same weight values), and check this module's analytic gradients against
central finite differences.  Only tests and the benchmark's checks import it.

The network has no counterpart in the reference (it is the learned-proposal
form of the placement search, an addition of this engine):

  item branch  (per orientation, 32^3 occupancy grid)
    conv3d 1->16, 16->32, 32->64, 64->64; kernel 3, stride 2, padding 1, ReLU
    -> 64 x 2^3 = 512 -> linear 512->64, ReLU
  tray branch  (per item, 32x32 pooled height map)
    linear 1024->64, ReLU
  head         (per orientation)
    [item 64 | tray 64] -> linear 128->64, ReLU -> linear 64->1 = logit
"""
from __future__ import annotations

import numpy as np

GRID = 32          # item grid side
HMAP = 32          # pooled height-map side
N_ORIENT = 24

# (name, shape) in the order of the flat parameter vector
CONV = [(1, 16), (16, 32), (32, 64), (64, 64)]
LAYERS = []
for i, (ci, co) in enumerate(CONV):
    LAYERS += [(f"c{i}.w", (co, ci, 27)), (f"c{i}.b", (co,))]
LAYERS += [("f1.w", (64, 512)), ("f1.b", (64,)),
           ("f2.w", (64, HMAP * HMAP)), ("f2.b", (64,)),
           ("h1.w", (64, 128)), ("h1.b", (64,)),
           ("h2.w", (1, 64)), ("h2.b", (1,))]


def n_params() -> int:
    return int(sum(np.prod(s) for _, s in LAYERS))


def unpack(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in LAYERS:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    return out


def pack(d: dict) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in LAYERS])


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, np.float32).copy()
    u = f.view(np.uint32)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def weights_as_used(flat: np.ndarray) -> dict:
    """Weights rounded to BF16 (the kernels' storage), biases kept FP32."""
    p = unpack(np.asarray(flat, np.float32).astype(np.float64))
    return {k: (bf16_round(v) if k.endswith(".w") else v) for k, v in p.items()}


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation (the training script's starting point)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in LAYERS:
        if name.endswith(".b"):
            d[name] = np.zeros(shape)
        else:
            fan_in = int(np.prod(shape[1:]))
            d[name] = rng.normal(0.0, np.sqrt(2.0 / fan_in), shape)
    return pack(d).astype(np.float32)


# --------------------------------------------------------------------------
# layers (float64)
# --------------------------------------------------------------------------
def _taps():
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                yield kd * 9 + kh * 3 + kw, kd, kh, kw


def conv_fwd(x, w, b):
    """x [S, Ci, D, D, D], w [Co, Ci, 27] -> [S, Co, D/2, D/2, D/2]; stride 2, pad 1."""
    S, Ci, D = x.shape[0], x.shape[1], x.shape[2]
    Do = D // 2
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    out = np.zeros((S, w.shape[0], Do, Do, Do)) + b[None, :, None, None, None]
    for t, kd, kh, kw in _taps():
        xt = xp[:, :, kd:kd + 2 * Do:2, kh:kh + 2 * Do:2, kw:kw + 2 * Do:2]
        out += np.einsum("scdhw,oc->sodhw", xt, w[:, :, t], optimize=True)
    return out


def conv_bwd(x, w, dy):
    """Gradients of conv_fwd: (dx, dw, db)."""
    S, Ci, D = x.shape[0], x.shape[1], x.shape[2]
    Do = D // 2
    xp = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1), (1, 1)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for t, kd, kh, kw in _taps():
        xt = xp[:, :, kd:kd + 2 * Do:2, kh:kh + 2 * Do:2, kw:kw + 2 * Do:2]
        dw[:, :, t] = np.einsum("sodhw,scdhw->oc", dy, xt, optimize=True)
        dxp[:, :, kd:kd + 2 * Do:2, kh:kh + 2 * Do:2, kw:kw + 2 * Do:2] += np.einsum(
            "sodhw,oc->scdhw", dy, w[:, :, t], optimize=True)
    db = dy.sum(axis=(0, 2, 3, 4))
    return dxp[:, :, 1:-1, 1:-1, 1:-1], dw, db


def relu(x):
    return np.maximum(x, 0.0)


def forward(p: dict, grids: np.ndarray, hmaps: np.ndarray):
    """grids [B, 24, 32, 32, 32], hmaps [B, 32, 32] -> logits [B, 24] and the
    activations the backward pass needs."""
    B = grids.shape[0]
    S = B * N_ORIENT
    a = [grids.reshape(S, 1, GRID, GRID, GRID).astype(np.float64)]
    for i in range(4):
        a.append(relu(conv_fwd(a[-1], p[f"c{i}.w"], p[f"c{i}.b"])))
    a4 = a[4].reshape(S, 512)
    f1 = relu(a4 @ p["f1.w"].T + p["f1.b"])
    hm = hmaps.reshape(B, HMAP * HMAP).astype(np.float64)
    t = relu(hm @ p["f2.w"].T + p["f2.b"])
    hin = np.concatenate([f1, np.repeat(t, N_ORIENT, axis=0)], axis=1)
    h1 = relu(hin @ p["h1.w"].T + p["h1.b"])
    logit = (h1 @ p["h2.w"].T + p["h2.b"]).reshape(B, N_ORIENT)
    cache = dict(a=a, a4=a4, f1=f1, hm=hm, t=t, hin=hin, h1=h1)
    return logit, cache


def loss_and_dlogit(logit, target, mask):
    """Masked softmax cross-entropy, mean over items with a valid target:
    loss = -sum_o q_o log p_o, p = softmax over the unmasked orientations."""
    z = np.where(mask > 0, logit, -np.inf)
    zmax = np.max(z, axis=1, keepdims=True)
    zmax = np.where(np.isfinite(zmax), zmax, 0.0)
    e = np.where(mask > 0, np.exp(z - zmax), 0.0)
    s = e.sum(axis=1, keepdims=True)
    p = np.where(s > 0, e / np.where(s > 0, s, 1.0), 0.0)
    has = (target.sum(axis=1) > 0) & (mask.sum(axis=1) > 0)
    nb = max(1, int(has.sum()))
    logp = np.where(mask > 0, z - zmax - np.log(np.where(s > 0, s, 1.0)), 0.0)
    loss = -(np.where(has[:, None], target * logp, 0.0)).sum() / nb
    dlogit = np.where(has[:, None] & (mask > 0), (p * target.sum(axis=1, keepdims=True) - target) / nb, 0.0)
    return loss, dlogit


def backward(p: dict, cache: dict, dlogit: np.ndarray) -> dict:
    B = dlogit.shape[0]
    S = B * N_ORIENT
    g = {}
    dl = dlogit.reshape(S, 1)
    g["h2.w"] = dl.T @ cache["h1"]
    g["h2.b"] = dl.sum(axis=0)
    dh1 = (dl @ p["h2.w"]) * (cache["h1"] > 0)
    g["h1.w"] = dh1.T @ cache["hin"]
    g["h1.b"] = dh1.sum(axis=0)
    dhin = dh1 @ p["h1.w"]
    df1 = dhin[:, :64] * (cache["f1"] > 0)
    dt = dhin[:, 64:].reshape(B, N_ORIENT, 64).sum(axis=1) * (cache["t"] > 0)
    g["f2.w"] = dt.T @ cache["hm"]
    g["f2.b"] = dt.sum(axis=0)
    g["f1.w"] = df1.T @ cache["a4"]
    g["f1.b"] = df1.sum(axis=0)
    da = (df1 @ p["f1.w"]).reshape(cache["a"][4].shape) * (cache["a"][4] > 0)
    for i in (3, 2, 1, 0):
        dx, dw, db = conv_bwd(cache["a"][i], p[f"c{i}.w"], da)
        g[f"c{i}.w"], g[f"c{i}.b"] = dw, db
        if i > 0:
            da = dx * (cache["a"][i] > 0)
    return g


def loss_and_grads(flat, grids, hmaps, target, mask):
    """Loss and the gradient of every parameter (flat, in LAYERS order), with
    the weights rounded to BF16 as the kernels use them."""
    p = weights_as_used(flat)
    logit, cache = forward(p, grids, hmaps)
    loss, dl = loss_and_dlogit(logit, target, mask)
    g = backward(p, cache, dl)
    return loss, logit, pack(g)


# --------------------------------------------------------------------------
# inputs: oriented item grids, pooled height maps, soft targets
# --------------------------------------------------------------------------
def item_grid(item: np.ndarray) -> np.ndarray:
    """The item's occupancy embedded at the origin of a 32^3 grid, each axis
    scaled by s = ceil(max extent / 32): a cell is the fraction of occupied
    voxels of its s^3 block."""
    e = item.shape
    s = max(1, -(-max(e) // GRID))
    g = np.zeros((GRID, GRID, GRID))
    idx = np.argwhere(item > 0)
    if len(idx):
        c = idx // s
        np.add.at(g, (c[:, 0], c[:, 1], c[:, 2]), 1.0 / s ** 3)
    return g


def height_map(tray: np.ndarray) -> np.ndarray:
    """Per (x, y): 1 + the highest occupied z (0 for an empty column), over nz,
    averaged over ceil(nx/32) x ceil(ny/32) blocks into 32 x 32 (blocks past
    the tray edge average the columns they hold; empty blocks are 0)."""
    nx, ny, nz = tray.shape
    occ = tray > 0
    top = np.where(occ.any(axis=2), nz - np.argmax(occ[:, :, ::-1], axis=2), 0).astype(np.float64) / nz
    bx, by = -(-nx // HMAP), -(-ny // HMAP)
    out = np.zeros((HMAP, HMAP))
    for i in range(HMAP):
        for j in range(HMAP):
            blk = top[i * bx:(i + 1) * bx, j * by:(j + 1) * by]
            if blk.size:
                out[i, j] = blk.mean()
    return out


def soft_target(found, score, temperature: float) -> np.ndarray:
    """Target distribution over orientations: exp(-(s_o - s_min) / T) over the
    orientations that found a placement, normalised; all zero when none did."""
    found = np.asarray(found, bool)
    score = np.asarray(score, np.float64)
    q = np.zeros(len(found))
    if found.any():
        m = score[found].min()
        q[found] = np.exp(-(score[found] - m) / temperature)
        q /= q.sum()
    return q


def oriented_grids(item: np.ndarray, maps: np.ndarray) -> np.ndarray:
    """[n_orient, 32, 32, 32]: the item's base grid turned by each map
    (src_axis[3], flip[3]) within the grid extent G_a = ceil(e_a / s)."""
    base = item_grid(item)
    s = max(1, -(-max(item.shape) // GRID))
    G = [-(-e // s) for e in item.shape]
    out = np.zeros((len(maps), GRID, GRID, GRID))
    for o, row in enumerate(maps):
        axes, flips = list(row[:3]), list(row[3:])
        sub = base[:G[0], :G[1], :G[2]]
        g = np.transpose(sub, axes)
        sl = tuple(slice(None, None, -1) if flips[a] else slice(None) for a in range(3))
        g = g[sl]
        out[o, :g.shape[0], :g.shape[1], :g.shape[2]] = g
    return out
