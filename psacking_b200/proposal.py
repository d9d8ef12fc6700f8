"""Learned orientation proposal: training data from the plain method, training
with the engine's own forward/backward kernels, and the gated packing loop.

The network (psacking_b200/csrc/psb_proposal.cuh) reads an item turned into
each of its 24 orientations (32^3 occupancy grids) and the tray's 32x32
pooled height map, and gives every orientation a logit.  The packing loop
then searches only the k best orientations exactly, or all 24 when the
top-k softmax mass is below a margin.  The plain method stays the judge:
its per-orientation results are the training targets and its densities the
reference the tests compare against.

Everything here drives the C ABI (include/psb200.h) through ctypes; device
buffers are torch tensors (memory only: the arithmetic is the engine's).
Nothing here has a counterpart in the reference.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from pathlib import Path
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from .rotations import orientation_maps

PKG = Path(__file__).resolve().parent
GRID3 = 32 ** 3
HMAP = 32 * 32
N_ORIENT = 24
WEIGHTS = PKG / "proposal_weights.npz"


class PsbResult(ctypes.Structure):
    _fields_ = [("x", ctypes.c_int32), ("y", ctypes.c_int32), ("z", ctypes.c_int32), ("found", ctypes.c_int32),
                ("score", ctypes.c_double), ("orientation", ctypes.c_int32), ("diag", ctypes.c_uint32),
                ("n_candidates", ctypes.c_int32), ("err_ratio", ctypes.c_float)]


_LIB = None


def lib():
    """The engine library (the same one psacking_b200._core links)."""
    global _LIB
    if _LIB is None:
        from . import _core  # noqa: F401  (fails loudly without the extension)
        L = ctypes.CDLL(str(PKG / "libpsb200.so"))
        L.psb_last_error.argtypes = [ctypes.c_char_p, ctypes.c_size_t]
        vp = ctypes.c_void_p
        L.psb_prop_forward_backward.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int, vp, ctypes.POINTER(ctypes.c_float)]
        L.psb_prop_adam_step.argtypes = [vp, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        L.psb_prop_set_params.argtypes = [vp, vp, ctypes.c_size_t]
        L.psb_prop_get_params.argtypes = [vp, vp, ctypes.c_size_t]
        L.psb_prop_get_grads.argtypes = [vp, vp, ctypes.c_size_t]
        L.psb_prop_item_grids.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int, vp]
        L.psb_prop_destroy.argtypes = [vp]
        L.psb_tray_destroy.argtypes = [vp]
        L.psb_tray_set.argtypes = [vp, vp, vp]
        L.psb_tray_get.argtypes = [vp, vp, vp]
        L.psb_pack_stage.argtypes = [vp, vp, vp, ctypes.c_int]
        L.psb_pack_staged.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int32, vp, vp]
        L.psb_pack_staged_detail.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int32, vp, vp, vp, vp]
        L.psb_pack_staged_prop.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int32, ctypes.c_int,
                                           ctypes.c_float, vp, vp, vp]
        _LIB = L
    return _LIB


def check(st: int) -> None:
    if st != 0:
        buf = ctypes.create_string_buffer(4096)
        lib().psb_last_error(buf, 4096)
        raise RuntimeError(f"psb error {st}: {buf.value.decode()}")


def n_params() -> int:
    n = ctypes.c_size_t()
    check(lib().psb_prop_num_params(ctypes.byref(n)))
    return int(n.value)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, in the network's layer order."""
    rng = np.random.default_rng(seed)
    shapes = []
    for ci, co in [(1, 16), (16, 32), (32, 64), (64, 64)]:
        shapes += [(co, ci * 27), (co,)]
    shapes += [(64, 512), (64,), (64, HMAP), (64,), (64, 128), (64,), (1, 64), (1,)]
    parts = []
    for sh in shapes:
        if len(sh) == 1:
            parts.append(np.zeros(sh))
        else:
            parts.append(rng.normal(0.0, np.sqrt(2.0 / sh[1]), sh).ravel())
    out = np.concatenate(parts).astype(np.float32)
    assert out.size == n_params()
    return out


def _ptrs(arrays: Sequence[np.ndarray]):
    arr = (ctypes.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    dims = np.ascontiguousarray(np.array([a.shape for a in arrays], np.int32).reshape(-1))
    return arr, dims


class Proposal:
    """The network on one GPU: parameters, Adam state, work buffers."""

    def __init__(self, params: Optional[np.ndarray] = None):
        h = ctypes.c_void_p()
        check(lib().psb_prop_create(ctypes.byref(h)))
        self.h = h
        self.set_params(init_params() if params is None else params)

    def close(self):
        if self.h:
            lib().psb_prop_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(lib().psb_prop_set_params(self.h, p.ctypes.data, p.size))

    def params(self) -> np.ndarray:
        out = np.zeros(n_params(), np.float32)
        check(lib().psb_prop_get_params(self.h, out.ctypes.data, out.size))
        return out

    def grads(self) -> np.ndarray:
        out = np.zeros(n_params(), np.float32)
        check(lib().psb_prop_get_grads(self.h, out.ctypes.data, out.size))
        return out

    def run(self, grids, hmaps, mask=None, target=None, want_logits=True):
        """grids [B*24, 32^3], hmaps [B, 1024], mask/target [B, 24] (torch
        CUDA float32).  Returns (logits [B, 24] or None, loss or None)."""
        import torch
        B = hmaps.shape[0]
        logits = torch.empty((B, N_ORIENT), dtype=torch.float32, device=hmaps.device) if want_logits else None
        loss = ctypes.c_float(0.0)
        check(lib().psb_prop_forward_backward(
            self.h, grids.data_ptr(), hmaps.data_ptr(), mask.data_ptr() if mask is not None else None,
            target.data_ptr() if target is not None else None, B, logits.data_ptr() if logits is not None else None,
            ctypes.byref(loss)))
        return logits, (float(loss.value) if target is not None else None)

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8) -> None:
        check(lib().psb_prop_adam_step(self.h, lr, beta1, beta2, eps))


def item_grids(items: Sequence[np.ndarray], maps: Optional[np.ndarray] = None, device=None):
    """Oriented 32^3 grids of items, on the GPU: [len(items) * n_orient, 32^3]."""
    import torch
    maps = orientation_maps(N_ORIENT) if maps is None else np.ascontiguousarray(maps, np.int32)
    items = [np.ascontiguousarray(i, np.int32) for i in items]
    out = torch.empty((len(items) * len(maps), GRID3), dtype=torch.float32, device=device or "cuda")
    arr, dims = _ptrs(items)
    check(lib().psb_prop_item_grids(arr, dims.ctypes.data, len(items), maps.ctypes.data, len(maps), out.data_ptr()))
    return out


# --------------------------------------------------------------------------
# training data: the plain method's per-orientation results
# --------------------------------------------------------------------------
@dataclass
class Record:
    item: np.ndarray          # the item array (as packed: the run's order)
    hmap: np.ndarray          # [1024] pooled height map before the item
    found: np.ndarray         # [24] bool
    score: np.ndarray         # [24] float64
    fits: np.ndarray          # [24] bool: the orientation fits the tray


class Tray:
    """A device tray for plain / detailed / gated packing runs (empty start)."""

    def __init__(self, dims: Tuple[int, int, int]):
        self.dims = tuple(int(d) for d in dims)
        h = ctypes.c_void_p()
        check(lib().psb_tray_create(*self.dims, ctypes.byref(h)))
        self.h = h
        self.empty = np.zeros(self.dims, np.int32)

    def close(self):
        if self.h:
            lib().psb_tray_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stage(self, seq):
        check(lib().psb_tray_set(self.h, self.empty.ctypes.data, None))
        arr, dims = _ptrs(seq)
        check(lib().psb_pack_stage(self.h, arr, dims.ctypes.data, len(seq)))

    def pack_detail(self, seq: Sequence[np.ndarray], maps: np.ndarray, interlock: bool = False):
        """Plain run; returns (placements, per-orientation results, height maps, final tray)."""
        self._stage(seq)
        n, no = len(seq), len(maps)
        res = (PsbResult * n)()
        per = (PsbResult * (n * no))()
        hm = np.zeros((n, HMAP), np.float32)
        final = np.zeros(self.dims, np.int32)
        check(lib().psb_pack_staged_detail(self.h, maps.ctypes.data, no, int(interlock), 0, res, final.ctypes.data,
                                           per, hm.ctypes.data))
        return list(res), list(per), hm, final

    def pack(self, seq, maps, interlock=False, prop: Optional[Proposal] = None, topk: int = 4,
             margin: float = 0.0):
        """Plain run (prop None) or the gated run; returns (placements, final
        tray, [items gated, fallbacks])."""
        self._stage(seq)
        n, no = len(seq), len(maps)
        res = (PsbResult * n)()
        final = np.zeros(self.dims, np.int32)
        stats = np.zeros(2, np.int32)
        if prop is None:
            check(lib().psb_pack_staged(self.h, maps.ctypes.data, no, int(interlock), 0, res, final.ctypes.data))
        else:
            check(lib().psb_pack_staged_prop(self.h, prop.h, maps.ctypes.data, no, int(interlock), 0, int(topk),
                                             float(margin), res, final.ctypes.data, stats.ctypes.data))
        return list(res), final, stats


def sorted_by_volume(items: Sequence[np.ndarray]) -> List[np.ndarray]:
    """The packer's order (packer.py:421-425: argsort of volumes, reversed)."""
    vols = [int(np.sum(i > 0)) for i in items]
    return [np.ascontiguousarray(items[i].astype(np.int32)) for i in np.argsort(vols)[::-1]]


def generate(seeds: Iterable[int], tray_dims=(128, 128, 128), make_items=None) -> List[Record]:
    """Run the plain method (24 orientations) on each seed's items and keep,
    for every item, its height map and every orientation's result."""
    from . import workloads
    make_items = make_items or workloads.config2_items
    maps = orientation_maps(N_ORIENT)
    tray = Tray(tray_dims)
    out = []
    try:
        for seed in seeds:
            seq = sorted_by_volume(make_items(seed))
            _, per, hm, _ = tray.pack_detail(seq, maps)
            for k, it in enumerate(seq):
                rs = per[k * N_ORIENT:(k + 1) * N_ORIENT]
                out.append(Record(it, hm[k].copy(), np.array([bool(r.found) for r in rs]),
                                  np.array([r.score for r in rs], np.float64),
                                  np.array([not (r.diag & 0x200) for r in rs])))
    finally:
        tray.close()
    return out


def target_of(rec: Record) -> np.ndarray:
    """Soft target over orientations: weight 2^-rank by score among the
    orientations that found a placement (equal scores share a rank, so an
    item's symmetric twins share the best weight); zero when none did."""
    q = np.zeros(N_ORIENT)
    if rec.found.any():
        s = np.round(rec.score[rec.found], 6)
        uniq = np.unique(s)
        rank = np.searchsorted(uniq, s)
        q[rec.found] = 0.5 ** rank
        q /= q.sum()
    return q


def best_set(rec: Record) -> np.ndarray:
    """Orientations achieving the plain method's best score."""
    if not rec.found.any():
        return np.zeros(N_ORIENT, bool)
    m = rec.score[rec.found].min()
    return rec.found & (rec.score == m)


def batch_tensors(recs: Sequence[Record], device="cuda"):
    import torch
    grids = item_grids([r.item for r in recs], device=device)
    hm = torch.from_numpy(np.stack([r.hmap for r in recs]).astype(np.float32)).to(device)
    mask = torch.from_numpy(np.stack([r.fits for r in recs]).astype(np.float32)).to(device)
    tgt = torch.from_numpy(np.stack([target_of(r) for r in recs]).astype(np.float32)).to(device)
    return grids, hm, mask, tgt


def topk_recall(prop: Proposal, recs: Sequence[Record], k: int = 4, batch: int = 64) -> float:
    """Fraction of placeable items whose top-k orientations hold a best one."""
    hit = tot = 0
    for i in range(0, len(recs), batch):
        part = [r for r in recs[i:i + batch]]
        g, hm, mask, _ = batch_tensors(part)
        logits, _ = prop.run(g, hm)
        lg = logits.cpu().numpy()
        for r, z in zip(part, lg):
            if not r.found.any():
                continue
            z = np.where(r.fits, z, -np.inf)
            top = np.argsort(-z, kind="stable")[:k]
            hit += bool(best_set(r)[top].any())
            tot += 1
    return hit / max(1, tot)


def train(recs: Sequence[Record], epochs: int = 4, batch: int = 64, lr: float = 1e-3, seed: int = 0,
          params: Optional[np.ndarray] = None, log=print) -> Proposal:
    """Adam on the masked softmax cross-entropy, minibatches of items."""
    rng = np.random.default_rng(seed)
    prop = Proposal(params if params is not None else init_params(seed))
    usable = [r for r in recs if r.found.any()]
    for ep in range(epochs):
        order = rng.permutation(len(usable))
        tot, nb = 0.0, 0
        for i in range(0, len(order), batch):
            part = [usable[j] for j in order[i:i + batch]]
            g, hm, mask, tgt = batch_tensors(part)
            _, loss = prop.run(g, hm, mask, tgt, want_logits=False)
            prop.adam(lr * 0.5 * (1.0 + np.cos(np.pi * ep / max(1, epochs))))
            tot += loss
            nb += 1
        log(f"epoch {ep}: mean loss {tot / max(1, nb):.4f} over {nb} batches")
    return prop


def save(prop: Proposal, path: Path = WEIGHTS, **meta) -> None:
    np.savez_compressed(path, params=prop.params(), **{k: np.asarray(v) for k, v in meta.items()})


def load(path: Path = WEIGHTS) -> Proposal:
    with np.load(path) as z:
        return Proposal(z["params"])
