"""BinPacker: the greedy packing loop over the B200 engine.

Mirrors spectral_packer.packer (BinPacker / PackingResult / PlacementInfo,
spectral_packer/packer.py:33-608): same constructor checks, item order
(np.argsort(volumes)[::-1]), orientation loop with strict `<` across
orientations, item ids id_offset + k, and statistics.

Two engines produce identical results:
  engine="native" (default) one C-ABI call (psb_pack) runs the whole loop with
                  the tray, its spectra and its distance field resident on the
                  GPU; orientations are gathered on the device.
  engine="calls"  the reference's call pattern, one _core call per
                  orientation (packer.py:447-528), for drop-in comparisons.
"""
from __future__ import annotations

import hashlib
import os
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _core
from .rotations import get_orientations, make_contiguous, orientation_maps


@dataclass
class PlacementInfo:
    """One item's outcome (packer.py:33-60)."""
    item_index: int
    position: Optional[Tuple[int, int, int]]
    score: Optional[float]
    success: bool
    volume: int = 0
    orientation_index: int = 0


@dataclass
class PackingResult:
    """Results of a packing run (packer.py:86-165)."""
    tray: np.ndarray
    placements: List[PlacementInfo] = field(default_factory=list)
    num_placed: int = 0
    num_failed: int = 0
    density: float = 0.0
    total_volume: int = 0
    bounding_box: Optional[Tuple[Tuple[int, int, int], Tuple[int, int, int]]] = None
    mesh_placements: Optional[list] = None
    diagnostics: Optional[dict] = None

    def get_item_mask(self, item_id: int) -> np.ndarray:
        return self.tray == item_id

    def save_vox(self, path: Union[str, Path]) -> None:
        from .vox import save_vox
        save_vox(self.tray, str(path))

    def summary(self) -> str:
        lines = [
            "Packing Result Summary",
            "=" * 40,
            f"Items placed:    {self.num_placed}",
            f"Items failed:    {self.num_failed}",
            f"Success rate:    {self.num_placed / max(1, self.num_placed + self.num_failed):.1%}",
            f"Packing density: {self.density:.1%}",
            f"Total volume:    {self.total_volume} voxels",
            f"Tray size:       {self.tray.shape}",
        ]
        if self.bounding_box:
            lo, hi = self.bounding_box
            lines.append(f"Bounding box:    {lo} to {hi}")
        return "\n".join(lines)


class BinPacker:
    """Greedy spectral packer (packer.py:168-251).

    height_penalty is stored but, as in the reference, the search always uses
    1e8 (packer.py:248 vs spectral_packing/constants.h:7)."""

    def __init__(self, tray_size: Tuple[int, int, int], voxel_resolution: int = 128,
                 height_penalty: float = 1e8, num_orientations: int = 1,
                 interlocking_free: bool = False, engine: str = "native"):
        if len(tray_size) != 3:
            raise ValueError(f"tray_size must be a 3-tuple, got {len(tray_size)} elements")
        if any(s <= 0 for s in tray_size):
            raise ValueError(f"tray_size dimensions must be positive, got {tray_size}")
        if voxel_resolution <= 0:
            raise ValueError(f"voxel_resolution must be positive, got {voxel_resolution}")
        if num_orientations not in (1, 4, 6, 24):
            raise ValueError(f"num_orientations must be 1, 4, 6, or 24, got {num_orientations}")
        if engine not in ("native", "calls"):
            raise ValueError("engine must be 'native' or 'calls'")
        self.tray_size = tuple(int(s) for s in tray_size)
        self.voxel_resolution = voxel_resolution
        self.height_penalty = height_penalty
        self.num_orientations = num_orientations
        self.interlocking_free = interlocking_free
        self.engine = engine

    # ------------------------------------------------------------------ files
    def pack_files(self, paths: Sequence[Union[str, Path]], sort_by_volume: bool = True,
                   validate_meshes: bool = True, repair_meshes: bool = True) -> PackingResult:
        """Pack STL meshes (packer.py:253-295 of the reference): each file is
        voxelized at `voxel_resolution` by voxelize_stl (the path the
        reference's Voxelizer.voxelize_file takes for .stl files), then the
        grids are packed by pack_voxels.  Other mesh formats, and STL files
        voxelize_stl rejects, go through trimesh in the reference, which is
        not part of this engine: they raise NotImplementedError.  The
        validate/repair flags only concern that loader and are accepted for
        interface compatibility."""
        from .voxelize import voxelize_stl
        voxels = []
        for path in paths:
            path = Path(path)
            if not path.exists():
                raise FileNotFoundError(f"Mesh file not found: {path}")
            if path.suffix.lower() != ".stl":
                raise NotImplementedError(f"{path}: only STL meshes are voxelized by this engine")
            try:
                voxels.append(voxelize_stl(path, self.voxel_resolution))
            except RuntimeError as e:
                raise NotImplementedError(f"{path}: voxelize_stl failed ({e}); the reference would fall back "
                                          "to its trimesh voxelizer, which this engine does not include") from e
        return self.pack_voxels(voxels, sort_by_volume=sort_by_volume)

    # ------------------------------------------------------------------ voxels
    def _prepare(self, items, sort_by_volume, initial_tray):
        if len(items) == 0:
            raise ValueError("items list cannot be empty")
        processed = []
        for i, item in enumerate(items):
            if not isinstance(item, np.ndarray):
                raise ValueError(f"Item {i} is not a numpy array")
            if item.ndim != 3:
                raise ValueError(f"Item {i} must be 3D, got {item.ndim}D")
            processed.append(np.ascontiguousarray(item, dtype=np.int32))   # no copy when already int32
        volumes = [int(v) for v in _core.positive_counts(processed)]   # np.sum(item > 0) per item
        if sort_by_volume:
            order = list(np.argsort(volumes)[::-1])
        else:
            order = list(range(len(items)))
        if initial_tray is not None:
            if initial_tray.shape != self.tray_size:
                raise ValueError(f"initial_tray shape {initial_tray.shape} does not match "
                                 f"tray_size {self.tray_size}")
            tray = initial_tray.astype(np.int32).copy()
            id_offset = int(np.max(tray))
        else:
            tray = np.zeros(self.tray_size, dtype=np.int32)
            id_offset = 0
        return processed, volumes, order, tray, id_offset

    def pack_voxels(self, items: Sequence[np.ndarray], sort_by_volume: bool = True,
                    initial_tray: Optional[np.ndarray] = None) -> PackingResult:
        processed, volumes, order, tray, id_offset = self._prepare(items, sort_by_volume, initial_tray)
        if self.engine == "native":
            return self._pack_native(processed, volumes, order, tray, id_offset, len(items))
        return self._pack_calls(processed, volumes, order, tray, id_offset, len(items))

    def _pack_native(self, processed, volumes, order, tray, id_offset, n_items):
        maps = orientation_maps(self.num_orientations)
        seq = [np.ascontiguousarray(processed[i]) for i in order]
        final, res, stats = _core.pack_native(seq, tray, maps, bool(self.interlocking_free), int(id_offset))
        placements = []
        diag_or, ncand, err = 0, 0, 0.0
        for k, orig in enumerate(order):
            pos, found, score, orient, diag, nc, er = res[k]
            diag_or |= int(diag)
            ncand += int(nc)
            err = max(err, float(er))
            if found:
                placements.append(PlacementInfo(int(orig), tuple(int(v) for v in pos), float(score), True,
                                                volumes[orig], int(orient)))
            else:
                placements.append(PlacementInfo(int(orig), None, None, False, volumes[orig], 0))
        return self._finish(final, placements, n_items,
                            {"diag": diag_or, "candidates": ncand, "max_err_ratio": err}, stats)

    def _pack_calls(self, processed, volumes, order, tray, id_offset, n_items):
        # a fresh run never inherits a cached tray context (the reference's
        # generation counter restarts at 0 every run, bindings.cpp:209/236)
        _core.gpu_tray_cleanup()
        generation = 0
        placements = []
        num_placed = 0
        for orig in order:
            item = processed[orig]
            best_pos, best_score, best_o, best_item, found_any = None, float("inf"), 0, item, False
            orients = get_orientations(item, self.num_orientations)
            if self.num_orientations > 1 or self.interlocking_free:
                tray_distance = _core.calculate_distance(tray)
            if self.interlocking_free:
                valid, vidx = [], []
                for o, r in enumerate(orients):
                    r = make_contiguous(r.astype(np.int32))
                    if not any(r.shape[a] > self.tray_size[a] for a in range(3)):
                        valid.append(r)
                        vidx.append(o)
                if valid:
                    pos, found, score, bo = _core.fft_search_batch_interlocking_free(
                        valid, tray, tray_distance, generation)
                    if found and bo >= 0:
                        best_pos, best_score, best_o, best_item, found_any = pos, score, vidx[bo], valid[bo], True
            else:
                for o, r in enumerate(orients):
                    r = make_contiguous(r.astype(np.int32))
                    if any(r.shape[a] > self.tray_size[a] for a in range(3)):
                        continue
                    if self.num_orientations > 1:
                        pos, found, score = _core.fft_search_placement_with_cache(r, tray, tray_distance, generation)
                    else:
                        pos, found, score = _core.fft_search_placement(r, tray)
                    if found and score < best_score:
                        best_pos, best_score, best_o, best_item, found_any = pos, score, o, r, True
            if found_any:
                tray = _core.place_in_tray(best_item, tray, best_pos, id_offset + num_placed + 1)
                generation += 1
                num_placed += 1
                placements.append(PlacementInfo(int(orig), tuple(best_pos), float(best_score), True,
                                                volumes[orig], best_o))
            else:
                placements.append(PlacementInfo(int(orig), None, None, False, volumes[orig], 0))
        return self._finish(tray, placements, n_items, None)

    def _finish(self, tray, placements, n_items, diag, stats=None):
        placements.sort(key=lambda p: p.item_index)
        num_placed = sum(1 for p in placements if p.success)
        if stats is None:
            density, total, bbox = self._calculate_stats(tray)
        else:
            density, total, bbox = self._stats_from_counts(*stats)
        return PackingResult(tray=tray, placements=placements, num_placed=num_placed,
                             num_failed=n_items - num_placed, density=density, total_volume=total,
                             bounding_box=bbox, diagnostics=diag)

    def pack_many(self, trays: Sequence[Tuple[Tuple[int, int, int], Sequence[np.ndarray]]],
                  sort_by_volume: bool = True, concurrency: int = 8,
                  checkpoint: Optional[Union[str, Path]] = None) -> List[PackingResult]:
        """Pack independent trays (each (dims, items), starting empty) with
        this packer's orientation and interlocking settings.  Equivalent to one
        BinPacker(dims, ...).pack_voxels(items) per tray; up to `concurrency`
        trays run at once on separate CUDA streams.

        checkpoint: an .npz path.  The trays are then packed `concurrency` at
        a time, and after each group the final tray and the per-item results
        of every finished tray are written there (to a temporary file, then
        renamed over it).  A call given an existing checkpoint reads the
        finished trays back and packs only the others; the file records a
        digest of every tray's dimensions, items and the packer's settings,
        and a checkpoint written for other inputs raises ValueError."""
        jobs, metas = [], []
        for dims, items in trays:
            sub = BinPacker(dims, self.voxel_resolution, self.height_penalty, self.num_orientations,
                            self.interlocking_free)
            processed, volumes, order, _, _ = sub._prepare(items, sort_by_volume, None)
            jobs.append((tuple(int(d) for d in dims), [np.ascontiguousarray(processed[i]) for i in order]))
            metas.append((sub, volumes, order, len(items)))
        if checkpoint is None:
            outs = _core.pack_many(jobs, orientation_maps(self.num_orientations), bool(self.interlocking_free),
                                   int(concurrency))
        else:
            outs = self._pack_many_checkpointed(jobs, int(concurrency), Path(checkpoint))
        results = []
        for (sub, volumes, order, n_items), (final, res) in zip(metas, outs):
            placements = []
            for k, orig in enumerate(order):
                pos, found, score, orient = res[k][:4]
                if found:
                    placements.append(PlacementInfo(int(orig), tuple(int(v) for v in pos), float(score), True,
                                                    volumes[orig], int(orient)))
                else:
                    placements.append(PlacementInfo(int(orig), None, None, False, volumes[orig], 0))
            results.append(sub._finish(final, placements, n_items, None))
        return results

    def _job_digest(self, dims, items) -> str:
        h = hashlib.sha256()
        h.update(repr((tuple(dims), int(self.num_orientations), bool(self.interlocking_free))).encode())
        for it in items:
            h.update(repr(it.shape).encode())
            h.update(np.ascontiguousarray(it, dtype=np.int32).tobytes())
        return h.hexdigest()

    def _pack_many_checkpointed(self, jobs, concurrency: int, path: Path):
        """_core.pack_many's (final tray, results) per job, `concurrency` jobs
        per call, with the finished ones kept in the checkpoint file."""
        keys = [self._job_digest(dims, items) for dims, items in jobs]
        done = {}
        if path.exists():
            with np.load(path) as z:
                if [str(k) for k in z["keys"]] != keys:
                    raise ValueError(f"checkpoint {path} was written for other trays, items or settings")
                for i in z["done"].tolist():
                    done[int(i)] = (np.array(z[f"final_{i}"]), np.array(z[f"rec_{i}"]))
        todo = [i for i in range(len(jobs)) if i not in done]
        maps = orientation_maps(self.num_orientations)
        step = max(1, concurrency)
        for c in range(0, len(todo), step):
            part = todo[c:c + step]
            outs = _core.pack_many([jobs[i] for i in part], maps, bool(self.interlocking_free), concurrency)
            for i, (final, res) in zip(part, outs):
                # per item: found, x, y, z, score, orientation (float64 holds them exactly)
                rec = np.asarray([[float(bool(r[1])), *(float(v) for v in r[0]), float(r[2]), float(r[3])]
                                  for r in res], dtype=np.float64).reshape(-1, 6)
                done[i] = (np.asarray(final, dtype=np.int32), rec)
            arrays = {"keys": np.asarray(keys), "done": np.asarray(sorted(done), dtype=np.int64)}
            for i, (final, rec) in done.items():
                arrays[f"final_{i}"], arrays[f"rec_{i}"] = final, rec
            tmp = path.with_name(path.name + ".tmp")
            with open(tmp, "wb") as f:
                np.savez(f, **arrays)
            os.replace(tmp, path)
        outs = []
        for i in range(len(jobs)):
            final, rec = done[i]
            outs.append((final, [((int(r[1]), int(r[2]), int(r[3])), bool(r[0]), float(r[4]), int(r[5])) for r in rec]))
        return outs

    def pack_single(self, item: np.ndarray,
                    tray: Optional[np.ndarray] = None) -> Tuple[Optional[Tuple[int, int, int]], bool, float]:
        """packer.py:546-580: (position or None, found, score)."""
        if tray is None:
            tray = np.zeros(self.tray_size, dtype=np.int32)
        pos, found, score = _core.fft_search_placement(item.astype(np.int32), tray)
        if found:
            return tuple(pos), True, score
        return None, False, 0.0

    @staticmethod
    def _stats_from_counts(occupied, lo, hi):
        """_calculate_stats from the occupied-cell count and bounding box
        the engine computed on the device (psb_tray_stats)."""
        if occupied == 0:
            return 0.0, 0, None
        lo, hi = tuple(int(v) for v in lo), tuple(int(v) for v in hi)
        vol = int(np.prod([b - a + 1 for a, b in zip(lo, hi)]))
        return (float(occupied / vol) if vol > 0 else 0.0), int(occupied), (lo, hi)

    def _calculate_stats(self, tray: np.ndarray):
        """packer.py:582-601: density = occupied / bounding-box volume."""
        occ = tray > 0
        occupied = int(np.count_nonzero(occ))
        if occupied == 0:
            return 0.0, 0, None
        # bounding box from per-axis projections (no coordinate list)
        lo, hi = [], []
        for axes in ((1, 2), (0, 2), (0, 1)):
            nz = np.flatnonzero(occ.any(axis=axes))
            lo.append(int(nz[0]))
            hi.append(int(nz[-1]))
        lo, hi = tuple(lo), tuple(hi)
        vol = int(np.prod([b - a + 1 for a, b in zip(lo, hi)]))
        return (float(occupied / vol) if vol > 0 else 0.0), occupied, (lo, hi)

    def __repr__(self) -> str:
        return (f"BinPacker(tray_size={self.tray_size}, voxel_resolution={self.voxel_resolution}, "
                f"num_orientations={self.num_orientations})")
