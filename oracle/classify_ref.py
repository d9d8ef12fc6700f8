"""Classify where the reference's own cuFFT search differs from the oracle --
TEST INFRASTRUCTURE ONLY.

    python oracle/classify_ref.py <ref_cuda sample output> [--out FILE]

Input: the output of `oracle/ref_cuda.py sample` over the benchmark stream
(committed as tests/golden/ref_cuda_sample_config3.json): for each search
position, the reference's result (its BinPacker on the tray state replayed
from the oracle's trace), compared with the oracle's record.  For
every item where they differ, the reference's choice is evaluated exactly on
that tray state (the oracle is the arbiter):

  same_cell     the same orientation and cell, but the reference reports a
                score its FP32 proximity rounded to another integer
  exact_tie     another cell that is ok with an exact score equal to the
                oracle's best: FP32 noise broke an exact tie another way
  worse         the reference's cell is ok but its exact score is higher:
                FP32 noise made a worse cell look best
  not_ok        the reference's cell collides or is unreachable (its FP32
                collision count rounded to 0, or the flood fill on the noisy
                counts let it through)
  found_differs one side found a placement and the other did not

and the reference's reported score is compared with the exact score of the
same cell (its FP32 proximity error).
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO))

from oracle import psb_oracle as O  # noqa: E402
from oracle.trace_replay import load_trace, oriented, replay_states, trace_items  # noqa: E402


def exact_score_of(item, tray, phi, pos, interlock=True):
    """(ok, exact score) of placing `item` (already oriented) at `pos`."""
    x, y, z = pos
    ex, ey, ez = item.shape
    nx, ny, nz = tray.shape
    _, hi = O.bounds(item)
    if x + hi[0] >= nx or y + hi[1] >= ny or z + hi[2] >= nz or min(pos) < 0:
        return False, None
    sub_t = tray[x:x + ex, y:y + ey, z:z + ez]
    sub_i = item[:sub_t.shape[0], :sub_t.shape[1], :sub_t.shape[2]]
    if np.any((sub_t > 0) & (sub_i > 0)):
        return False, None
    prox = int(np.sum(sub_i.astype(np.int64) * phi[x:x + ex, y:y + ey, z:z + ez][:sub_i.shape[0], :sub_i.shape[1],
                                                                                 :sub_i.shape[2]]))
    if interlock:
        ok, _ = O._search_fields(item, tray, phi, True)
        if not ok[x, y, z]:
            return False, O.score_block(prox, z, nz)
    return True, O.score_block(prox, z, nz)


def classify(doc):
    trace = load_trace("config3_seed1")
    seq = trace_items(trace)
    rows = doc["rows"]
    for r in rows:   # the oracle's record of each position, from the trace
        r["oracle"] = trace["records"][r["position"]]
        r["same"] = r["result"] == r["oracle"]
    diffs = [r for r in rows if not r["same"]]
    states = replay_states(trace, seq, [r["position"] for r in diffs])
    out, counts = [], {"same": len(rows) - len(diffs)}
    for r in diffs:
        pos = r["position"]
        got, want = r["result"], r["oracle"]
        tray = states[pos]
        if bool(got[0]) != bool(want[0]):
            cls, exact = "found_differs", None
        elif got[1:5] == want[1:5]:
            cls, exact = "same_cell", want[5]
        else:
            phi = O.calculate_distance(tray)
            item = oriented(seq[pos], got[4], 24)
            ok, exact = exact_score_of(item, tray, phi, tuple(got[1:4]))
            if not ok:
                cls = "not_ok"
            elif exact == want[5]:
                cls = "exact_tie"
            elif exact > want[5]:
                cls = "worse"
            else:
                cls = "better_than_oracle"   # never expected: the oracle is exact
        counts[cls] = counts.get(cls, 0) + 1
        out.append({"position": pos, "class": cls, "reference": got, "oracle": want, "reference_cell_exact": exact,
                    "reference_fp32_error": None if exact is None else got[5] - exact})
    return {"items": len(rows), "counts": counts, "rows": out}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("sample")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = classify(json.loads(Path(a.sample).read_text()))
    print(json.dumps({"items": res["items"], "counts": res["counts"]}))
    if a.out:
        Path(a.out).write_text(json.dumps(res, indent=1) + "\n")


if __name__ == "__main__":
    main()
