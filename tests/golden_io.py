"""Reader for tests/golden/ref_kats.npz (see tests/golden/make_golden.py)."""
import hashlib
import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_kats.npz"


def load_records():
    z = np.load(GOLDEN, allow_pickle=False)
    recs = json.loads(str(z["index"]))

    def dec(x):
        if isinstance(x, dict) and "__a__" in x:
            return z[f"a{x['__a__']}"]
        if isinstance(x, dict) and "v" in x:
            v = [dec(e) for e in x["v"]]
            return tuple(v) if x["__t__"] else v
        return x
    out = []
    for r in recs:
        out.append({"test": r["test"], "fn": r["fn"], "args": dec(r["args"]),
                    "out": r["out"] if isinstance(r["out"], dict) and "__sha__" in r["out"] else dec(r["out"])})
    return out


def same_output(got, want):
    """Compare an output against a golden value (array, sha-pinned array, tuple)."""
    if isinstance(want, dict) and "__sha__" in want:
        g = np.ascontiguousarray(np.asarray(got), dtype=np.int32)
        return list(g.shape) == want["shape"] and hashlib.sha256(g.tobytes()).hexdigest() == want["__sha__"]
    if isinstance(want, np.ndarray):
        return np.array_equal(np.asarray(got), want)
    if isinstance(want, (tuple, list)):
        got = tuple(got)
        if len(got) != len(want):
            return False
        return all(same_output(g, w) for g, w in zip(got, want))
    if isinstance(want, float):
        return float(got) == want
    return got == want
