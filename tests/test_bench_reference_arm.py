"""The benchmark's reference arm (`bench.py --impl reference`) times the
reference's algorithm (the oracle) on the host cores and must load none of
this repository's native code: no module of the psacking_b200 package is
imported and no library under psacking_b200/ is mapped into the process, so
the ratio of the two arms compares the reference with this engine and
nothing else.  Runs one step of the arm in a child process (about 15 s on 8
cores) and reads its JSON line."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

CHILD = r"""
import json, runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '0', '--no-cuda-reference']
runpy.run_path('bench.py', run_name='__main__')
mods = [m for m in sys.modules if m.split('.')[0] == 'psacking_b200']
maps = sorted({l.split()[-1] for l in open('/proc/self/maps') if 'psacking_b200' in l})
print('LOADED', json.dumps({'mods': mods, 'maps': maps}))
"""


def test_reference_arm_loads_no_repository_native_code():
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    line = json.loads(next(l for l in lines if l.startswith("{")))
    loaded = json.loads(next(l for l in lines if l.startswith("LOADED "))[len("LOADED "):])
    assert loaded == {"mods": [], "maps": []}, loaded
    assert line["impl"] == "reference" and line["unit"] == "items/s" and line["value"] > 0
    assert line["config"]["items_per_run"] == 350 and line["config"]["items_placed_per_run"] == 174
    # each timed item reproduces the oracle trace's record of the same stream
    done, total = (int(v) for v in line["config"]["sample_parity_vs_trace"].split("/"))
    assert total > 0 and done == total
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] == "port"


def test_learned_leg_reports_and_never_fails_the_line(monkeypatch):
    """The learned-proposal object of the headline line copies the config-4
    run's figures, and any exception there becomes an `unavailable` entry
    instead of ending the bench (host logic; run_learned is stubbed)."""
    sys.path.insert(0, str(ROOT))
    import bench
    doc = {"value": 2000.0, "config": {"workload": "config4: w", "plain_items_per_s": 1250.0,
                                       "speedup_vs_plain": 1.6, "density_learned": 0.44,
                                       "density_plain": 0.45, "density_gap_pp": 0.8, "fallback_rate": 0.03}}
    seen = {}

    def fake(args, rank, world, local_rank):
        seen.update(steps=args.steps, warmup=args.warmup, rank=rank, world=world, local_rank=local_rank)
        return doc
    monkeypatch.setattr(bench, "run_learned", fake)
    out = bench.learned_leg(None, 0)
    assert seen == {"steps": 1, "warmup": 1, "rank": 0, "world": 1, "local_rank": 0}
    assert out["items_per_s"] == 2000.0 and out["speedup_vs_plain"] == 1.6 and out["density_gap_pp"] == 0.8

    def boom(*a):
        raise RuntimeError("no device")
    monkeypatch.setattr(bench, "run_learned", boom)
    assert bench.learned_leg(None, 0) == {"unavailable": "RuntimeError: no device"}
