"""Guard bands: the memory-safety check of the workspace (in place of the
reference's memcheck gate, run_memcheck.py:18-132; compute-sanitizer is
closed on this pool).

A child process loads the library with CG3M_GUARD_BANDS set, so every region
of each call's workspace (packed planes, split partials, the rounding region's
path plane, packed rows, energies, flags, exact-recompute slices and partial
sums) is followed by a 4 KB band of a fixed pattern that the call fills before
its first kernel and checks after its last.  A kernel writing past its region
damages a band and fails this test.  The same calls in this process (no
bands, the shipped layout) must give the same bytes.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import ctypes, json, sys
sys.path[:0] = [{root!r} + "/tests", {root!r} + "/ascend-open-source-contributions_b200", {root!r} + "/oracle"]
import torch
import cg3m
import oracle as O
from guard_battery import run_battery
dev = torch.device("cuda:0")
torch.cuda.set_device(dev)
out = run_battery(cg3m, O, torch, dev)
en, dmg = ctypes.c_int(0), ctypes.c_int(-1)
st = cg3m.lib.cg3mDiagGuardStatus(ctypes.byref(en), ctypes.byref(dmg))
print(json.dumps({{"status": st, "enabled": en.value, "damaged": dmg.value, "calls": out}}))
"""


def test_workspace_guard_bands_stay_intact(cg3m, oracle, cuda):
    import ctypes

    import torch

    from guard_battery import run_battery

    env = dict(os.environ, CG3M_GUARD_BANDS="1")
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    child = json.loads(r.stdout.strip().splitlines()[-1])
    assert child["status"] == 0 and child["enabled"] == 1
    assert child["damaged"] == 0, child
    en, dmg = ctypes.c_int(-1), ctypes.c_int(-1)
    assert cg3m.lib.cg3mDiagGuardStatus(ctypes.byref(en), ctypes.byref(dmg)) == 0 and en.value == 0
    here = run_battery(cg3m, oracle, torch, cuda)
    assert set(here) == set(child["calls"])
    for name, rec in here.items():
        assert list(rec) == child["calls"][name], name
