"""Every alternative kernel schedule gives the bits of the default one.

The library reads these switches once per process, so each case runs the
128^3 benchmark workload (65,536 chain beads, 4-point kernel, the Verlet
list, the 128-point plane passes) for a few steps in a fresh process and
compares positions, forces and the velocity field bit for bit with the
default process:

* FLUAMSL_PDL=0: ordinary launches instead of programmatic dependent ones;
* FLUAMSL_PLANE_V=0: the generic register plane passes instead of the
  conflict-free 128-point ones;
* FLUAMSL_FFT_SCHEDULE=lines / plane: the five-pass schedule, or the plane
  schedule, instead of the autotuner's pick;
* FLUAMSL_FUSED_FORCES=0: the Verlet-list forces in their own launch
  instead of inside the spread;
* FLUAMSL_SPREAD_BOX=0: one global atomic per product instead of the
  warp's shared box.

A further case compares the default step with the per-stage profiled step,
which keeps everything on one stream (the noise, and the field clear that
the W build then does itself).  A batch of small instances of several size
classes (Verlet-list, cell-mode and empty instances among them) compares
FLUAMSL_BLOCK_LISTS=0 and =1, the separate list kernels and the build of
one block per instance, with the default, where each class's tuner picks;
the same batch and an instance at 64^3 compare FLUAMSL_PLANE_CAND=0, 1, 2
(the planes-per-block candidates of the plane passes) with the tuner's
pick.
"""
import hashlib
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STEPS = 4

_SCRIPT = r"""
import hashlib, json, sys
sys.path.insert(0, sys.argv[1])
from fluam_b200 import StokesLimit, workloads
cfg, q, bonds = workloads.build("plain_128", seed=3)
sim = StokesLimit(cfg, q)
if bonds is not None:
    sim.load_bonds(*bonds)
profiled = sys.argv[3] == "1"
if profiled:
    sim.profile(True)
sim.step(int(sys.argv[2]))
sim.sync()
st = sim.status()
out = {k: hashlib.sha1(a.tobytes()).hexdigest()
       for k, a in (("q", sim.positions()), ("F", sim.forces()), ("v", sim.velocity()))}
out["errors"] = st["error_bits"]
print(json.dumps(out))
sim.close()
"""


_BATCH_SCRIPT = r"""
import hashlib, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import fluam_b200 as fsl
rng = np.random.default_rng(11)
cfgs, qs = [], []
for i in range(24):
    m = int(rng.choice((16, 24, 32)))
    n = 0 if i == 5 else int(round(np.exp(rng.uniform(np.log(8), np.log(3000)))))
    if i == 7:  # dense: the Verlet list overflows into cell mode
        q = rng.uniform(-2.0, 2.0, (3, 500))
    else:
        q = rng.uniform(-0.5, 0.5, (3, n)) * m
    cfgs.append(fsl.make_config((m, m, m), (float(m),) * 3, eta=float(rng.uniform(0.5, 2.0)), kT=0.01,
                                dt=0.01, cutoff=1.5, kernel=int(rng.choice((3, 4))), pair=fsl.PAIR_SOFT,
                                seed=500 + i))
    qs.append(q)
b = fsl.Batch(cfgs, qs)
b.step(int(sys.argv[2]))
b.sync()
h = hashlib.sha1()
errors = 0
for i in range(len(cfgs)):
    h.update(b.positions(i).tobytes())
    h.update(b.forces(i).tobytes())
    errors |= b.status(i)["error_bits"]
print(json.dumps({"qF": h.hexdigest(), "errors": errors}))
b.close()
"""

# one instance at 64^3 (20,000 particles, 4-point kernel, soft repulsion):
# the edge whose plane passes have three planes-per-block candidates
_SCRIPT64 = r"""
import hashlib, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import fluam_b200 as fsl
rng = np.random.default_rng(17)
q = rng.uniform(-32.0, 32.0, (3, 20000))
cfg = fsl.make_config((64, 64, 64), (64.0,) * 3, kT=0.01, dt=0.01, cutoff=1.5, kernel=4,
                      pair=fsl.PAIR_SOFT, seed=77)
sim = fsl.StokesLimit(cfg, q)
sim.step(int(sys.argv[2]))
sim.sync()
out = {k: hashlib.sha1(a.tobytes()).hexdigest()
       for k, a in (("q", sim.positions()), ("F", sim.forces()), ("v", sim.velocity()))}
out["errors"] = sim.status()["error_bits"]
print(json.dumps(out))
sim.close()
"""

_SWITCHES = ("FLUAMSL_PDL", "FLUAMSL_PLANE_V", "FLUAMSL_FFT_SCHEDULE", "FLUAMSL_FUSED_FORCES",
             "FLUAMSL_SPREAD_BOX", "FLUAMSL_BLOCK_LISTS", "FLUAMSL_PLANE_CAND")


def _run(env_extra, profiled=False, script=_SCRIPT):
    env = dict(os.environ)
    for k in _SWITCHES:
        env.pop(k, None)
    env.update(env_extra)
    r = subprocess.run([sys.executable, "-c", script, ROOT, str(STEPS), "1" if profiled else "0"],
                       capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out.pop("errors") == 0
    return out


@pytest.fixture(scope="module")
def default_run():
    return _run({})


@pytest.mark.parametrize("env", [
    {"FLUAMSL_PDL": "0"},
    {"FLUAMSL_PLANE_V": "0"},
    {"FLUAMSL_FFT_SCHEDULE": "lines"},
    {"FLUAMSL_FFT_SCHEDULE": "plane"},
    {"FLUAMSL_FUSED_FORCES": "0"},
    {"FLUAMSL_SPREAD_BOX": "0"},
], ids=lambda e: ",".join(f"{k}={v}" for k, v in e.items()))
def test_switch_gives_same_bits(default_run, env):
    assert _run(env) == default_run


def test_profiled_step_gives_same_bits(default_run):
    assert _run({}, profiled=True) == default_run


@pytest.fixture(scope="module")
def default_batch_run():
    return _run({}, script=_BATCH_SCRIPT)


@pytest.mark.parametrize("value", ["0", "1"])
def test_batch_list_build_gives_same_bits(default_batch_run, value):
    assert _run({"FLUAMSL_BLOCK_LISTS": value}, script=_BATCH_SCRIPT) == default_batch_run


@pytest.mark.parametrize("value", ["0", "1", "2"])
def test_batch_planes_per_block_gives_same_bits(default_batch_run, value):
    assert _run({"FLUAMSL_PLANE_CAND": value}, script=_BATCH_SCRIPT) == default_batch_run


@pytest.mark.parametrize("value", ["0", "1", "2"])
def test_planes_per_block_gives_same_bits_64(value):
    assert _run({"FLUAMSL_PLANE_CAND": value}, script=_SCRIPT64) == _run({}, script=_SCRIPT64)
