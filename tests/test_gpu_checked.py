"""The bounds-checked build (MP_CHECKED=1 -> libmantlepar_b200_checked.so):
every stage element checks the cell and edge indices it derives before any
access and would record MP_ERR_ARG_OUTOFRANGE (part PART_CHECK) instead of
touching memory outside its arrays. On valid inputs no check may fire and
the results must equal the default build's bit for bit: a child process
loads the checked library and runs a single instance (stage, device-resident
and host-driven steps, mixed precision) and a batch; the parent runs the same
cases on the default build."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = r'''
import json, sys
import numpy as np
sys.path.insert(0, ROOT)
from mantlepar_b200 import synthetic as sy
from mantlepar_b200.transport import Transport, TransportConfig
from mantlepar_b200.batch import Batch
out = {}
for name, w, prec, dev in (("w20", sy.Workload(nx=20, ny=20), 0, True), ("w37x23", sy.Workload(nx=37, ny=23, seed=3, noise_H=0.1), 1, True),
                           ("w7x4_host", sy.Workload(nx=7, ny=4, seed=9), 0, False)):
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3, precision=prec))
    t.set_device_steps(dev)
    t.set_face_velocity(*sy.face_velocity(w))
    t.set_state(*sy.initial_state(w))
    r = t.rhs()
    out[name + "_rhs"] = [r[k].tolist() for k in ("rhsH", "rhsC", "T", "phi", "rate")]
    t.step(12)
    out[name + "_steps"] = [a.tolist() for a in t.get_state()]
    t.close()
ws = [sy.Workload(nx=20, ny=20), sy.Workload(nx=12, ny=30, seed=4), sy.Workload(nx=2, ny=2, seed=5)]
b = Batch(ws, TransportConfig(cfl=0.4, integrator=3))
for i, w in enumerate(ws):
    b.set_face_velocity(i, *sy.face_velocity(w))
    b.set_state(i, *sy.initial_state(w))
b.step(8)
for i in range(len(ws)):
    g = b.get_state(i)
    out["batch%d" % i] = [g[k].tolist() for k in ("H", "C", "T", "phi")] + [g["status"]]
b.close()
print(json.dumps(out))
'''


def run_cases(env_checked: bool):
    env = dict(os.environ, MP_CHECKED="1" if env_checked else "0")
    code = "ROOT = %r\n" % ROOT + CASES
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_checked_build_equals_default_build(cuda_lib):
    from mantlepar_b200 import build
    build.build_checked()
    checked = run_cases(True)
    default = run_cases(False)
    assert checked.keys() == default.keys()
    for k in checked:
        for a, b in zip(checked[k], default[k]):
            assert np.array_equal(np.asarray(a), np.asarray(b)), k
    for i in range(3):
        assert checked["batch%d" % i][-1] == 0
