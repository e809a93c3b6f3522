"""The two PGS kernels for worlds without joints give the same trajectory, bit for bit.

A plain world of more than 1,024 bodies without joints is solved by the chunked kernel
(Morton-ordered chunks, neighbour waits); BGPU_PGS=team in the environment selects the
team-barrier kernel instead (read once per process, so each runs in a child process). Both
solve the groups in the same (colour, pair) order, so the states after every step must be
identical, not merely close. The oracle lockstep tests pin the chunked kernel against the
reference's restatement; this test ties the team kernel to it.
"""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

CHILD = r"""
import json, os, sys
sys.path[:0] = [os.path.join(sys.argv[1], "bullet-physics_b200"), os.path.join(sys.argv[1], "tests")]
import numpy as np
import bgpu, scenes
sc = scenes.large_pile_fast(16, 16, 16, seed=5, steps=90)
w = sc.build_gpu(bgpu)
digests = []
for step in range(sc.steps):
    w.step(sc.dt)
    bits = np.frombuffer(w.state().astype(np.float32).tobytes(), np.uint32).astype(np.uint64)
    digests.append(int((bits * np.arange(1, bits.size + 1, dtype=np.uint64)).sum() % (1 << 61)))
st = w.stats()
np.save(sys.argv[2], w.state().astype(np.float32))
print(json.dumps({"digests": digests, "status": int(st["device_status"]), "colours": int(st["num_colours"]),
                  "contacts": int(st["num_contacts"])}))
"""


def _run(tmp_path, mode):
    env = dict(os.environ)
    env.pop("BGPU_PGS", None)
    if mode:
        env["BGPU_PGS"] = mode
    out = tmp_path / f"state_{mode or 'chunk'}.npy"
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(out)], env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("{")][-1]
    return json.loads(line), np.load(out)


def test_chunked_and_team_kernels_step_identically(tmp_path):
    chunk, s_chunk = _run(tmp_path, None)
    team, s_team = _run(tmp_path, "team")
    assert chunk["status"] == 0 and team["status"] == 0
    assert chunk["contacts"] > 4000 and chunk["colours"] >= 4
    first = next((k for k, (a, b) in enumerate(zip(chunk["digests"], team["digests"])) if a != b), None)
    assert first is None, f"the kernels' states first differ after step {first + 1}"
    np.testing.assert_array_equal(s_chunk, s_team)
