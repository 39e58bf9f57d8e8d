"""The cost kernels' two ways of reading the sampled volume give identical results:
texture gathers (the default) and byte loads (what volumes beyond the 2-D texture
limits use, forced here with REGB_TEXTURE=0 in a child process).  The correlation
cases include the integer-shift copy and the swapped roles (a larger fixed volume)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import tipl_b200 as tb
from tipl_b200 import phantom as ph
rng = np.random.default_rng(31)
shape = (45, 52, 41)
t, mv, _ = ph.affine_pair(shape, rng=rng)
f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(mv)
Ts = np.array([tb.affine_to_matrix(ph.random_affine(rng, rot_deg=6, trans_vox=3), shape, (1, 1, 1), shape,
                                   (1, 1, 1)) for _ in range(6)])
Ts[0] = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 2, -1, 1], np.float32)  # an integer shift (correlation copy path)
out = {"mi": tb.mi_cost(f8, m8, Ts).tolist(), "mi32": tb.mi32_cost(f8, m8, Ts).tolist(),
       "corr": tb.corr_cost(f8, m8, Ts).tolist(), "corr_swap": tb.corr_cost(f8, np.ascontiguousarray(m8[:40]), Ts).tolist()}
c, a, e = tb.reg.linear(f8, (1, 1, 1), m8, (1, 1, 1))
out["linear"] = [float(c), a.tolist(), int(e)]
print(json.dumps(out))
"""


def run(texture: bool):
    env = dict(os.environ)
    env["REGB_TEXTURE"] = "1" if texture else "0"
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_texture_and_byte_paths_agree():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    a, b = run(True), run(False)
    for k in ("mi", "mi32", "corr", "corr_swap"):
        assert a[k] == b[k], k  # bit-identical doubles
    assert a["linear"] == b["linear"]
