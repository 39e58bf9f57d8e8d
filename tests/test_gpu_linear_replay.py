"""The device affine search against the same search replayed on the CPU with the
oracle's costs (tests/cpp/linear_cpu: the library's LinearRunner with the oracle's MI /
correlation in place of the device evaluator).  The replay is pinned to the reference's
own tipl::reg::linear on the CPU (tests/test_linear_cpu.py: bit-identical on the
single-threaded narrow-bound path; on the full search within the reference's
run-to-run spread, which comes from its racing threads).  Here the device run must give
the replay's result: final cost, parameters and evaluation count, on several seeded
pairs, for MI and correlation, with the full search (reg bound, mask start) -- so the
device's search is the reference's algorithm evaluation for evaluation."""
import os
import subprocess

import numpy as np
import pytest

import tipl_b200 as tb
from tipl_b200 import phantom as ph

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "linear_cpu")


@pytest.fixture(scope="module")
def pairs():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp"), "linear_cpu"])
    rng = np.random.default_rng(ph.seed_for(2, 300))
    out = []
    for shape in ((48, 52, 44), (40, 56, 48), (52, 44, 40)):
        t, m, _ = ph.affine_pair(shape, rng=rng)
        out.append((ph.normalize_to_u8(t), ph.normalize_to_u8(m)))
    return out


def replay(tmp_path, f8, m8, cost_type):
    fp, mp, op = tmp_path / "f.u8", tmp_path / "m.u8", tmp_path / "o.bin"
    f8.tofile(fp)
    m8.tofile(mp)
    z, y, x = f8.shape
    z2, y2, x2 = m8.shape
    subprocess.run([EXE, str(x), str(y), str(z), str(fp), str(x2), str(y2), str(z2), str(mp), str(cost_type), "0",
                    str(op)], check=True, capture_output=True, timeout=900)
    o = np.fromfile(op, np.uint8)
    return o[:4].view(np.float32)[0], o[4:52].view(np.float32).copy(), int(o[52:60].view(np.int64)[0])


@pytest.mark.parametrize("cost_type", [tb.reg.MI, tb.reg.CORR])
def test_device_search_equals_cpu_replay(pairs, tmp_path, cost_type):
    for f8, m8 in pairs:
        cost, arg, evals = tb.reg.linear(f8, (1, 1, 1), m8, (1, 1, 1), param=tb.reg.linear_param(cost_type=cost_type))
        c_cpu, a_cpu, e_cpu = replay(tmp_path, f8, m8, cost_type)
        assert np.float32(cost).view(np.uint32) == c_cpu.view(np.uint32), (cost, c_cpu)
        assert np.array_equal(np.asarray(arg, np.float32).view(np.uint32), a_cpu.view(np.uint32)), (arg, a_cpu)
        assert evals == e_cpu, (evals, e_cpu)


def test_full_size_mi_search_equals_cpu_replay(tmp_path):
    """The affine workload's own pair (182x218x182 uint8 template and subject 0 of the
    bench, seed 20261203 + 2000): the device's MI registration equals the CPU replay
    with the oracle's costs -- cost, parameters and all ~2,300 evaluations."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp"), "linear_cpu"])
    rng = np.random.default_rng(ph.seed_for(2, 0))
    t, m, _ = ph.affine_pair((182, 218, 182), rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    cost, arg, evals = tb.reg.linear(torch.from_numpy(f8).cuda(), (1, 1, 1), torch.from_numpy(m8).cuda(), (1, 1, 1))
    c_cpu, a_cpu, e_cpu = replay(tmp_path, f8, m8, tb.reg.MI)
    assert np.float32(cost).view(np.uint32) == c_cpu.view(np.uint32), (cost, c_cpu)
    assert np.array_equal(np.asarray(arg, np.float32).view(np.uint32), a_cpu.view(np.uint32))
    assert evals == e_cpu and evals > 1000
