"""CDM at the workloads' own shapes against the reference's CPU cdm_common.

Fixture tests/golden/cdm_full.npz (tests/golden/make_golden.py --only cdm_full) holds,
per case, the SHA-256 of the reference's field and of its inputs.  The inputs are too
large to store (the 182x218x182 subject carries Rician noise), so the tests regenerate
them from their seeds and first check them against the stored input digests.

* full: the 182x218x182 uint8 pair of the nonlinear workload at min_dimension 32 (the
  23, 46 and 91 levels iterate, the field moves by about 2 voxels), through tb.reg.cdm
  and through one engine job (CDM stage only);
* c1_blob: the 64^3 float blob pair of the plain CDM workload at the default cdm_param:
  the reference never improves on its first iteration there and returns the zero field;
* c1_class, c1_class_u8: a 64^3 class-phantom pair, float and uint8, at the default
  cdm_param (levels 16 and 32 iterate; the field moves).
The bar is bit-for-bit equality of the field (reg/cdm.hpp:373-474)."""
import hashlib
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def inputs(g, name):
    from make_golden import CDM_FULL_CASES, cdm_full_inputs

    gen, dt = {c[0]: (c[1], c[2]) for c in CDM_FULL_CASES}[name]
    It, Is = cdm_full_inputs(gen, dt)
    assert digest(It) == str(g[f"{name}_It_sha256"]) and digest(Is) == str(g[f"{name}_Is_sha256"]), (
        "the regenerated inputs differ from the fixture's (the host's numpy/scipy arithmetic differs)")
    return It, Is


def params(name):
    from make_golden import CDM_FULL_CASES

    import tipl_b200 as tb

    kw = {c[0]: c[3] for c in CDM_FULL_CASES}[name]
    return tb.reg.cdm_param(**kw)


@pytest.fixture(scope="module")
def g(golden):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return golden("cdm_full")


@pytest.mark.parametrize("name", ["full", "c1_blob", "c1_class", "c1_class_u8"])
def test_cdm_equals_reference(g, name):
    import torch

    import tipl_b200 as tb

    It, Is = inputs(g, name)
    field, ok = tb.reg.cdm(torch.from_numpy(It).cuda(), torch.from_numpy(Is).cuda(), params(name))
    assert int(ok) == int(g[f"{name}_ok"])
    f = field.cpu().numpy()
    assert digest(f) == str(g[f"{name}_sha256"])
    assert float(np.abs(f).max()) == float(g[f"{name}_maxabs"])
    if name == "c1_blob":
        assert not f.any()  # the reference's own result on this generator
    else:
        assert float(g[f"{name}_maxabs"]) > 0.5  # the field moves


def test_full_size_engine_job_equals_reference(g):
    """One engine job with only the CDM stage (identity affine: the subject is copied
    onto the template grid) gives the reference's field at 182x218x182."""
    import tipl_b200 as tb

    It, Is = inputs(g, "full")
    out = np.zeros(It.shape + (3,), np.float32)
    with tb.Engine() as eng:
        jid = eng.submit(Is, fixed=It, linear=False, cdm=True, cdm_param=params("full"), field_out=out)
        r = eng.wait(jid)
    assert r["status"] == 0 and r["cdm_ok"]
    assert digest(out) == str(g["full_sha256"])
