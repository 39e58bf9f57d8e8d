"""The 2-D CDM (cdm_common<out, unsigned char, 2>, the reference's cdm_cuda<tipl::out,
unsigned char, 2> instantiation of reg/cdm_cu.hpp:12-17) through the C ABI
(regb_cdm2d_multi, via tb.reg.cdm on 2-D arrays) against the reference's own CPU
branch: fixture tests/golden/cdm2d.npz (tests/golden/make_golden.py --only cdm2d) holds
the inputs and the SHA-256 of the reference's field.  The bar is bit-for-bit equality
(reg/cdm.hpp:373-474 at dimension 2)."""
import hashlib
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g(golden):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return golden("cdm2d")


def cases():
    from make_golden import CDM2D_CASES

    return list(enumerate(CDM2D_CASES))


@pytest.mark.parametrize("k,case", cases())
def test_cdm2d_equals_reference(g, k, case):
    import tipl_b200 as tb

    shape, res, md, gt, nmod, _ = case
    It = [g[f"c{k}_It{i}"] for i in range(nmod)]
    Is = [g[f"c{k}_Is{i}"] for i in range(nmod)]
    p = tb.reg.cdm_param(resolution=res, min_dimension=md)
    field, ok = tb.reg.cdm(It if nmod > 1 else It[0], Is if nmod > 1 else Is[0], p,
                           gradient_types=gt if gt else None)
    assert int(ok) == int(g[f"c{k}_ok"])
    if ok:
        assert field.shape == tuple(shape) + (2,)
        assert hashlib.sha256(np.ascontiguousarray(field).tobytes()).hexdigest() == str(g[f"c{k}_sha256"])
        assert float(np.abs(field).max()) == float(g[f"c{k}_maxabs"])


def test_cdm2d_device_tensors_and_arguments(g):
    """Device-resident 2-D images give the host result; float 2-D images and
    min_dimension 0 on a one-pixel axis are argument errors."""
    import torch

    import tipl_b200 as tb
    from tipl_b200 import _lib

    It, Is = g["c0_It0"], g["c0_Is0"]
    host, ok = tb.reg.cdm(It, Is)
    dev, ok2 = tb.reg.cdm(torch.from_numpy(It).cuda(), torch.from_numpy(Is).cuda())
    assert ok and ok2 and np.array_equal(dev.cpu().numpy().view(np.uint32), host.view(np.uint32))
    with pytest.raises(_lib.RegbError):
        tb.reg.cdm(It.astype(np.float32), Is.astype(np.float32))
    with pytest.raises(_lib.RegbError):
        tb.reg.cdm(It[:1], Is[:1], tb.reg.cdm_param(min_dimension=0))
