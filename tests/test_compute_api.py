"""The Python force compute keeps the reference's surface (pymodule/compute.py:16-64)."""
import inspect
import math

import numpy as np
import pytest


def test_signature_matches_reference(product_lib):
    from conductorrigid_b200.compute import ConductorRigid

    sig = inspect.signature(ConductorRigid.__init__)
    names = list(sig.parameters)[1:9]
    assert names == ["group", "body", "charge", "field", "xi", "errortol", "fileprefix", "period"]
    d = {k: v.default for k, v in sig.parameters.items()}
    assert d["field"] == [0.0, 0.0, 0.0] and d["xi"] == 0.5 and d["errortol"] == 1e-3
    assert d["fileprefix"] == "" and d["period"] == 0
    for m in ("update_field", "update_parameters", "update_coeffs"):
        assert callable(getattr(ConductorRigid, m))


def test_refuses_without_cuda(product_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from conductorrigid_b200 import systems
    from conductorrigid_b200.compute import ConductorRigid

    s = systems.workload("plain_small", scale=0.3).system
    with pytest.raises(RuntimeError, match="Error creating ConductorRigid"):
        ConductorRigid("all", s.body, s.body_charge, system=s)
