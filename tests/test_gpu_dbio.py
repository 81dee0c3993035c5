"""A device-resident time-step vector saved in the reference's on-disk format and loaded
back onto the device (one device-to-host and one host-to-device copy), then evaluated:
the residual of the reloaded vector equals the oracle's residual of the original."""
import numpy as np
import pytest

from bosss_b200 import dbio
from bosss_b200 import problems as P
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_device_vector_round_trip_and_residual(tmp_path):
    import torch
    pr = P.euler3d(n=6, k=2, seed=71)
    U = torch.tensor(pr.U, device="cuda")
    names = [f.name for f in pr.dom]
    vid = dbio.SaveFieldData(tmp_path, pr.dom, U)
    V = dbio.LoadFieldData(tmp_path, vid, pr.dom, names, device="cuda")
    assert V.is_cuda and torch.equal(U, V)
    with pr.evaluator() as ev:
        out = torch.zeros(ev.n_codomain, dtype=torch.float64, device="cuda")
        ev.Evaluate(1.0, 0.0, out, V)
        torch.cuda.synchronize()
    ref = orc.evaluate(*pr.descs(), pr.U)
    r = out.cpu().numpy()
    assert np.linalg.norm(r - ref) <= 1e-12 * np.linalg.norm(ref)
