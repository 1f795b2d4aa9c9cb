"""Failure detection without a GPU fault: every wait in the cache kernels is
bounded in time and reports through an error flag the host turns into
TFG_E_TIMEOUT.  The diagnostic entry runs that path on a wait that can never
complete (an mbarrier nothing arrives on) with a short limit; afterwards the
context is intact and the cache kernels run normally."""
import time

import numpy as np
import pytest
import torch

from tfg_b200 import TfgError, _lib
from tfg_b200.nrc import ColorMLP
from tfg_b200.structs import DATOS_MLP

pytestmark = pytest.mark.gpu

TFG_E_TIMEOUT = 10003


def test_stuck_wait_reports_timeout_and_the_context_survives(built):
    t0 = time.perf_counter()
    with pytest.raises(TfgError) as ei:
        _lib.call("tfgMlpSelfTestWait", 2000)          # 2 ms limit
    assert ei.value.code == TFG_E_TIMEOUT
    assert time.perf_counter() - t0 < 5.0
    assert _lib.lib.tfgMlpStatus() == 0                 # the flag was consumed
    # the device still works: a cache inference afterwards is finite
    m = ColorMLP(batch=1024, seed=1)
    n = 300
    d = np.zeros(n, DATOS_MLP)
    d["posicion"]["x"] = np.linspace(-1, 1, n)
    out = torch.zeros(n * 3, device="cuda")
    m.inference(torch.from_numpy(d.view(np.uint8).copy()).cuda(), out, n)
    torch.cuda.synchronize()
    assert np.isfinite(out.cpu().numpy()).all()
    m.close()


def test_self_test_rejects_unbounded_limits(built):
    for bad in (0, 3_000_000):
        with pytest.raises(TfgError):
            _lib.call("tfgMlpSelfTestWait", bad)
