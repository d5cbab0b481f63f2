"""GPU test of the bounded device wait: a wait that can never finish gives up, the host reads
the timeout as a status, and the context keeps working.  Nothing faults, traps or hangs: the
waiting warp stops after its time limit and the kernel exits normally."""
import time

import numpy as np
import pytest

from neural_wavelet_prt_demo_b200 import netconfig
from oracle import oracle as O
from tests.helpers import make_case, rel_err

pytestmark = pytest.mark.gpu


def test_device_wait_timeout_is_reported_and_the_context_survives(cuda):
    from neural_wavelet_prt_demo_b200 import engine as eng
    case = make_case(netconfig.CONFIG_SMALL, 24, 16, 16, seed=5, hash_scale=0.5)
    e = eng.RenderEngine(case.cfg)
    e.loadWeights(case.weights)
    env = e.addEnvironmentMap(eng.EnvironmentMap(top_coefficients=case.idx, top_strength=case.strength))
    fr = eng.FullFrame.from_gbuffer(case.gbuf)
    e.setFrame(0, fr)
    e.TCNNPass_p1(0)
    t0 = time.perf_counter()
    e.selftestDeviceWait(50)
    with pytest.raises(eng.NwprtError) as ei:
        e.TCNNSync()
    dt = time.perf_counter() - t0
    assert ei.value.status == eng._lib.TIMEOUT
    assert 0.04 < dt < 5.0                       # it waited about its limit, then gave up
    e.TCNNSync()                                  # the error word was cleared
    with pytest.raises(eng.NwprtError):
        e.selftestDeviceWait(0)                   # limit outside [1, 2000] ms
    # the context still relights correctly
    e.TCNNPass_p2(env, 0, eng.RenderConfig(precision="fp32"))
    e.TCNNSync()
    ind = fr.fbPredictedIndirect.cpu().numpy()
    rind, _ = O.relight_f32(case.bound, case.idx, case.strength)
    assert rel_err(ind[:, :3], rind[:, :3])[0] <= 1e-5
    e.close()
