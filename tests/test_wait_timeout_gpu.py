"""The failure path of the step kernels' bounded waits, made to run out without any GPU fault.

The 2-D acoustic FMA step kernels (tile and x-marching) wait for their TMA box loads on an
mbarrier with a time limit; when it runs out the CTA sets an error flag, waits (again with a
limit) for its own copies in flight and returns, and the call reports SFD_ERR_TIMEOUT.  The test
hook sfd_test_wait_timeout makes one CTA of one step issue no loads at all (so no copy is in
flight when it gives up) with a 100 us limit.  Checked for every schedule: the call returns
SFD_ERR_TIMEOUT, and after the hook is removed a forward on the same context returns SFD_OK with
records bit-identical to those of a fresh context."""
import numpy as np
import pytest

from conftest import bits_equal
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu


def engine_case():
    case = W.small_varden()
    rx, rz = case.receivers()
    w = S.wavelet(S.WAVELET_RIC, 120, case.dt, case.f0, 40)
    shots = [S.ShotSpec(case.src_x[0], case.src_z[0], rx, rz, w), S.ShotSpec(case.src_x[0] + 20, 30, rx, rz, w)]
    return case, shots


@pytest.mark.parametrize("env", [{"SFD_FMA_STAGES": "1"}, {"SFD_FMA_STAGES": "2"}, {"SFD_MARCH_SEG": "64"}],
                         ids=["tile", "persistent", "march"])
def test_timeout_is_reported_and_context_recovers(monkeypatch, env):
    for k in ("SFD_FMA_STAGES", "SFD_MARCH_SEG"):
        monkeypatch.delenv(k, raising=False)
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    case, shots = engine_case()
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model(case.vp, case.den)
        e.set_shots(shots)
        ref = e.forward().copy()
    with S.Engine(S.ACOUSTIC_2D, case.Nx, case.Nz, case.dx, case.dz, case.dt, case.PML, order=16) as e:
        e.set_model(case.vp, case.den)
        e.set_shots(shots)
        e.test_wait_timeout(0, 37, 1e-4)
        with pytest.raises(S.SfdError) as ei:
            e.forward()
        assert ei.value.status == S.ERR_TIMEOUT
        e.test_wait_timeout(-1, 0)
        got = e.forward().copy()
    assert np.abs(ref).max() > 0
    assert bits_equal(got, ref)
