"""Physics pin of the GPU viscoacoustic path (SFD_VISCOAC_2D through the C ABI, in both modes:
the reference-order kernels of SFD_EXACT and the default step and band kernels): measured attenuation and
dispersion against the 1-SLS law with the reference's Blanch tau (QS:473-551), at Q = 20, 60 and
200 on a homogeneous model, at the configuration's time step and at half of it (tests/qlaw.py
states the method and the laws).

  * discrete-time law of the reference's update (QS:993-1269): within 1 % at both time steps;
  * continuous 1-SLS law: within 6 % at dt = 0.5 ms, within 3.5 % at dt = 0.25 ms, and the gap
    shrinks by at least 40 % when dt halves -- the scheme converges to the analytic law, and the
    remaining gap is the first-order error of its explicit memory step."""
import numpy as np
import pytest

import oracle_lib as ol
from qlaw import GEOM, measure, rel_err
from seismic_code_github_b200 import seisfd as S

pytestmark = pytest.mark.gpu

QS = (20.0, 60.0, 200.0)


def gpu_records(q, dt, nt, flags):
    g = GEOM
    npx, nrz0 = g["npx"], g["nz"] // 2
    vp = np.full((g["nx"], g["nz"]), g["vp"], np.float32)
    vpp, rhop, qp = (S.pad_model(a, npx, npx, npx, npx) for a in (vp, np.full_like(vp, g["rho"]), np.full_like(vp, q)))
    decay = ol.q_decay(g["f0"], dt)
    with S.Engine(S.VISCOAC_2D, vpp.shape[0], vpp.shape[1], g["dx"], g["dx"], dt, npx, order=10, f0=g["f0"],
                  flags=flags) as e:
        e.set_model(vpp, rhop, qp)
        rx = np.arange(npx, vpp.shape[0] - npx, dtype=np.int32)
        rz = np.full_like(rx, npx + nrz0)
        e.set_shots([S.ShotSpec(npx + g["sx"], npx + nrz0, rx, rz, S.wavelet(S.WAVELET_Q, nt + decay, dt, g["f0"]))])
        rec = e.forward().reshape(len(rx), nt + decay)
    return rec[:, decay:]


@pytest.fixture(scope="module", params=[S.EXACT, 0], ids=["exact", "fused"])
def errors(request):
    g = GEOM
    out = {}
    for dt, nt in ((5e-4, 1200), (2.5e-4, 2400)):
        ref = gpu_records(1e5, dt, nt, request.param)
        for q in QS:
            m = measure(gpu_records(q, dt, nt, request.param), ref, g["sx"] + g["r1"], g["sx"] + g["r2"], g["r1"] * g["dx"],
                        g["r2"] * g["dx"], g["vp"], g["f0"], dt, q)
            out[(dt, q)] = {f"{k}_{law}": rel_err(m[k], m[f"{k}_{law}"]) for k in ("alpha", "disp")
                            for law in ("disc", "cont")}
            print(f"dt={dt} Q={q}: " + ", ".join(f"{k} {v:.4f}" for k, v in out[(dt, q)].items()))
    return out


@pytest.mark.parametrize("q", QS)
def test_gpu_attenuation_and_dispersion_follow_blanch_sls(errors, q):
    coarse, fine = errors[(5e-4, q)], errors[(2.5e-4, q)]
    for e in (coarse, fine):
        assert e["alpha_disc"] <= 0.01 and e["disp_disc"] <= 0.01
    assert coarse["alpha_cont"] <= 0.06 and coarse["disp_cont"] <= 0.05
    assert fine["alpha_cont"] <= 0.035 and fine["disp_cont"] <= 0.035
    assert fine["alpha_cont"] <= 0.6 * coarse["alpha_cont"]
