"""The C-ABI gradients behind torch.autograd (tests/autograd_harness.py): an L2 loss written in
torch back-propagates through the library's adjoint to the same model gradient sfd_gradient
returns directly, and a torch-level central difference along a smooth direction agrees with it."""
import numpy as np
import pytest
import torch
from scipy.ndimage import gaussian_filter

from autograd_harness import AcousticRecords, ViscoacousticRecords
from conftest import rel_l2
from seismic_code_github_b200 import seisfd as S
from seismic_code_github_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_acoustic_autograd_matches_c_abi_gradient():
    PML = 10
    vp = W.pad_edges(W.layered_model(40, 30, 3, 1800.0, 2600.0, seed=2, anomalies=1, radius=5.0, amp=150.0),
                     PML, PML)
    den = np.full(vp.shape, 2100.0, np.float32)
    rx = np.arange(PML, vp.shape[0] - PML, 2, dtype=np.int32)
    shots = [S.ShotSpec(25, PML + 3, rx, np.full_like(rx, PML + 2), S.wavelet(S.WAVELET_RIC, 150, 1e-3, 25.0, 40))]
    with S.Engine(S.ACOUSTIC_2D, vp.shape[0], vp.shape[1], 10.0, 10.0, 1e-3, PML, order=16) as e:
        e.set_model((vp * 1.03).astype(np.float32), den)
        e.set_shots(shots)
        obs = e.forward()
        m = torch.tensor(vp, requires_grad=True)
        rec = AcousticRecords.apply(m, e, den)
        loss = 0.5 * torch.sum((rec.double() - torch.from_numpy(obs).double()) ** 2)
        loss.backward()
        e.set_model(vp, den)
        J, g, _ = e.gradient(obs)
        err = rel_l2(m.grad.numpy(), g)
        print(f"acoustic: torch loss {loss.item():.6e} vs misfit {J:.6e}; gradient relL2 {err:.2e}")
        assert abs(loss.item() - J) <= 1e-5 * J
        assert err <= 1e-5
        d = torch.from_numpy(gaussian_filter(np.random.default_rng(4).standard_normal(vp.shape), 4))
        d = 1e-3 * torch.from_numpy(vp).double() * d / d.abs().max()
        Js = []
        for sgn in (1.0, -1.0):
            with torch.no_grad():
                r = AcousticRecords.apply((torch.from_numpy(vp).double() + sgn * d).float(), e, den)
                Js.append(0.5 * torch.sum((r.double() - torch.from_numpy(obs).double()) ** 2).item())
        fd = (Js[0] - Js[1]) / 2.0
        an = float(torch.sum(m.grad.double() * d))
        assert abs(fd - an) <= 2e-2 * abs(an), (fd, an)


def test_viscoacoustic_autograd_matches_c_abi_gradient():
    NPX, F0, DT, DX = 8, 20.0, 5e-4, 10.0
    rng = np.random.default_rng(0)
    pad = lambda a: S.pad_model(a.astype(np.float32), NPX, NPX, NPX, NPX)
    vp = pad(2000 + 400 * gaussian_filter(rng.random((40, 32)), 3))
    rho = pad(1900 + 400 * rng.random((40, 32)))
    q = pad(30 + 120 * gaussian_filter(rng.random((40, 32)), 2))
    rx = np.arange(NPX, vp.shape[0] - NPX, 2, dtype=np.int32)
    shots = [S.ShotSpec(27, NPX + 4, rx, np.full_like(rx, NPX + 2), S.wavelet(S.WAVELET_Q, 160, DT, F0))]
    with S.Engine(S.VISCOAC_2D, vp.shape[0], vp.shape[1], DX, DX, DT, NPX, order=10, f0=F0, flags=S.EXACT) as e:
        e.set_model((vp * 1.02).astype(np.float32), rho, (q * 0.8).astype(np.float32))
        e.set_shots(shots)
        obs = e.forward()
        m = torch.tensor(vp, requires_grad=True)
        iq = torch.tensor((1.0 / q.astype(np.float64)).astype(np.float32), requires_grad=True)
        rec = ViscoacousticRecords.apply(m, iq, e, rho)
        loss = 0.5 * torch.sum((rec.double() - torch.from_numpy(obs).double()) ** 2)
        loss.backward()
        e.set_model(vp, rho, q)
        J, gv, gq = e.gradient(obs, want_invq=True)
        ev, eq = rel_l2(m.grad.numpy(), gv), rel_l2(iq.grad.numpy(), gq)
        print(f"viscoacoustic: torch loss {loss.item():.6e} vs misfit {J:.6e}; relL2 vp {ev:.2e}, 1/Q {eq:.2e}")
        assert abs(loss.item() - J) <= 1e-5 * J
        assert ev <= 1e-5 and eq <= 1e-5
