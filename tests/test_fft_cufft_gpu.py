"""Cross-check of the device's hand-written FFT passes against cuFFT.

The PM solve's spectral pipeline (forward 3D transform of the density,
Green's function x Gaussian filter x spectral gradient, three inverse 3D
transforms: crates/gadget-ng-pm/src/fft_poisson.rs:306-550, :724-813) is
restated with torch.fft on the GPU in float64 (torch's CUDA FFT is cuFFT), on
the device's own density mesh, and compared with the device's force meshes.
cuFFT serves here only as a second transform to check against; it is not on
the solver's path.  Tolerance: 2e-6 of the rms force (the device transforms in
FP32).
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cufft_forces(rho, g, nm, box, r_split):
    import torch
    dev = torch.device("cuda", 0)
    cl = box / nm
    r = torch.from_numpy(rho.astype(np.float64).reshape(nm, nm, nm)).to(dev) / (cl * (cl * cl))
    rk = torch.fft.fftn(r.to(torch.complex128))  # axes (z, y, x), unnormalised
    j = torch.arange(nm, device=dev, dtype=torch.float64)
    k = (2.0 * math.pi / box) * torch.where(j <= nm // 2, j, j - nm)  # freq_index
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    filt = torch.exp(-0.5 * k2 * r_split * r_split)
    green = torch.where(k2 < 1e-30, torch.zeros_like(k2), -4.0 * math.pi * g * filt / torch.where(k2 < 1e-30, 1.0, k2))
    phi = rk * green
    out = []
    for kk in (kx, ky, kz):
        f = torch.complex(kk * phi.imag, -kk * phi.real)  # -i k phi
        out.append((torch.fft.ifftn(f).real).reshape(-1).cpu().numpy())  # ifftn includes 1 / nm^3
    return out


@pytest.mark.parametrize("nm,kind", [(64, "clustered"), (32, "lattice")])
def test_device_fft_passes_match_cufft(nm, kind):
    import treepm
    from treepm import ics
    if kind == "clustered":
        box = ics.clustered_box(nm, 50.0, 0.3, 20, min_halo=100, max_halo=5000, r_min=0.1, r_max=0.5, seed=71)
    else:
        box = ics.lattice_box(nm, 100.0, 1.0, seed=72)
    phys = ics.physics(box, nm, 0.1)
    s = treepm.TreePmSolver(nm, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"], device=0)
    s.accelerations_for_indices(box.positions(), box.mass, phys["eps2"], 1.0, [0])
    rho, fx, fy, fz = s.mesh()
    s.close()
    want = _cufft_forces(rho, 1.0, nm, box.box_size, phys["r_split"])
    for got, ref in zip((fx, fy, fz), want):
        rms = math.sqrt(float(np.mean(ref * ref)))
        err = math.sqrt(float(np.mean((got.astype(np.float64) - ref) ** 2)))
        assert err < 2e-6 * rms, (err / rms)
