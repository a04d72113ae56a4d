"""Dataset preprocessing on the GPU (centre of mass + intensity normalisation,
PtychographyDatasetRaster.preprocess) against the reference's own set-up
products (golden fixtures) and against the host path on a larger, off-centre
dataset with a plane CoM fit."""
import numpy as np
import pytest
import torch

from tests.conftest import load_golden, rel
from tests.test_host_setup import build_from_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["single64", "mixed64"])
def test_gpu_preprocess_matches_reference(cuda_device, case):
    z = load_golden(case)
    pt = build_from_golden(z, device="cuda")
    d = pt.dset
    assert d._preprocessed_on == "gpu"
    assert d.targets.is_cuda
    assert abs(d.mean_diffraction_intensity - float(z["mean_intensity"])) / float(z["mean_intensity"]) < 1e-6
    assert rel(d.targets.cpu().numpy(), z["targets"]) < 1e-5  # FP32 transforms vs the reference's FP64 numpy


@pytest.mark.parametrize("n", [96, 128])
def test_gpu_preprocess_matches_host_path(cuda_device, n):
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster

    rng = np.random.default_rng(n)
    nscan = 12
    yy, xx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    data = np.empty((nscan, nscan, n, n), np.float32)
    for i in range(nscan):
        for j in range(nscan):  # a bright disc whose centre drifts over the scan (descan)
            cy, cx = n / 2 + 3.0 * i / nscan + 0.37, n / 2 - 2.0 * j / nscan + 0.11
            disc = ((yy - cy) ** 2 + (xx - cx) ** 2 < (n / 6) ** 2).astype(np.float32)
            data[i, j] = rng.poisson(200.0 * disc + 0.5)
    data[0, 0, 5, 5] = -3.0  # negative counts are clipped like the reference
    out = {}
    for dev in ("cpu", "cuda"):
        d4 = Dataset4dstem.from_array(data, sampling=(1.0, 1.0, 0.05, 0.05), units=("A", "A", "A^-1", "A^-1"))
        pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
        pd.preprocess(com_fit_function="plane", force_com_rotation=0, force_com_transpose=False,
                      plot_rotation=False, plot_com=False, probe_energy=300e3, device=dev)
        out[dev] = pd
    h, g = out["cpu"], out["cuda"]
    assert h._preprocessed_on == "host" and g._preprocessed_on == "gpu"
    assert np.abs(np.asarray(g.com_measured) - np.asarray(h.com_measured)).max() < 1e-4
    assert np.abs(np.asarray(g.com_fit) - np.asarray(h.com_fit)).max() < 1e-4
    assert abs(g.mean_diffraction_intensity - h.mean_diffraction_intensity) / h.mean_diffraction_intensity < 1e-6
    assert rel(g.centered_amplitudes.cpu().numpy(), h.centered_amplitudes.numpy()) < 1e-5
    assert rel(g.amplitudes.cpu().numpy(), h.amplitudes.numpy()) < 1e-6
    assert g.com_rotation_rad == h.com_rotation_rad and g.com_transpose == h.com_transpose


@pytest.mark.parametrize("fit", ["plane", "constant"])
def test_gpu_bilinear_centring_matches_reference(cuda_device, fit):
    """preprocess(bilinear=True) on the GPU (ptycho_pattern_bilinear) against the reference's
    own centred targets (fixture bilinear64) and the host path."""
    from quantem_b200.diffractive_imaging import Dataset4dstem, PtychographyDatasetRaster

    z = load_golden("bilinear64")
    H, nscan = int(z["H"]), int(z["nscan"])
    px, step = float(z["px"]), float(z["step_px"])
    rs = 1.0 / (H * px)
    out = {}
    for dev in (cuda_device, "cpu"):
        d4 = Dataset4dstem.from_array(z["data"].reshape(nscan, nscan, H, H),
                                      sampling=(step * px, step * px, rs, rs), units=("A", "A", "A^-1", "A^-1"))
        pd = PtychographyDatasetRaster.from_dataset4dstem(d4, verbose=0)
        pd.preprocess(com_fit_function=fit, force_com_rotation=0, force_com_transpose=False, bilinear=True,
                      plot_rotation=False, plot_com=False, probe_energy=float(z["energy"]), device=dev)
        out[str(dev)] = pd
    g = out[str(cuda_device)]
    assert g._preprocessed_on == "gpu" and out["cpu"]._preprocessed_on == "host"
    assert rel(g.targets.cpu().numpy(), z[f"targets_{fit}"]) < 1e-6
    assert rel(g.targets.cpu().numpy(), out["cpu"].targets.numpy()) < 1e-6
    assert abs(g.mean_diffraction_intensity - float(z[f"mean_intensity_{fit}"])) <= 1e-6 * g.mean_diffraction_intensity
