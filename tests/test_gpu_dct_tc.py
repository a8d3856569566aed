"""The tcgen05 (3xBF16 split products, FP32 accumulate) Poisson solve against
the FP64 oracle and against the FP32 CUDA-core path.

Tolerances: the field and potential within 1e-4 of max|E| (max|phi|) of the
FP64 dense DCT restatement on the engine's own density map; a whole mGP run
reaches the same overflow target with iterations within 10% and HPWL within
0.5% of the FP32 path's run from the same start."""
import numpy as np
import pytest

from eplace_b200 import placer, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _engine(nl, mode, bins, keep=1):
    bx, by = bins if isinstance(bins, tuple) else (bins, bins)
    return placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=bx, bins_y=by,
                                                   dct_mode=mode, keep_maps=keep))


# 512 x 512 runs the split-K GEMMs (4-CTA clusters); the non-square grids
# give the two transforms different sizes
@pytest.mark.parametrize("bins", [(128, 128), (256, 256), (512, 512), (256, 128), (128, 384)])
def test_tensor_core_field_matches_fp64_oracle(bins):
    nl = synth.blob_start(synth.standard_cell(20_000, seed=5), sigma_frac=0.15)
    e = _engine(nl, placer.DCT_BF16X3, bins)
    assert (e.info.bins_x, e.info.bins_y) == bins and e.info.dct_mode == placer.DCT_BF16X3
    e.initialize()
    m = e.bin_maps()
    i = e.info
    bin_area = np.float64(np.float32(i.bin_step_x) * np.float32(i.bin_step_y))
    rho = (m["node"].astype(np.float64) + m["base"] + m["filler"] + m["terminal"]) / bin_area
    ex, ey, phi = O.poisson(rho, i.bin_step_x, i.bin_step_y)
    scale = max(np.abs(ex).max(), np.abs(ey).max())
    err_e = max(np.abs(m["ex"] - ex).max(), np.abs(m["ey"] - ey).max()) / scale
    err_p = np.abs(m["phi"] - phi).max() / np.abs(phi).max()
    assert err_e < 1e-4, err_e
    assert err_p < 1e-4, err_p


def test_tensor_core_run_matches_fp32_run():
    nl = synth.blob_start(synth.standard_cell(30_000, seed=6))
    out = {}
    for mode in (placer.DCT_FP32, placer.DCT_BF16X3):
        e = _engine(nl, mode, 128, keep=0)
        e.initialize()
        out[mode] = e.nesterov_run()
        e.close()
    a, b = out[placer.DCT_FP32], out[placer.DCT_BF16X3]
    assert b["overflow"] < 0.1
    assert abs(a["iterations"] - b["iterations"]) <= max(2, 0.1 * a["iterations"])
    assert b["hpwl"] == pytest.approx(a["hpwl"], rel=0.005)
