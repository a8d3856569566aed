"""The fast-transform (FP32 FFT) Poisson solve against the FP64 oracle and
against the FP32 dense path.

Tolerances: the field and potential within 2e-6 of max|E| (max|phi|) of the
FP64 dense DCT restatement on the engine's own density map (the FP32 dense
path itself stays within 6e-6 on these maps); a whole mGP run reaches the
same overflow target with iterations within 5% and HPWL within 0.2% of the
FP32 dense path's run from the same start."""
import numpy as np
import pytest

from eplace_b200 import placer, synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _engine(nl, mode, bx, by, keep=1):
    return placer.Engine(nl, placer.default_params(target_density=1.0, bins_x=bx, bins_y=by,
                                                   dct_mode=mode, keep_maps=keep))


@pytest.mark.parametrize("bx,by", [(8, 8), (16, 64), (128, 128), (256, 64), (512, 512), (1024, 1024)])
def test_fft_field_matches_fp64_oracle(bx, by):
    nl = synth.blob_start(synth.standard_cell(20_000, seed=5), sigma_frac=0.15)
    e = _engine(nl, placer.DCT_FFT, bx, by)
    assert e.info.dct_mode == placer.DCT_FFT
    e.initialize()
    m = e.bin_maps()
    i = e.info
    bin_area = np.float64(np.float32(i.bin_step_x) * np.float32(i.bin_step_y))
    rho = (m["node"].astype(np.float64) + m["base"] + m["filler"] + m["terminal"]) / bin_area
    ex, ey, phi = O.poisson(rho, i.bin_step_x, i.bin_step_y)
    scale = max(np.abs(ex).max(), np.abs(ey).max())
    err_e = max(np.abs(m["ex"] - ex).max(), np.abs(m["ey"] - ey).max()) / scale
    err_p = np.abs(m["phi"] - phi).max() / np.abs(phi).max()
    assert err_e < 2e-6, err_e
    assert err_p < 2e-6, err_p


def test_fft_rejects_other_bin_counts():
    nl = synth.standard_cell(2_000, seed=1)
    with pytest.raises(placer.EPError) as ex:
        _engine(nl, placer.DCT_FFT, 96, 96)
    assert ex.value.status == placer.EP_ERR_UNSUPPORTED


def test_fft_run_matches_fp32_run():
    nl = synth.blob_start(synth.standard_cell(30_000, seed=6))
    out = {}
    for mode in (placer.DCT_FP32, placer.DCT_FFT):
        e = _engine(nl, mode, 128, 128, keep=0)
        e.initialize()
        out[mode] = e.nesterov_run()
        e.close()
    a, b = out[placer.DCT_FP32], out[placer.DCT_FFT]
    assert b["overflow"] < 0.1
    assert abs(a["iterations"] - b["iterations"]) <= max(2, 0.05 * a["iterations"])
    assert b["hpwl"] == pytest.approx(a["hpwl"], rel=0.002)
