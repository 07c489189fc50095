"""Mixed-precision (split-BF16 tcgen05) Fourier transform vs the FP64 oracle.

Tolerance: the split BF16x3 product with FP32 accumulation is at the FP32 level; the normwise
relative error of each output column must be <= 2e-6 and every element within 1e-5 of the column
maximum (the |g|^2 budget of 1e-5 relative needs g at <= 5e-6).
"""
import numpy as np
import pytest

from oracle import epb_oracle as O
from epb200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def B(gpu_lib):
    from epb200 import batched

    return batched


def _dev_obj(irvec, op, ndata=None):
    from epb200.wannier import WannierObject, to_device

    return to_device(WannierObject(irvec, op, ndata=ndata))


@pytest.mark.parametrize("ndata,rmax,nk,decay", [(64, 3, 300, 1.5), (256, 4, 129, 1.5), (7, 2, 5, 0.0),
                                                (384, 2, 257, 2.0)])
def test_fourier_mixed(B, ndata, rmax, nk, decay):
    rng = np.random.default_rng(ndata + nk)
    irvec = synth.irvec_box(rmax)
    nr = irvec.shape[0]
    w = np.exp(-np.linalg.norm(irvec, axis=1) / decay) if decay else np.ones(nr)
    op = np.asfortranarray((rng.standard_normal((ndata, nr)) + 1j * rng.standard_normal((ndata, nr))) * w[None, :])
    obj = _dev_obj(irvec, op)
    xk = rng.random((3, nk))
    out = B.host(B.get_fourier_batched(B.get_interpolator(obj), xk, prec=B.PREC_MIXED))
    ref = O.fourier_batched(op, ndata, irvec, xk)
    colnorm = np.linalg.norm(ref, axis=0)
    rel = np.linalg.norm(out - ref, axis=0) / colnorm
    assert rel.max() <= 2e-6, rel.max()
    assert np.max(np.abs(out - ref) / np.abs(ref).max(axis=0)) <= 1e-5
