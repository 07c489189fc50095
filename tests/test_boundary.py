"""Entry points that take the reference methods' own operands: fourier_phase!(phase, irvec_mat, xkmat)
on device matrices and views (src/wannier/batched_fourier_core.jl:24-30; call sites
src/calculator/run_eph_over_k_and_kq.jl:821,856 and batched_fourier_core.jl:104), and batched_gemm!
(src/common/gpu_utils.jl:71-78) with every op combination, padded leading dimensions and strided batches.
"""
import numpy as np
import pytest

from epb200 import synth
from oracle import epb_oracle as O


@pytest.mark.gpu
def test_fourier_phase_mat_views(gpu_lib):
    """P_mk[:, 1:nk] .= cispi(2 R . x) from the (nr x 3) FP64 R matrix and a column view of the k list:
    within 4 eps of the oracle (the reference's own phase test bar, test/test_gpu.jl:127-144); the
    columns outside the view are untouched."""
    import torch

    from epb200 import batched as B

    irvec = synth.irvec_box(2)
    nr = irvec.shape[0]
    xall = synth.random_kpoints(40, 71) * 3 - 1  # coordinates outside [0, 1) too
    irvec_mat = B.jl(irvec.astype(np.float64))   # (nr, 3) column-major
    xkmat = B.jl(xall)                           # (3, 40)
    phase = B.jl(np.full((nr, 48), 7.0 + 0j))    # (nr, 48); the view is columns 5..34
    view = phase[5:35, :]
    B.fourier_phase_mat(view, irvec_mat, xkmat[3:33, :])
    torch.cuda.synchronize()
    got = B.host(phase)
    ref = O.fourier_phase(irvec, np.asfortranarray(xall[:, 3:33]))
    assert np.abs(got[:, 5:35] - ref).max() <= 4 * np.finfo(float).eps
    assert np.all(got[:, :5] == 7.0) and np.all(got[:, 35:] == 7.0)


def _op(t, x):
    return x if t == "N" else (np.swapaxes(x, 0, 1) if t == "T" else np.conj(np.swapaxes(x, 0, 1)))


@pytest.mark.gpu
@pytest.mark.parametrize("m,n,k,nb", [(5, 7, 3, 4), (16, 192, 16, 3), (33, 17, 40, 2), (256, 12, 12, 5)])
def test_batched_gemm_all_ops(gpu_lib, m, n, k, nb):
    """Every (transA, transB) in {N, T, C}^2 against numpy (FP64, 1e-13 relative), operands taken as
    views with a padded leading dimension and a strided batch axis."""
    import torch

    from epb200 import batched as B

    rng = np.random.default_rng(m * 1000 + n)
    for ta in "NTC":
        for tb in "NTC":
            ash = (m, k) if ta == "N" else (k, m)
            bsh = (k, n) if tb == "N" else (n, k)
            a_big = synth.cnormal(rng, (ash[0] + 3, ash[1], 2 * nb))   # lda = rows + 3, every other batch
            b_big = synth.cnormal(rng, (bsh[0] + 1, bsh[1], nb))
            A = B.jl(a_big)[::2, :, :ash[0]]
            Bm = B.jl(b_big)[:, :, :bsh[0]]
            C = B.jl_empty((m, n, nb), torch.complex128)
            B.batched_gemm(ta, tb, A, Bm, C)
            torch.cuda.synchronize()
            a, b = a_big[:ash[0], :, ::2], b_big[:bsh[0], :, :]
            ref = np.stack([_op(ta, a[:, :, i]) @ _op(tb, b[:, :, i]) for i in range(nb)], axis=2)
            got = B.host(C)
            assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max()) * np.sqrt(k), (ta, tb)


@pytest.mark.gpu
def test_batched_gemm_rejects_bad_arguments(gpu_lib):
    from epb200 import _lib

    lib = gpu_lib
    ctx = _lib.default_context()
    st = lib.epb_batched_zgemm(ctx.h, b"X", b"N", 2, 2, 2, None, 2, 4, None, 2, 4, None, 2, 4, 1)
    assert st == _lib.EPB_ERR_ARG
    st = lib.epb_batched_zgemm(ctx.h, b"N", b"N", 4, 2, 2, 1, 2, 8, 1, 2, 4, 1, 4, 8, 1)  # lda < m
    assert st == _lib.EPB_ERR_ARG
