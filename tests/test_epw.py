"""EPW model reader (src/model_new.jl): the text parsers on CPU, the epmatwp streaming reader on the GPU
bit-exact against the numpy restatement of read_epmat (both layouts, per-orbital and scalar
Wigner-Seitz degeneracies, zeros, pre-divided files, the skipped phonon-side division), and the
FP64 e-ph pass on the loaded model equal to the pass on the model that was written."""
import os

import numpy as np
import pytest

from epb200 import synth
from oracle import epb_oracle as O
from oracle import epw_oracle as EO

from epw_files import write_epw_folder

NATOM = 2


def _model(seed=7, nw=4):
    return synth.config2_model(seed=seed, n_el=1, n_ph=1, nw=nw, natom=NATOM)


def _sorted_equal(a_op, b_op, rtol):
    np.testing.assert_allclose(a_op, b_op, rtol=rtol, atol=rtol * np.abs(b_op).max())


@pytest.mark.parametrize("intel,new_wigner,per_orb", [(False, False, True), (True, False, False),
                                                     (False, True, True), (True, True, False)])
def test_parsers_round_trip(tmp_path, intel, new_wigner, per_orb):
    from epb200 import epw

    m = _model()
    write_epw_folder(str(tmp_path), m, NATOM, intel=intel, new_wigner=new_wigner, ndegen_per_orbital=per_orb)
    em = epw.load_model_from_epw(str(tmp_path), "out", "test", load_epmat=False)
    assert (em.nw, em.nmodes) == (m.nw, m.nmodes)
    np.testing.assert_array_equal(em.el_ham.irvec, m.el_ham.irvec)
    np.testing.assert_array_equal(em.ph_dyn.irvec, m.ph_dyn.irvec)
    np.testing.assert_array_equal(em.mass, m.mass)
    _sorted_equal(em.el_ham.op_r, m.el_ham.op_r, 1e-15)
    _sorted_equal(em.ph_dyn.op_r, m.ph_dyn.op_r, 1e-15)
    assert em.epmat is None and em.epmat_outer_momentum == "nothing"


def test_oracle_read_epmat_round_trip(tmp_path):
    """The restatement recovers the written model in both layouts (pins it against the writer)."""
    from epb200 import epw
    from epb200.wannier import sort_irvec

    m = _model()
    info = write_epw_folder(str(tmp_path), m, NATOM)
    st = epw.parse_structure(str(tmp_path))
    w = epw.read_wigner(str(tmp_path), st["ws_method"], st["ndegen_pre_divided"])
    nw, nm = m.nw, m.nmodes
    ie, ip = sort_irvec(w["el"][0]), sort_irvec(w["ep"][0])
    fn = os.path.join(str(tmp_path), "out", "test.epmatwp")
    el = EO.read_epmat(fn, nw, nm, w["nr_el"], w["nr_ep"], ie, ip, w["el"][1][:, :, ie], w["ep"][1][:, :, ip])
    _sorted_equal(el, m.epmat.op_r, 1e-15)
    ph = EO.read_epmat(fn, nw, nm, w["nr_el"], w["nr_ep"], ie, ip, w["el"][1][:, :, ie], w["ep"][1][:, :, ip],
                       layout="ph")
    np.testing.assert_array_equal(ph, O.epmat_el_to_ph(el, nw, nm, w["nr_el"], w["nr_ep"]))


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["el", "ph"])
@pytest.mark.parametrize("case", ["per_orbital", "scalar", "zeros", "predivided", "skip_ep"])
def test_read_epmat_bit_exact(gpu_lib, tmp_path, layout, case):
    from epb200 import epw
    from epb200.wannier import sort_irvec

    kw = dict(per_orbital=dict(), scalar=dict(ndegen_per_orbital=False), zeros=dict(zero_ndegen=True),
              predivided=dict(new_wigner=True, ws_method=2), skip_ep=dict(new_wigner=True, ws_method=3))[case]
    m = _model(seed=11, nw=5)
    info = write_epw_folder(str(tmp_path), m, NATOM, seed=3, **kw)
    em = epw.load_model_from_epw(str(tmp_path), "out", "test", epmat_outer_momentum=layout)
    st = epw.parse_structure(str(tmp_path))
    w = epw.read_wigner(str(tmp_path), st["ws_method"], st["ndegen_pre_divided"])
    ie, ip = sort_irvec(w["el"][0]), sort_irvec(w["ep"][0])
    ref = EO.read_epmat(os.path.join(str(tmp_path), "out", "test.epmatwp"), m.nw, m.nmodes, w["nr_el"], w["nr_ep"],
                        ie, ip, w["el"][1][:, :, ie], w["ep"][1][:, :, ip], layout=layout,
                        skip_ndegen_ep=w["skip_eph_ndegen"], ndegen_pre_divided=st["ndegen_pre_divided"])
    got = em.epmat.op_r.cpu().numpy().T
    np.testing.assert_array_equal(got, ref)
    if case != "zeros":
        want = m.epmat.op_r if layout == "el" else O.epmat_el_to_ph(m.epmat.op_r, m.nw, m.nmodes, w["nr_el"],
                                                                      w["nr_ep"])
        _sorted_equal(got, want, 1e-15)


@pytest.mark.gpu
def test_epw_model_runs_the_pass(gpu_lib, tmp_path):
    """The FP64 e-ph pass on the loaded model equals the pass on the written model."""
    from epb200 import epw, pipeline

    m = _model(seed=13, nw=8)
    write_epw_folder(str(tmp_path), m, NATOM, seed=5)
    em = epw.load_model_from_epw(str(tmp_path), "out", "test")
    xk = synth.random_kpoints(6, 1)
    xq = synth.random_kpoints(40, 2)
    r0 = pipeline.run_eph_over_k_and_q(pipeline.DeviceModel(m), xk, xq, sample_stride=1)
    r1 = pipeline.run_eph_over_k_and_q(pipeline.DeviceModel(em), xk, xq, sample_stride=1)
    np.testing.assert_allclose(r1.g2sum.cpu().numpy(), r0.g2sum.cpu().numpy(), rtol=1e-12)
    np.testing.assert_allclose(r1.g2_sample.cpu().numpy(), r0.g2_sample.cpu().numpy(), rtol=1e-10, atol=1e-14)


@pytest.mark.gpu
def test_read_epmat_errors(gpu_lib, tmp_path):
    import torch

    from epb200 import _lib
    from epb200._lib import EpbError

    m = _model()
    write_epw_folder(str(tmp_path), m, NATOM)
    fn = os.path.join(str(tmp_path), "out", "test.epmatwp")
    nw, nm, ne, npp = m.nw, m.nmodes, m.el_ham.irvec.shape[0], m.epmat.irvec_next.shape[0]
    out = torch.empty(nw * nw * nm * ne * npp, dtype=torch.complex128, device="cuda")
    ie = np.arange(1, ne + 1, dtype=np.int64)
    ip = np.arange(1, npp + 1, dtype=np.int64)
    one = np.ones(max(ne, npp), dtype=np.int32)
    ctx = _lib.default_context()
    call = lambda f, ie_, ip_, nr_ep: _lib.check(_lib.lib().epb_read_epmat(
        ctx.h, f, nw, nm, ne, nr_ep, ie_.ctypes.data, ip_.ctypes.data, one.ctypes.data, 1, one.ctypes.data, 1, 1, 0, 0,
        0, out.data_ptr()))
    call(fn.encode(), ie, ip, npp)  # valid
    with pytest.raises(EpbError, match="expected"):  # file shorter than the sizes say
        call(fn.encode(), np.arange(1, ne + 1, dtype=np.int64), np.arange(1, npp + 2, dtype=np.int64), npp + 1)
    bad = ie.copy()
    bad[0] = bad[1]
    with pytest.raises(EpbError, match="permutation"):
        call(fn.encode(), bad, ip, npp)
    with pytest.raises(EpbError, match="cannot open"):
        call(b"/nonexistent/x.epmatwp", ie, ip, npp)
