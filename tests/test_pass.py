"""The whole e-ph pass: CPU batched port vs the per-pair oracle (CPU), and the GPU pass vs both.

Comparisons of g2 per band are gauge-sensitive only through degenerate bands; random models have
none, so per-band values are compared directly, and band/q sums (gauge invariant) tightly.
"""
import numpy as np
import pytest

from oracle import cpu_pass, epb_oracle as O
from epb200 import synth


def _small(seed=21, nw=6, natom=2):
    return synth.config2_model(seed=seed, n_el=2, n_ph=1, nw=nw, natom=natom)


def test_cpu_pass_matches_per_pair_oracle():
    m = _small()
    xks = synth.random_kpoints(3, 1)
    xqs = synth.random_kpoints(10, 2)
    res = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=3)
    pairs = O.eph_pairs(m, xks, xqs, [(k, q) for k in range(3) for q in range(10)])
    for k in range(3):
        tot = sum(p["g2"].sum(axis=(0, 1)) for p in pairs if p["ik"] == k)
        np.testing.assert_allclose(res["g2sum"][:, k], tot, rtol=1e-10)
        for j, q in enumerate(range(0, 10, 3)):
            ref = [p for p in pairs if p["ik"] == k and p["iq"] == q][0]["g2"]
            np.testing.assert_allclose(res["g2_sample"][:, :, :, j, k], ref, rtol=1e-8, atol=1e-12 * ref.max())


@pytest.mark.gpu
@pytest.mark.parametrize("nw,natom,nk,nq,kb", [(6, 2, 7, 40, 3), (16, 4, 5, 64, 2)])
def test_gpu_pass_fp64(gpu_lib, nw, natom, nk, nq, kb):
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=31, n_el=2, n_ph=1, nw=nw, natom=natom)
    xks = synth.random_kpoints(nk, 3)
    xqs = synth.random_kpoints(nq, 4)
    dm = pipeline.DeviceModel(m)
    r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_FP64, k_batch=kb, sample_stride=7)
    ref = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=7)
    np.testing.assert_allclose(host(r.ek), ref["ek"], atol=1e-11 * np.abs(ref["ek"]).max())
    np.testing.assert_allclose(host(r.omega), ref["omega"], rtol=1e-10)
    np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-9)
    s, sr = host(r.g2_sample), ref["g2_sample"]
    np.testing.assert_allclose(s, sr, rtol=1e-7, atol=1e-10 * sr.max())
    assert r.n_elements == nk * nq * nw * nw * 3 * natom


def _block_rel_err(s, sr):
    """Per sampled (k, q) block: ||g2 - g2_ref||_F / ||g2_ref||_F (max over blocks)."""
    d = s - sr
    num = np.sqrt((np.abs(d) ** 2).sum(axis=(0, 1, 2)))
    den = np.sqrt((np.abs(sr) ** 2).sum(axis=(0, 1, 2)))
    return (num / den).max()


def _force_kq_form(ctx, nq, form):
    """Load a kR->kq GEMM form (0 streamed operands, 1 A tile resident in shared memory) for the
    mixed pass of nw = 16, nm = 12 and this q count into the context's tuning table."""
    from epb200 import _lib, pipeline

    _lib.TuneTable(f"pass_kq/16/12/{nq}/{pipeline.PREC_MIXED} {form}\n").import_into(ctx)


@pytest.mark.gpu
@pytest.mark.parametrize("kq", [1, 0])
@pytest.mark.parametrize("rot", [0, 1])
@pytest.mark.parametrize("nk,nq,kb", [(5, 64, 2), (3, 200, 3)])
def test_gpu_pass_mixed(gpu_lib, nk, nq, kb, rot, kq):
    """Mixed-precision pass vs the FP64 CPU port: |g|^2 normwise error per (k, q) block <= 1e-5,
    band/q sums <= 1e-6, electron energies (FP64 k side) and phonons at the FP64 level; both rotation
    kernels (0: warp tensor cores, 1: FP32 CUDA cores) and both kR->kq GEMM forms."""
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=41, n_el=2, n_ph=1, nw=16, natom=4)
    xks = synth.random_kpoints(nk, 5)
    xqs = synth.random_kpoints(nq, 6)
    dm = pipeline.DeviceModel(m, mixed=True)
    dm.ctx.set_rotation_variant(rot)
    _force_kq_form(dm.ctx, nq, kq)
    try:
        r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=kb, sample_stride=5)
    finally:
        dm.ctx.set_rotation_variant(-1)
        _force_kq_form(dm.ctx, nq, 1)
    assert r.kq_form == kq
    ref = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=5)
    np.testing.assert_allclose(host(r.ek), ref["ek"], atol=1e-11 * np.abs(ref["ek"]).max())
    np.testing.assert_allclose(host(r.omega), ref["omega"], rtol=1e-10)
    np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-6)
    err = _block_rel_err(host(r.g2_sample), ref["g2_sample"])
    print("max per-block |g|^2 normwise rel err", err)
    assert err <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("nw,natom", [(8, 2), (12, 3), (20, 1)])
def test_gpu_pass_mixed_other_shapes(gpu_lib, nw, natom):
    """Shapes other than nw = 16, nm = 12 take the generic rotation kernel of the mixed pass (and, for
    nw > 16, the shared-memory eigensolver): same bars as the config-2 shape against the FP64 CPU port."""
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=51 + nw, n_el=2, n_ph=1, nw=nw, natom=natom)
    xks = synth.random_kpoints(6, 15)
    xqs = synth.random_kpoints(40, 16)
    dm = pipeline.DeviceModel(m, mixed=True)
    r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=4, sample_stride=3)
    ref = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=3)
    np.testing.assert_allclose(host(r.ek), ref["ek"], atol=1e-11 * np.abs(ref["ek"]).max())
    np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-6)
    assert _block_rel_err(host(r.g2_sample), ref["g2_sample"]) <= 1e-5


@pytest.mark.gpu
def test_gpu_pass_autotuned_k_batch(gpu_lib):
    """k_batch <= 0: the library times the candidates, keeps one, and the pass equals an explicit run."""
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=43, n_el=2, n_ph=1, nw=16, natom=4)
    xks = synth.random_kpoints(40, 7)
    xqs = synth.random_kpoints(96, 8)
    dm = pipeline.DeviceModel(m, mixed=True)
    r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=0)
    assert r.k_batch in (4, 8, 16, 32)
    r2 = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=0)
    assert r2.k_batch == r.k_batch  # cached in the context
    r3 = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=r.k_batch)
    np.testing.assert_array_equal(host(r.g2sum), host(r3.g2sum))


@pytest.mark.gpu
def test_gpu_pass_side_stream_equals_serial(gpu_lib):
    """The mixed pass runs its kR->kq GEMM on a side stream beside the eigensolver, except while the
    per-family profile is recorded (everything on the caller's stream): both schedules give the same
    energies, mode sums and sampled blocks (several inner batches, so the fork / join repeats)."""
    from epb200 import pipeline
    from epb200.batched import host

    m = synth.config2_model(seed=45, n_el=2, n_ph=1, nw=16, natom=4)
    dm = pipeline.DeviceModel(m, mixed=True)
    xks = synth.random_kpoints(40, 12)
    xqs = synth.random_kpoints(96, 13)
    side = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=5)
    dm.ctx.profile(True)
    try:
        serial = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=5)
        prof = dm.ctx.profile_read(reset=True)
    finally:
        dm.ctx.profile(False)
    assert any(v[1] > 0 for v in prof.values())  # the serial run was profiled
    np.testing.assert_array_equal(host(side.ek), host(serial.ek))
    np.testing.assert_allclose(host(side.g2sum), host(serial.g2sum), rtol=1e-12)
    np.testing.assert_array_equal(host(side.g2_sample), host(serial.g2_sample))


@pytest.mark.gpu
def test_gpu_pass_graph_mode(gpu_lib):
    """Graph mode: eager, captured and replayed passes on the same buffers give bit-identical results;
    new inputs copied into the same buffers are picked up by the replay."""
    import torch

    from epb200 import pipeline
    from epb200.batched import host, jl

    m = synth.config2_model(seed=44, n_el=2, n_ph=1, nw=16, natom=4)
    dm = pipeline.DeviceModel(m, mixed=True)
    xk = jl(synth.random_kpoints(24, 9))
    xq = jl(synth.random_kpoints(64, 10))
    ref = pipeline.run_eph_over_k_and_q(dm, xk, xq, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=7)
    ref = [host(ref.ek).copy(), host(ref.g2sum).copy(), host(ref.g2_sample).copy()]
    dm.ctx.set_graph_mode(True)
    try:
        out = None
        for _ in range(3):  # eager, capture, replay
            out = pipeline.run_eph_over_k_and_q(dm, xk, xq, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=7, out=out)
            for a, b in zip([host(out.ek), host(out.g2sum), host(out.g2_sample)], ref):
                np.testing.assert_array_equal(a, b)
        xk2 = synth.random_kpoints(24, 11)
        xk.copy_(torch.from_numpy(np.ascontiguousarray(xk2.T)).cuda())
        out = pipeline.run_eph_over_k_and_q(dm, xk, xq, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=7, out=out)
        dm.ctx.set_graph_mode(False)
        ref2 = pipeline.run_eph_over_k_and_q(dm, jl(xk2), xq, prec=pipeline.PREC_MIXED, k_batch=8, sample_stride=7)
        np.testing.assert_array_equal(host(out.g2sum), host(ref2.g2sum))
    finally:
        dm.ctx.set_graph_mode(False)


@pytest.fixture(scope="module")
def config2_full():
    """The config-2 model at its own sizes (nw = 16, 12 modes, Re 9^3 = 729, Rp 5^3 = 125; the 4.48 GB
    g(Re, Rp) generated on the host), uploaded once with the mixed operand planes, plus the CPU port's
    result on 3 k x 256 q of it (and the host model)."""
    from epb200 import pipeline

    m = synth.config2_model(seed=2)
    assert m.el_ham.irvec.shape[0] == 729 and m.epmat.irvec_next.shape[0] == 125 and m.nmodes == 12
    xks = synth.random_kpoints(3, 61)
    xqs = synth.random_kpoints(256, 62)
    ref = cpu_pass.eph_pass_cpu(m, xks, xqs, sample_stride=3)
    dm = pipeline.DeviceModel(m, mixed=True)
    yield dm, xks, xqs, ref, m
    dm.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed", "mixed-fp32rot", "mixed-kq-streamed"])
def test_gpu_pass_config2_grids(gpu_lib, config2_full, prec):
    """The pass at the headline configuration's own R grids (the FP16x2 kR->kq pre-scale grows with the Re
    grid, so the small-grid tests above do not cover it): FP64 at the FP64 bars, mixed at |g|^2 <= 1e-5
    per (k, q) block and band/q sums <= 1e-6, against the CPU port of the reference's batched path."""
    from epb200 import pipeline
    from epb200.batched import host

    dm, xks, xqs, ref, _ = config2_full
    p = pipeline.PREC_FP64 if prec == "fp64" else pipeline.PREC_MIXED
    dm.ctx.set_rotation_variant(1 if prec == "mixed-fp32rot" else 0)
    kq = 0 if prec == "mixed-kq-streamed" else 1
    _force_kq_form(dm.ctx, xqs.shape[1], kq)
    try:
        r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=p, k_batch=2, sample_stride=3)
    finally:
        dm.ctx.set_rotation_variant(-1)
        _force_kq_form(dm.ctx, xqs.shape[1], 1)
    if p == pipeline.PREC_MIXED:
        assert r.kq_form == kq
    np.testing.assert_allclose(host(r.ek), ref["ek"], atol=1e-11 * np.abs(ref["ek"]).max())
    np.testing.assert_allclose(host(r.omega), ref["omega"], rtol=1e-10)
    err = _block_rel_err(host(r.g2_sample), ref["g2_sample"])
    print(prec, "config-2 grids: max per-block |g|^2 normwise rel err", err)
    if prec == "fp64":
        np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-9)
        assert err <= 1e-9
    else:
        np.testing.assert_allclose(host(r.g2sum), ref["g2sum"], rtol=1e-6)
        assert err <= 1e-5


@pytest.mark.gpu
def test_gpu_pass_near_degenerate_kq(gpu_lib, config2_full):
    """A (k, q) of the config-2 bench lists whose k+q bands 7 and 8 lie 0.018 Ry apart (6.5e-4 of max
    |lambda|): formed at the FP32 level its eigenvectors turned by ~1e-4 and its |g|^2 block carried a
    1.0e-5 error; the refinement lists it and the FP64 re-solve brings it to the level of the others."""
    from epb200 import pipeline
    from epb200.batched import host

    dm, _, _, _, m = config2_full
    xk = synth.random_kpoints(2048, 1000)[:, 282:283].copy()
    xq_all = synth.random_kpoints(8192, 2000)
    xqs = np.ascontiguousarray(np.concatenate([xq_all[:, 3072:3073], xq_all[:, :7]], axis=1))
    r = pipeline.run_eph_over_k_and_q(dm, xk, xqs, prec=pipeline.PREC_MIXED, k_batch=1, sample_stride=1)
    ref = cpu_pass.eph_pass_cpu(m, xk, xqs, sample_stride=1)
    a, b = host(r.g2_sample), ref["g2_sample"]
    e0 = _block_rel_err(a[..., :1, :], b[..., :1, :])
    print("near-degenerate block |g|^2 normwise rel err", e0, "all", _block_rel_err(a, b))
    assert e0 <= 3e-6
    assert _block_rel_err(a, b) <= 1e-5
