"""The autotuner's table (epb_tune_table_*): host logic only, no GPU. Set / overwrite / get, the text
round trip, comment lines, rejection of malformed text (table unchanged) and of bad keys; on a GPU, a
pass whose choices come from an imported table equals the autotuned pass bit for bit."""
import numpy as np
import pytest

KB, ROT, KQ = "pass_kb/16/12/8192/1", "pass_rot/16/12/8192/1", "pass_kq/16/12/8192/1"


def test_table_set_get_overwrite(cpu_lib):
    from epb200._lib import TuneTable

    t = TuneTable()
    assert len(t) == 0 and t.get(KB) is None
    t.set(KB, 16)
    t.set(ROT, 0)
    t.set(KB, 32)  # a later measurement replaces the earlier one
    assert len(t) == 2 and t.get(KB) == 32 and t.get(ROT) == 0 and t.get(KQ) is None


def test_table_text_round_trip(cpu_lib):
    from epb200._lib import TuneTable

    t = TuneTable()
    for k, v in ((KB, 8), (ROT, 1), (KQ, 0), ("pass_kb/8/6/64/0", -5)):
        t.set(k, v)
    txt = t.text()
    assert txt.splitlines() == [f"{KB} 8", f"{ROT} 1", f"{KQ} 0", "pass_kb/8/6/64/0 -5"]
    u = TuneTable("# measured on one B200\n\n" + txt + "   \n")
    assert len(u) == 4 and all(u.get(k) == t.get(k) for k in (KB, ROT, KQ, "pass_kb/8/6/64/0"))
    u.parse(f"{KB} 4\n")  # parse adds / overwrites
    assert u.get(KB) == 4 and len(u) == 4


@pytest.mark.parametrize("bad", ["pass_kb 1 2\n", "pass_kb\n", "pass_kb x\n", f"{KB} 4\nnot-a-number?\n"])
def test_table_rejects_malformed_text_unchanged(cpu_lib, bad):
    from epb200._lib import EPB_ERR_ARG, EpbError, TuneTable

    t = TuneTable(f"{ROT} 1\n")
    with pytest.raises(EpbError) as e:
        t.parse(bad)
    assert e.value.status == EPB_ERR_ARG
    assert len(t) == 1 and t.get(ROT) == 1 and t.get(KB) is None


@pytest.mark.parametrize("key", ["", "has space", "x" * 121, "tab\tkey"])
def test_table_rejects_bad_keys(cpu_lib, key):
    from epb200._lib import EpbError, TuneTable

    with pytest.raises(EpbError):
        TuneTable().set(key, 1)


@pytest.mark.gpu
def test_imported_table_equals_autotuned_pass(gpu_lib):
    """The pass autotunes (k batch, rotation kernel, kR->kq form) on a fresh context; a second context that
    imports the exported table runs the same configuration without timing and gives bit-identical
    results; a table forcing the other rotation kernel is honoured and stays within the mixed bar."""
    from epb200 import _lib, pipeline, synth
    from epb200.batched import host

    m = synth.config2_model(seed=47, n_el=2, n_ph=1, nw=16, natom=4)
    xks = synth.random_kpoints(24, 17)
    xqs = synth.random_kpoints(96, 18)
    dm = pipeline.DeviceModel(m, mixed=True, ctx=_lib.Context(0))  # a fresh table: every choice is timed
    r = pipeline.run_eph_over_k_and_q(dm, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=0, sample_stride=5)
    assert r.k_batch in (4, 8, 16, 32) and r.rot_variant in (0, 1) and r.kq_form in (0, 1)
    t = _lib.TuneTable()
    t.export_from(dm.ctx)
    key = f"pass_rot/16/12/{xqs.shape[1]}/{pipeline.PREC_MIXED}"
    assert t.get(key) == r.rot_variant
    ctx2 = _lib.Context(0)
    t.import_into(ctx2)
    dm2 = pipeline.DeviceModel(m, mixed=True, ctx=ctx2)
    r2 = pipeline.run_eph_over_k_and_q(dm2, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=0, sample_stride=5)
    assert (r2.k_batch, r2.rot_variant, r2.kq_form) == (r.k_batch, r.rot_variant, r.kq_form)
    np.testing.assert_array_equal(host(r2.g2_sample), host(r.g2_sample))
    np.testing.assert_allclose(host(r2.g2sum), host(r.g2sum), rtol=1e-12)
    # the other rotation kernel through the table
    t.set(key, 1 - r.rot_variant)
    t.import_into(ctx2)
    r3 = pipeline.run_eph_over_k_and_q(dm2, xks, xqs, prec=pipeline.PREC_MIXED, k_batch=0, sample_stride=5)
    assert r3.rot_variant == 1 - r.rot_variant
    np.testing.assert_allclose(host(r3.g2sum), host(r.g2sum), rtol=1e-6)
    dm2.close()
    dm.close()
