"""Learned window pre-filter: the surrogate's kernels against the CPU oracle, the tridiagonal window
test against LAPACK + searchsorted, and the kept (k, q) pair set with and without the surrogate.

Tolerances (FP32 network kernels vs the FP64 oracle on the same parameters and features):
  forward outputs: max |diff| <= 2e-5 (outputs are O(1));
  loss: relative 1e-5; gradient: normwise relative 1e-4, every entry within 1e-4 of the largest;
  one Adam step: parameters within 1e-6 + 1e-4 |update|.
Window ranges, kept pairs: bit-exact (integer).
Band energies: FP64 path within 1e-9 Ry of LAPACK (the path's contract is 1e-8 Ry).
"""
import numpy as np
import pytest

from oracle import epb_oracle as O
from oracle import mlp_oracle as M
from epb200 import synth
from epb200.wannier import WannierObject

# ---------------------------------------------------------------------------------------------
# CPU: the oracle itself


def _rand_params(shapes, nparam, rng, scale=0.3):
    p = np.zeros(nparam)
    for fi, fo, w, b in shapes:
        p[w:w + fi * fo] = rng.uniform(-1, 1, fi * fo) * np.sqrt(6.0 / (fi + fo))
        p[b:b + fo] = rng.normal(0, scale, fo)
    return p


def test_oracle_gradient_finite_difference():
    rng = np.random.default_rng(0)
    shapes, nparam = M.layer_shapes(8, 12, 2, 4)
    p = _rand_params(shapes, nparam, rng)
    X = rng.normal(size=(6, 8))
    Y = rng.normal(size=(6, 4))
    loss, g = M.loss_grad(p, shapes, X, Y)
    idx = rng.choice(nparam, 40, replace=False)
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_grad(pp, shapes, X, Y)[0] - M.loss_grad(pm, shapes, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(fd), (i, fd, g[i])
    # padding entries carry no gradient
    used = np.zeros(nparam, bool)
    for fi, fo, w, b in shapes:
        used[w:w + fi * fo] = True
        used[b:b + fo] = True
    assert np.all(g[~used] == 0)


def test_feature_vectors_half_space():
    from epb200.learned import feature_vectors

    f = feature_vectors(128).T
    assert f.shape == (128, 3)
    s = {tuple(v) for v in f}
    assert len(s) == 128
    assert all(tuple(-v) not in s for v in f)
    n2 = (f * f).sum(1)
    assert np.all(np.diff(n2) >= 0)
    assert n2[0] == 1


def test_oracle_window_ranges_match_counts():
    rng = np.random.default_rng(1)
    E = np.sort(rng.normal(size=(9, 200)), axis=0)
    bmin, bmax = M.window_ranges(E, -0.3, 0.4)
    for k in range(200):
        lo = int((E[:, k] < -0.3).sum())
        hi = int((E[:, k] <= 0.4).sum())
        if hi >= lo + 1:
            assert (bmin[k], bmax[k]) == (lo + 1, hi)
        else:
            assert (bmin[k], bmax[k]) == (0, 0)


# ---------------------------------------------------------------------------------------------
# GPU


@pytest.fixture(scope="module")
def L(gpu_lib):
    from epb200 import learned

    return learned


def _ham(nw, n_el, seed, decay=1.5):
    rng = np.random.default_rng(seed)
    irvec = synth.irvec_box(n_el)
    return WannierObject(irvec, synth.hermitian_op_r(rng, nw, irvec, decay))


@pytest.mark.gpu
def test_mlp_features(L):
    s = L.Surrogate(nf=64, hidden=32, nhidden=2, nout=8, seed=3)
    x = np.random.default_rng(2).random((3, 300)) * 4 - 2
    F = s.features(x).cpu().numpy()
    ref = M.features(s.fvec.T.reshape(-1), x)
    assert np.max(np.abs(F - ref)) <= 2e-6


@pytest.mark.gpu
def test_mlp_forward_matches_oracle(L):
    s = L.Surrogate(nf=64, hidden=64, nhidden=3, nout=16, seed=5)
    s.set_inference(0)  # the FP32 kernels of training
    shapes, nparam = M.layer_shapes(s.nin, 64, 3, 16)
    assert nparam == s.nparam
    rng = np.random.default_rng(4)
    p = _rand_params(shapes, nparam, rng).astype(np.float32)
    s.set_params(p)
    mu, sc = rng.normal(size=16), rng.uniform(0.5, 2.0, 16)
    s.set_scaling(mu, sc)
    x = rng.random((3, 257))
    E = s.predict(x).cpu().numpy().T  # (nout, n)
    F = s.features(x).cpu().numpy().astype(np.float64)
    out, _ = M.forward(p.astype(np.float64), shapes, F)
    ref = (out * sc.astype(np.float32).astype(np.float64)[None, :] + mu.astype(np.float32)[None, :]).T
    assert np.max(np.abs(E - ref)) <= 2e-5 * max(1.0, np.max(np.abs(ref)))


@pytest.mark.gpu
@pytest.mark.parametrize("nf,hidden,nhidden,nout", [(64, 64, 3, 16), (128, 256, 3, 32), (32, 128, 2, 48)])
def test_mlp_tensor_core_inference(L, nf, hidden, nhidden, nout):
    """tcgen05 BF16 inference vs a BF16-rounding emulation of the same network (FP64 accumulation)."""
    s = L.Surrogate(nf=nf, hidden=hidden, nhidden=nhidden, nout=nout, seed=21)
    assert s.inference_path() == 1
    shapes, nparam = M.layer_shapes(s.nin, hidden, nhidden, nout)
    rng = np.random.default_rng(22)
    p = _rand_params(shapes, nparam, rng).astype(np.float32)
    s.set_params(p)
    s.set_scaling(np.zeros(nout), np.ones(nout))
    x = rng.random((3, 1000)) * 2 - 0.5  # 8 tiles, the last one ragged
    E = s.predict(x).cpu().numpy()  # torch shape (n, nout) = Julia (nout, n)
    F = s.features(x).cpu().numpy().astype(np.float64)
    ref = M.forward_bf16(p.astype(np.float64), shapes, F)
    err = np.abs(E - ref)
    scale = np.abs(ref).max()
    assert np.linalg.norm(E - ref) <= 2e-3 * np.linalg.norm(ref), np.linalg.norm(E - ref) / np.linalg.norm(ref)
    assert err.max() <= 2e-2 * scale, err.max() / scale
    # and it is close to the FP32 path (BF16 rounding only)
    s.set_inference(0)
    E32 = s.predict(x).cpu().numpy()
    assert np.linalg.norm(E - E32) <= 5e-2 * np.linalg.norm(E32)


@pytest.mark.gpu
def test_mlp_gradient_matches_oracle(L):
    s = L.Surrogate(nf=64, hidden=64, nhidden=3, nout=16, seed=6)
    shapes, nparam = M.layer_shapes(s.nin, 64, 3, 16)
    rng = np.random.default_rng(7)
    p = _rand_params(shapes, nparam, rng).astype(np.float32)
    s.set_params(p)
    mu, sc = rng.normal(size=16), rng.uniform(0.5, 2.0, 16)
    s.set_scaling(mu, sc)
    n = 520
    x = rng.random((3, n))
    E = rng.normal(size=(16, n)) * sc[:, None] + mu[:, None]
    loss, g = s.loss_grad(x, E)
    g = g.cpu().numpy().astype(np.float64)
    F = s.features(x).cpu().numpy().astype(np.float64)
    Y = M.normalised_targets(E, mu.astype(np.float32), sc.astype(np.float32))
    lref, gref = M.loss_grad(p.astype(np.float64), shapes, F, Y)
    assert abs(loss - lref) <= 1e-5 * lref
    err = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert err <= 1e-4, err
    assert np.max(np.abs(g - gref)) <= 1e-4 * np.max(np.abs(gref))


@pytest.mark.gpu
def test_mlp_adam_step_matches_oracle(L):
    s = L.Surrogate(nf=32, hidden=32, nhidden=2, nout=8, seed=8)
    shapes, nparam = M.layer_shapes(s.nin, 32, 2, 8)
    p0 = s.get_params().cpu().numpy().astype(np.float64)
    rng = np.random.default_rng(9)
    n = 64
    x = rng.random((3, n))
    E = rng.normal(size=(8, n)) * 3 + 1
    s.train(x, E, epochs=1, batch=n, lr=1e-3, lr_final=1e-3, use_graph=False)
    p1 = s.get_params().cpu().numpy().astype(np.float64)
    mu, sc = s.get_scaling()
    # the library's normalisation is the per-band mean / population std of E
    assert np.allclose(mu, E.mean(axis=1), rtol=1e-6, atol=1e-6)
    assert np.allclose(sc, E.std(axis=1), rtol=1e-5)
    F = s.features(x).cpu().numpy().astype(np.float64)
    Y = M.normalised_targets(E, mu, sc)
    _, g = M.loss_grad(p0, shapes, F, Y)
    pref, _, _ = M.adam_step(p0, np.zeros(nparam), np.zeros(nparam), g, 1, 1e-3)
    upd = np.abs(pref - p0)
    assert np.all(np.abs(p1 - pref) <= 1e-6 + 1e-3 * upd), np.max(np.abs(p1 - pref))


@pytest.mark.gpu
def test_mlp_training_graph_equals_eager(L):
    rng = np.random.default_rng(10)
    x = rng.random((3, 1024))
    E = rng.normal(size=(8, 1024))
    a = L.Surrogate(nf=32, hidden=32, nhidden=2, nout=8, seed=12)
    b = L.Surrogate(nf=32, hidden=32, nhidden=2, nout=8, seed=12)
    la = a.train(x, E, epochs=3, batch=256, use_graph=True)
    lb = b.train(x, E, epochs=3, batch=256, use_graph=False)
    # the reported loss is summed with atomics across blocks (order-dependent last bits); the
    # parameters come from fixed-order reductions and must agree bit for bit
    assert np.allclose(la, lb, rtol=1e-12, atol=0)
    assert np.array_equal(a.get_params().cpu().numpy(), b.get_params().cpu().numpy())


@pytest.mark.gpu
@pytest.mark.parametrize("nw,n_el", [(8, 2), (13, 2), (32, 3)])
def test_bands_eigvals_vs_lapack(L, nw, n_el):
    ham = _ham(nw, n_el, 20 + nw)
    bm = L.BandModel(ham)
    x = np.random.default_rng(nw).random((3, 97))
    E = bm.eigvals(x, prec=L.PREC_FP64).cpu().numpy().T
    ref = M.band_energies(ham.op_r, nw, ham.irvec, x)
    assert np.max(np.abs(E - ref)) <= 1e-9
    Em = bm.eigvals(x, prec=L.PREC_MIXED).cpu().numpy().T
    dev = np.max(np.abs(Em - ref))
    assert dev <= L.DEFAULT_GUARD / 10, dev


@pytest.mark.gpu
@pytest.mark.parametrize("nw,band", [(8, 1), (13, 7), (32, 16), (32, 32)])
def test_bands_band_energy(L, nw, band):
    ham = _ham(nw, 2, 90 + nw)
    bm = L.BandModel(ham)
    x = np.random.default_rng(band).random((3, 131))
    e = bm.band_energy(x, band).cpu().numpy()
    ref = M.band_energies(ham.op_r, nw, ham.irvec, x)[band - 1]
    assert np.max(np.abs(e - ref)) <= 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("nw,n_el", [(8, 2), (13, 2), (32, 3)])
def test_bands_window_vs_oracle(L, nw, n_el):
    ham = _ham(nw, n_el, 30 + nw)
    bm = L.BandModel(ham)
    x = np.random.default_rng(40 + nw).random((3, 2000))
    ref_E = M.band_energies(ham.op_r, nw, ham.irvec, x)
    med = float(np.median(ref_E[nw // 2]))
    wmin, wmax = med - 0.3, med + 0.2
    rb0, rb1 = M.window_ranges(ref_E, wmin, wmax)
    for prec in (L.PREC_FP64, L.PREC_MIXED):
        b0, b1, keep, st = bm.window(x, wmin, wmax, prec=prec)
        assert np.array_equal(b0.cpu().numpy(), rb0)
        assert np.array_equal(b1.cpu().numpy(), rb1)
        assert np.array_equal(keep.cpu().numpy(), np.nonzero(rb0 > 0)[0])
        assert st["kept"] == int((rb0 > 0).sum())


@pytest.mark.gpu
def test_bands_window_edge_exactness(L):
    """Windows placed exactly on computed eigenvalues: ranges stay LAPACK + searchsorted's
    (inclusive both ends) within the FP64 re-evaluation."""
    nw = 8
    ham = _ham(nw, 2, 77)
    bm = L.BandModel(ham)
    x = np.random.default_rng(78).random((3, 64))
    E = bm.eigvals(x, prec=L.PREC_FP64).cpu().numpy().T
    wmin, wmax = float(E[2, 5]) + 0.05, float(E[5, 7]) - 0.05
    ref = M.band_energies(ham.op_r, nw, ham.irvec, x)
    rb0, rb1 = M.window_ranges(ref, wmin, wmax)
    for prec in (L.PREC_FP64, L.PREC_MIXED):
        b0, b1, _, _ = bm.window(x, wmin, wmax, prec=prec)
        assert np.array_equal(b0.cpu().numpy(), rb0) and np.array_equal(b1.cpu().numpy(), rb1)


@pytest.mark.gpu
def test_pair_window_vs_oracle(L):
    nw = 8
    ham = _ham(nw, 2, 50)
    bm = L.BandModel(ham)
    rng = np.random.default_rng(51)
    xk, xq = rng.random((3, 24)), rng.random((3, 70))
    ref_E = M.band_energies(ham.op_r, nw, ham.irvec, rng.random((3, 500)))
    med = float(np.median(ref_E[4]))
    wmin, wmax = med - 0.2, med + 0.2
    kp, k0, k1, _ = M.pair_window(ham.op_r, nw, ham.irvec, xk, xq, wmin, wmax)
    for prec in (L.PREC_FP64, L.PREC_MIXED):
        p, b0, b1, st = L.pair_window(bm, xk, xq, wmin, wmax, prec=prec)
        assert np.array_equal(p.cpu().numpy(), kp)
        assert np.array_equal(b0.cpu().numpy(), k0) and np.array_equal(b1.cpu().numpy(), k1)
        assert st["tested"] == 24 * 70 and st["kept"] == len(kp)
    # a capacity below the kept count is reported, not overrun
    with pytest.raises(Exception):
        L.pair_window(bm, xk, xq, wmin, wmax, capacity=max(0, len(kp) - 1))


@pytest.mark.gpu
def test_learned_filter_identical_set_and_gain(L):
    """Train on plain-path energies, calibrate on held-out points, then the pair window with the
    surrogate must return exactly the pairs of the plain window (and of the FP64 window) while
    sending fewer points to the plain evaluation."""
    import torch

    # A smooth band structure (H(R) decaying as exp(-|R|/0.5)): the network learns it to a few
    # 10 meV. (For the rough exp(-|R|/1.5) models the held-out error exceeds 1 Ry and the surrogate
    # culls almost nothing; the kept set is still exact.)
    nw = 16
    ham = _ham(nw, 3, 60, decay=0.5)
    bm = L.BandModel(ham)
    rng = np.random.default_rng(61)
    xt, xh = rng.random((3, 1 << 14)), rng.random((3, 1 << 13))
    Et = bm.eigvals(xt)
    Eh = bm.eigvals(xh)
    s = L.Surrogate(nf=64, hidden=128, nhidden=3, nout=nw, seed=62)
    loss = s.train(xt, Et, epochs=150, batch=1024, lr=3e-3, lr_final=3e-5)
    assert loss[-1] < 0.05 * loss[0]
    margin = s.calibrate(xh, Eh)
    assert np.all(margin > 0)
    ef = float(torch.median(Eh[:, nw // 2 - 1]).item())
    wmin, wmax = ef - 0.05, ef + 0.05
    xk, xq = rng.random((3, 64)), rng.random((3, 2048))
    plain = L.pair_window(bm, xk, xq, wmin, wmax, prec=L.PREC_MIXED)
    fp64 = L.pair_window(bm, xk, xq, wmin, wmax, prec=L.PREC_FP64)
    learned = L.pair_window(bm, xk, xq, wmin, wmax, mlp=s, prec=L.PREC_MIXED)
    for a in (fp64, learned):
        assert torch.equal(a[0], plain[0]) and torch.equal(a[1], plain[1]) and torch.equal(a[2], plain[2])
    st = learned[3]
    assert st["culled"] + st["evaluated"] == st["tested"] == 64 * 2048 == st["screened"]
    assert st["audited"] > 0 and st["violations"] == 0 and st["fallback_chunks"] == 0, st
    # the gain: with margins of 1.5 x the maximum held-out error the plain evaluation still runs on
    # well under two thirds of the pairs
    assert st["evaluated"] <= 0.6 * plain[3]["evaluated"], st
    print(f"\nsurrogate: margin max {margin.max():.4f} Ry, culled {st['culled'] / st['tested']:.3f} of pairs, "
          f"kept {st['kept']}")


@pytest.mark.gpu
def test_learned_filter_audit_repairs_bad_margins(L):
    """Margins calibrated against the network's own predictions (zero held-out error) are far too
    small: the audit of culled pairs finds pairs inside the window, the affected chunks fall back to
    the plain evaluation, and the kept set is still the plain filter's."""
    import torch

    nw = 8
    ham = _ham(nw, 2, 70, decay=0.7)
    bm = L.BandModel(ham)
    rng = np.random.default_rng(71)
    xt = rng.random((3, 4096))
    s = L.Surrogate(nf=32, hidden=64, nhidden=2, nout=nw, seed=72)
    s.train(xt, bm.eigvals(xt), epochs=20, batch=512)
    xh = rng.random((3, 512))
    s.calibrate(xh, s.predict(xh), safety=1.0)  # zero margins
    ef = float(torch.median(bm.eigvals(xh)[:, 3]).item())
    xk, xq = rng.random((3, 40)), rng.random((3, 512))
    plain = L.pair_window(bm, xk, xq, ef - 0.1, ef + 0.1, prec=L.PREC_MIXED)
    learned = L.pair_window(bm, xk, xq, ef - 0.1, ef + 0.1, mlp=s, prec=L.PREC_MIXED)
    st = learned[3]
    assert st["violations"] > 0 and st["fallback_chunks"] > 0, st
    for a, b in zip(learned[:3], plain[:3]):
        assert torch.equal(a, b)


@pytest.mark.gpu
def test_learned_filter_screen_stops_when_it_culls_nothing(L):
    """A surrogate of a rough band structure (held-out errors far wider than the window) culls nothing;
    after 2^20 screened pairs the screen stops and the remaining chunks go straight to the plain
    evaluation (stats: screened < tested), with the kept set still the plain filter's."""
    import torch

    nw = 16
    ham = _ham(nw, 3, 80, decay=1.5)
    bm = L.BandModel(ham)
    rng = np.random.default_rng(81)
    xt, xh = rng.random((3, 4096)), rng.random((3, 2048))
    s = L.Surrogate(nf=32, hidden=64, nhidden=2, nout=nw, seed=82)
    s.train(xt, bm.eigvals(xt), epochs=10, batch=512)
    Eh = bm.eigvals(xh)
    s.calibrate(xh, Eh)
    ef = float(torch.median(Eh[:, nw // 2 - 1]).item())
    xk, xq = rng.random((3, 96)), rng.random((3, 16384))
    plain = L.pair_window(bm, xk, xq, ef - 0.02, ef + 0.02, prec=L.PREC_MIXED)
    learned = L.pair_window(bm, xk, xq, ef - 0.02, ef + 0.02, mlp=s, prec=L.PREC_MIXED)
    st = learned[3]
    assert st["tested"] == 96 * 16384 and st["screened"] >= (1 << 20) and st["screened"] < st["tested"], st
    assert st["culled"] * 5 < st["screened"], st
    assert st["culled"] + st["evaluated"] == st["tested"], st
    for a, b in zip(learned[:3], plain[:3]):
        assert torch.equal(a, b)
