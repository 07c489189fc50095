"""TiledDeviceOutput (src/calculator/tiled_device_output.jl) and ind_range_for_k_range
(src/band_states.jl:416-428): host logic against the oracle on CPU; on the GPU a mock device-resident
calculator scattering through eph_window_scatter! gives bit-identical outputs in block and full residency
(the property the reference's Boltzmann tests check with several tiles at nonzero offsets,
test/boltzmann/test_gpu_boltzmann_calculator.jl:178-190)."""
import numpy as np
import pytest

from oracle import epb_oracle as O


def _states(rng, nk, maxper=3):
    per = rng.integers(0, maxper + 1, nk)
    return np.repeat(np.arange(1, nk + 1), per).astype(np.int64)


@pytest.fixture(scope="module")
def T(cpu_lib):
    from epb200 import tiled

    return tiled


def test_ind_range_and_capacity_match_oracle(T):
    rng = np.random.default_rng(0)
    for trial in range(20):
        nk = int(rng.integers(1, 30))
        iks = _states(rng, nk)
        for _ in range(10):
            a = int(rng.integers(1, nk + 1))
            b = int(rng.integers(a - 1, nk + 1))
            assert T.ind_range_for_k_range(iks, nk, a, b) == O.ind_range_for_k_range(iks, a, b)
        for nb in (1, 2, 5, 64):
            assert T.tile_capacity(iks, nk, nb) == O.tile_capacity(iks, nk, nb)


def test_ind_range_non_contiguous_raises(T):
    from epb200._lib import EpbError

    iks = np.array([1, 2, 1, 3], dtype=np.int64)  # k = 1 states at 1 and 3, k = 2 in between
    with pytest.raises(EpbError, match="non-contiguous"):
        T.ind_range_for_k_range(iks, 3, 1, 1)
    with pytest.raises(ValueError):
        O.ind_range_for_k_range(iks, 1, 1)
    assert T.ind_range_for_k_range(iks, 3, 3, 3) == range(4, 5)
    assert T.ind_range_for_k_range(np.zeros(0, np.int64), 5, 1, 5) == range(1, 1)
    with pytest.raises(EpbError):  # k index outside 1..nk
        T.ind_range_for_k_range(np.array([1, 9], dtype=np.int64), 3, 1, 3)


def _mock_run(B, T, force_block, rng_seed=3, nk=23, nb_max=4, nm=3, n_f=17, nbkq=4, nbk=3, nkq=6, nqb=5):
    """An outer-k loop over k batches with a device-resident (nm, n_i, n_f) g2 output."""
    rng = np.random.default_rng(rng_seed)
    iks = _states(rng, nk)
    n_i = iks.size
    t = T.TiledDeviceOutput((nm, n_i, n_f), 2, iks, nk, narr=2, force_block=force_block, n_batch_max=nb_max)
    full_g = np.zeros((nm, n_i, n_f), order="F")
    full_o = np.zeros((nm, n_i, n_f), order="F")
    ref_g = np.zeros(nm * n_i * n_f)
    ref_o = np.zeros(nm * n_i * n_f)
    for ks in range(1, nk + 1, nb_max):
        ke = min(ks + nb_max - 1, nk)
        t.tile_begin(ks, ke)
        dg, do = t.device_array(1), t.device_array(2)
        i0, stride = t.tile_offset(), t.tile_stride()
        for k in range(ks, ke + 1):
            states = np.nonzero(iks == k)[0] + 1
            imap_i = np.zeros(nbk, dtype=np.int64)
            imap_i[: min(nbk, states.size)] = states[:nbk]
            g2 = rng.random((nbkq, nbk, nm, nqb))
            om = rng.random((nm, nqb)) + 0.01
            imap_f = np.zeros((nbkq, nkq), dtype=np.int64)
            mask = rng.random((nbkq, nkq)) < 0.6
            imap_f[mask] = rng.permutation(n_f)[: mask.sum()] + 1 if mask.sum() <= n_f else 0
            ikqs = (rng.permutation(nkq)[:nqb] + 1).astype(np.int64)
            B.eph_window_scatter(dg.view(-1), do.view(-1), B.jl(g2), B.jl(imap_i), B.jl(imap_f), B.jl(ikqs), B.jl(om),
                                 stride, i0)
            O.eph_window_scatter(ref_g, ref_o, g2, imap_i, imap_f, ikqs, om, n_i, 0)
        if t.is_block():
            r = O.ind_range_for_k_range(iks, ks, ke)
            assert (t.tile_offset(), t.tile_length()) == (r.start - 1, len(r))
            full_g[:, r.start - 1:r.stop - 1, :] = t.tile_download(1)
            full_o[:, r.start - 1:r.stop - 1, :] = t.tile_download(2)
    if not t.is_block():
        full_g, full_o = t.tile_download(1), t.tile_download(2)
    info = (t.is_block(), t.tile_stride())
    t.tile_free()
    assert not t.is_allocated()
    t.close()
    return full_g, full_o, ref_g.reshape(nm, n_i, n_f, order="F"), ref_o.reshape(nm, n_i, n_f, order="F"), info, iks


@pytest.mark.gpu
def test_tiled_block_equals_full(gpu_lib):
    from epb200 import batched as B
    from epb200 import tiled as T

    bg, bo, rg, ro, binfo, iks = _mock_run(B, T, True)
    fg, fo, rg2, ro2, finfo, _ = _mock_run(B, T, False)
    assert binfo[0] and not finfo[0]
    assert binfo[1] == O.tile_capacity(iks, 23, 4) < iks.size and finfo[1] == iks.size
    np.testing.assert_array_equal(rg, rg2)
    np.testing.assert_array_equal(bg, fg)
    np.testing.assert_array_equal(bo, fo)
    np.testing.assert_array_equal(fg, rg)
    np.testing.assert_array_equal(fo, ro)
    # automatic residency: a small output stays resident
    _, _, _, _, ainfo, _ = _mock_run(B, T, None)
    assert not ainfo[0]
    assert T.residency_use_block(10 ** 15) and not T.residency_use_block(10 ** 6)


@pytest.mark.gpu
def test_tiled_axis_positions(gpu_lib):
    """Any tiled-axis position: the tile region is zeroed at each begin and downloaded compactly."""
    import torch

    from epb200 import tiled as T

    rng = np.random.default_rng(5)
    nk = 9
    iks = _states(rng, nk, 2)
    n = iks.size
    for dims, ax in [((n, 4, 3), 1), ((2, 5, n), 3), ((3, n, 2), 2)]:
        t = T.TiledDeviceOutput(dims, ax, iks, nk, force_block=True, n_batch_max=2)
        out = np.zeros(dims, order="F")
        for ks in range(1, nk + 1, 2):
            t.tile_begin(ks, min(ks + 1, nk))
            d = t.device_array(1)
            i0, ni = t.tile_offset(), t.tile_length()
            sel = [slice(None)] * 3
            sel[ax - 1] = slice(0, ni)
            dv = d.permute(*reversed(range(3)))  # Julia index order
            assert float(dv[tuple(sel)].abs().sum()) == 0.0  # the active region is zeroed
            val = np.asfortranarray(rng.random(tuple(ni if a == ax - 1 else dims[a] for a in range(3))))
            dv[tuple(sel)] = torch.from_numpy(val).to("cuda")
            sel2 = list(sel)
            sel2[ax - 1] = slice(i0, i0 + ni)
            out[tuple(sel2)] = val
            got = t.tile_download(1)
            np.testing.assert_array_equal(got, val)
        t.close()
