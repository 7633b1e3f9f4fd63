"""Quasi-1-D and quasi-2-D runs (deck keys do_1D / do_2D) without a GPU: the deck
keys round-trip, fhd_create refuses what the reference's driver refuses (both
modes, bulk viscosity) and what this path does not run (mixed precision, the
particle reservoir), the batched and no-allocation steps and the restated oracle
refuse the modes, and the reference's own step in those modes (oracle/_ref)
keeps the transverse directions free of stochastic and diffusive stresses."""
import ctypes as C

import pytest
import torch

from fhdex_b200 import capi
from fhdex_b200.params import argon, mixture4, parse_inputs, stable_dt, with_walls


def _create_rc(p):
    h = C.c_void_p()
    cp = p.to_c()
    rc = capi.load().fhd_create(C.byref(h), C.byref(cp), 0)
    assert not h.value or rc == 0
    return rc


def test_mode_keys_round_trip():
    for mode in ("do_1D", "do_2D"):
        p = argon((8, 4, 4), dx=8e-6).replace(**{mode: 1})
        q = parse_inputs(p.to_inputs())
        assert (q.do_1D, q.do_2D) == (p.do_1D, p.do_2D)


@pytest.mark.parametrize("change,code", [
    (dict(do_1D=1, do_2D=1), "FHD_ERR_BAD_ARG"),
    (dict(do_1D=1, visc_type=3, zeta_ratio=1.0), "FHD_ERR_BAD_ARG"),
    (dict(do_2D=1, visc_type=-3, zeta_ratio=1.0), "FHD_ERR_BAD_ARG"),
    (dict(do_1D=2), "FHD_ERR_BAD_ARG"),
    (dict(do_2D=1, precision=1), "FHD_ERR_UNSUPPORTED"),
])
def test_create_refuses_without_gpu(change, code):
    assert _create_rc(mixture4((6, 5, 4), dx=8e-6).replace(**change)) == getattr(capi, code)


@pytest.mark.parametrize("n,mode,ok", [((8, 6, 1), "do_2D", True), ((8, 1, 1), "do_1D", True),
                                       ((8, 6, 1), "do_1D", True), ((8, 6, 1), None, False),
                                       ((8, 1, 6), "do_2D", False), ((1, 6, 6), "do_1D", False)])
def test_one_cell_directions_only_in_their_modes(n, mode, ok):
    """A one-cell direction is z of a quasi-2-D run or y / z of a quasi-1-D run, as the
    reference's driver has it (main_driver.cpp:125-140); elsewhere it is refused."""
    p = argon(n, dx=8e-6)
    if mode:
        p = p.replace(**{mode: 1})
    rc = _create_rc(p)
    if ok:
        assert rc not in (capi.FHD_ERR_BAD_ARG, capi.FHD_ERR_UNSUPPORTED)
    else:
        assert rc == capi.FHD_ERR_BAD_ARG


def test_create_refuses_the_particle_reservoir_in_1d():
    p = with_walls(argon((8, 4, 4), dx=8e-6), x=dict(vel=2, therm=2, mass=4, t=(300.0, 300.0),
                                                   Yk=((0.5, 0.5), (0.5, 0.5)))).replace(do_1D=1)
    assert _create_rc(p) == capi.FHD_ERR_UNSUPPORTED


def test_noalloc_and_oracle_refuse_the_modes(oracle):
    p = argon((6, 4, 4), dx=8e-6).replace(do_1D=1)
    cp = p.to_c()
    nf = capi.FhdFab()
    f3 = (capi.FhdFab * 3)()
    st = C.c_int()
    assert capi.load().fhd_rk3_step_stag_noalloc(C.byref(cp), nf, f3, nf, f3, 1e-13, 0, None, C.byref(st)) == \
        capi.FHD_ERR_UNSUPPORTED
    with pytest.raises(Exception):
        oracle.set_params(p)


@pytest.fixture(scope="module")
def ref():
    from oracle import ref as R
    if not R.available():
        pytest.skip("oracle/_ref was not built")
    return R


@pytest.mark.parametrize("mode", ["do_1D", "do_2D"])
def test_reference_step_has_no_transverse_stresses(ref, mode):
    """The reference's own step with the mode set: the transverse faces (y and z in
    1-D, z in 2-D) carry no heat flux, viscous heating or Dufour flux (their
    species fluxes are advection only), and mass is conserved."""
    p = mixture4((8, 5, 4), dx=8e-6).replace(**{mode: 1})
    st = ref.state_from_reference(p, seed=5)
    m0 = st.cu.valid()[0].sum().item()
    for s in range(2):
        ref.rk3_step(st, ref.step_noise(p, 60 + s), stable_dt(p), s)
    assert abs(st.cu.valid()[0].sum().item() - m0) <= 1e-13 * m0
    nv = p.nvars
    trans = [1, 2] if mode == "do_1D" else [2]
    for d in trans:
        f = st.faceflux[d].arr
        for c in (nv, nv + 1, nv + 2, nv + 3):
            assert not f[c].any(), (d, c)
    assert st.faceflux[0].arr[nv].abs().max() > 0
    for m in st.state_mfs():
        assert torch.isfinite(m.arr).all()


@pytest.mark.parametrize("all_correl", [0, 1])
def test_1d_correlation_files_equal_the_references(ref, tmp_path, monkeypatch, all_correl):
    """The reference's evaluateStatsStag1D over three samples fills spatialCrossMF;
    fhd_write_spatial_cross (host memory) writes the same WriteSpatialCross1D files
    byte for byte (one file, or five with all_correl)."""
    from fhdex_b200.stats import StatsState
    p = mixture4((12, 3, 4), dx=8e-6).replace(do_1D=1, cross_cell=5, all_correl=all_correl)
    stats = StatsState(p, cross=True)
    for s in range(1, 4):
        st = ref.state_from_reference(p, seed=20 + s)
        ref.eval_stats(st, stats, s, 15 | capi.STATS_CROSS)
    assert stats.spatialCross.shape[0] == (5 if all_correl else 1) * (37 + 4 + 3)
    assert stats.spatialCross[0].abs().max() > 0
    mine, theirs = tmp_path / "mine", tmp_path / "ref"
    mine.mkdir()
    theirs.mkdir()
    stats.write_spatial_cross(9, str(mine) + "/")
    monkeypatch.chdir(theirs)
    ref.write_spatial_cross_1d(p, stats.spatialCross, 9)
    names = sorted(f.name for f in theirs.iterdir())
    assert names == sorted(f.name for f in mine.iterdir()) and len(names) == (5 if all_correl else 1)
    for n in names:
        assert (mine / n).read_bytes() == (theirs / n).read_bytes(), n


def test_1d_checkpoint_keeps_spatial_cross_mf(tmp_path):
    """A quasi-1-D run's checkpoint: spatialCrossMF as a Level_0 MultiFab (bit for bit
    back), the Header's spatialCrossVec left at zero (Checkpoint.cpp:112-118, 251-256)."""
    import os
    from fhdex_b200.checkpoint import read_checkpoint, write_checkpoint
    from fhdex_b200.state import StagState
    from fhdex_b200.stats import StatsState
    p = argon((6, 3, 2), dx=8e-6).replace(do_1D=1, all_correl=1)
    st = StagState(p)
    stats = StatsState(p, cross=True)
    g = torch.Generator().manual_seed(3)
    stats.spatialCross.copy_(torch.randn(stats.spatialCross.shape, generator=g, dtype=torch.float64))
    path = write_checkpoint(p, str(tmp_path / "chk"), 2, 0.5, st, stats, stats_count=2)
    assert os.path.exists(os.path.join(path, "Level_0", "spatialCrossMF_H"))
    lines = open(os.path.join(path, "Header")).read().split("\n")
    vals = [v for v in lines[lines.index(")") + 1:] if v]
    assert vals == ["0"] * (6 * (37 + 2 + 3))
    back = StatsState(p, cross=True)
    read_checkpoint(p, str(tmp_path / "chk"), 2, StagState(p), back)
    assert torch.equal(back.spatialCross, stats.spatialCross)
