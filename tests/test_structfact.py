"""The structure-factor oracle (oracle/structfact.py) against known answers:
its unpacked half spectrum is the full complex FFT, Parseval's identity holds
for a single sample (sum over k of S_aa = sum over x of a^2), the pair and
default-pair conventions follow StructFact.cpp:45-69, and white noise gives a
flat S(k) at its variance."""
import numpy as np
import pytest

from oracle.structfact import StructFactOracle, default_pairs, unpacked_spectrum


@pytest.mark.parametrize("shape", [(4, 6, 8), (5, 3, 7), (6, 6, 6)])
def test_unpacked_spectrum_is_the_full_fft(shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape)
    re, im = unpacked_spectrum(a)
    full = np.fft.fftn(a) / np.sqrt(a.size)
    np.testing.assert_allclose(re, full.real, atol=1e-12)
    np.testing.assert_allclose(im, full.imag, atol=1e-12)


def test_parseval_and_cross_spectrum():
    rng = np.random.default_rng(2)
    v = rng.standard_normal((2, 6, 5, 8))
    sf = StructFactOracle(v.shape[1:], 2, [1.0, 1.0, 1.0])
    sf.fort_structure(v)
    re, im, mag = sf.finalize(zero_avg=0)
    assert sf.pa == [0, 1, 1] and sf.pb == [0, 0, 1]
    # S_aa summed over k equals sum of a^2 (FFT normalised by sqrt(N))
    assert re[0].sum() == pytest.approx((v[0] ** 2).sum(), rel=1e-12)
    assert re[2].sum() == pytest.approx((v[1] ** 2).sum(), rel=1e-12)
    # cross term: sum over k of Re(conj(F_b) F_a) = sum over x of a b
    assert re[1].sum() == pytest.approx((v[0] * v[1]).sum(), rel=1e-10, abs=1e-10)
    assert np.all(im[0] == 0) or np.abs(im[0]).max() < 1e-12
    np.testing.assert_allclose(mag, np.sqrt(re ** 2 + im ** 2), rtol=1e-15)


def test_white_noise_structure_factor_is_flat():
    rng = np.random.default_rng(3)
    shape = (8, 8, 8)
    sf = StructFactOracle(shape, 1, [1.0])
    for s in range(200):
        sf.fort_structure(2.0 * rng.standard_normal((1,) + shape))
    re, _, _ = sf.finalize(zero_avg=1)
    s = re[0]
    assert s[4, 4, 4] == 0.0                       # k = 0, shifted to n/2, zeroed
    assert s.sum() / (s.size - 1) == pytest.approx(4.0, rel=0.02)


def test_default_pairs_match_reference_order():
    assert default_pairs(3) == ([0, 1, 2, 1, 2, 2], [0, 0, 0, 1, 1, 2])


def test_structure_factor_stack_refusals():
    """Stacks refuse an unknown kind and x pencils of a box with n_cells[1] !=
    n_cells[2] (the reference's pencil enumeration would leave the box) before
    touching a device."""
    import ctypes as C
    from fhdex_b200 import capi
    lib = capi.load()
    h = C.c_void_p()
    sc = (C.c_double * 1)(1.0)
    n = (C.c_int * 3)(8, 4, 3)
    assert lib.fhd_sf_create_stack(C.byref(h), n, 2, 1, 1, None, None, sc, 0) == capi.FHD_ERR_UNSUPPORTED
    assert lib.fhd_sf_create_stack(C.byref(h), n, 3, 1, 1, None, None, sc, 0) == capi.FHD_ERR_BAD_ARG
    n1 = (C.c_int * 3)(1, 4, 4)
    assert lib.fhd_sf_create_stack(C.byref(h), n1, 2, 1, 1, None, None, sc, 0) == capi.FHD_ERR_BAD_ARG


def test_stack_oracle_members_are_box_oracles():
    """A z-slice stack of one slice is the box structure factor of that slice."""
    import numpy as np
    from oracle.structfact import StructFactOracle, StructFactStackOracle
    rng = np.random.default_rng(2)
    v = rng.standard_normal((2, 1, 6, 8))
    a = StructFactStackOracle((1, 6, 8), "z_slices", 2, [1.0, 2.0, 0.5])
    b = StructFactOracle((1, 6, 8), 2, [1.0, 2.0, 0.5])
    a.fort_structure(v)
    b.fort_structure(v)
    mag, ri = a.stack_average(1)
    re, im, m = b.finalize(1)
    assert np.array_equal(mag, m * 1.0) and np.array_equal(ri[:3], re) and np.array_equal(ri[3:], im)
