"""The T-matrix file mirror: the reference's dataset names, packing of every
wavelength's nm x nm blocks (column-major, back to back), T_empty leaving an
existing file alone, single-wavelength updates, and truncation_order."""
import numpy as np
import pytest

from scadyn_b200 import tfile


def _T(rng, Nmax):
    n = 2 * tfile.nm_of(Nmax)
    return rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))


def test_truncation_order():
    assert tfile.truncation_order(0.5) == 4 and tfile.truncation_order(1.0) == 4
    assert tfile.truncation_order(2.0) == 7        # floor(2 + 4 * 1.2599)
    assert tfile.truncation_order(8.0) == 16       # floor(8 + 4 * 2)
    assert tfile.nmax_of_grid(1.0, 64, 54, 40, 0.25) == tfile.truncation_order(8.0)


def test_round_trip_and_packing(tmp_path):
    rng = np.random.default_rng(5)
    Nmaxs, wl = [1, 3, 2], [1.0, 0.7, 0.5]
    Ts = [_T(rng, n) for n in Nmaxs]
    p = str(tmp_path / "T.npz")
    tfile.write_T(p, Ts, Nmaxs, wl, [2.25, 0.01, 1.5])
    z = np.load(p)
    assert set(tfile.DATASETS) | {"T-ref-a", "T-wavlens", "Nmaxs"} == set(z.files)
    assert z["Taai_r"].shape == (3 ** 2 + 15 ** 2 + 8 ** 2,)
    # wavelength 1 (Nmax 3, nm 15), block Tba, element (r, c) at 9 + r + 15 c
    r, c = 4, 11
    v = Ts[1][15 + r, c]
    assert z["Tbai_r"][9 + r + 15 * c] == v.real and z["Tbai_i"][9 + r + 15 * c] == v.imag
    blocks, wls, ref_a, Nm = tfile.read_T(p)
    assert Nm == Nmaxs and np.array_equal(wls, wl) and np.array_equal(ref_a, [2.25, 0.01, 1.5])
    for T, b in zip(Ts, blocks):
        assert np.array_equal(np.block([[b[0], b[1]], [b[2], b[3]]]), T)


def test_empty_then_single_writes(tmp_path):
    rng = np.random.default_rng(6)
    Nmaxs, wl = [2, 1, 2], [1.0, 0.8, 0.6]
    p = str(tmp_path / "T.npz")
    assert tfile.T_empty(p, Nmaxs, wl, [2.5, 0.05, 1.0])
    assert tfile.wavelengths_missing(p) == [0, 1, 2]
    T1 = _T(rng, 1)
    tfile.write_single_T(p, 1, T1)
    assert not tfile.T_empty(p, Nmaxs, wl, [2.5, 0.05, 1.0])     # existing file kept
    assert tfile.wavelengths_missing(p) == [0, 2]
    blocks, _, _, _ = tfile.read_T(p)
    assert np.array_equal(np.block([[blocks[1][0], blocks[1][1]], [blocks[1][2], blocks[1][3]]]), T1)
    assert not np.any(blocks[0][0]) and not np.any(blocks[2][3])
    with pytest.raises(ValueError):
        tfile.write_single_T(p, 0, T1)                          # Nmax 1 block into an Nmax 2 slot
    with pytest.raises(IndexError):
        tfile.write_single_T(p, 3, T1)
    with pytest.raises(ValueError):
        tfile.read_T(p, Nmaxs=[2, 2, 2])
