"""The reference's T-matrix file, mirrored as .npz with the same datasets.

scadyn stores the T-matrices of all wavelengths of a run in one HDF5 file
(src/h5io.f90:429-558 T_write2file, :138-313 read_T, :562-678 T_empty,
:682-830 singleT_write2file).  HDF5 is not available here, so the file is an
.npz holding exactly those datasets:

- ``Taai_r``, ``Taai_i``, ``Tabi_r``, ``Tabi_i``, ``Tbai_r``, ``Tbai_i``,
  ``Tbbi_r``, ``Tbbi_i``: 1-D float64 of length T_size = sum_i nm_i**2,
  nm_i = (Nmax_i + 1)**2 - 1 (src/T_matrix.f90:108-112); wavelength i's
  nm_i x nm_i block starts at offset sum_{j<i} nm_j**2 and is stored
  column-major (Fortran ``reshape``);
- ``T-ref-a``: [Re eps(1), Im eps(1), a];
- ``T-wavlens``: the wavelengths 2 pi / k_i.

The reference does not store Nmax: read_T recomputes it from k_i with
``truncation_order`` (src/h5io.f90:280-291, src/common.f90:724-735).  The
mirror adds one dataset, ``Nmaxs``, so that a file written here reads back
without the mesh; :func:`read_T` uses it unless Nmaxs are passed.
"""
from __future__ import annotations

import math
import os

import numpy as np

BLOCKS = ("Taa", "Tab", "Tba", "Tbb")
DATASETS = tuple(f"{b}i_{p}" for b in BLOCKS for p in "ri")


def truncation_order(ka: float) -> int:
    """floor(ka + 4 ka^(1/3)) for ka > 1, else 4 (src/common.f90:724-735)."""
    return int(math.floor(ka + 4.0 * ka ** (1.0 / 3.0))) if ka > 1 else 4


def nmax_of_grid(k: float, Nx: int, Ny: int, Nz: int, delta: float) -> int:
    """Nmax that read_T assigns a wavelength of a mesh run: the truncation
    order of k times half the longest grid side (src/h5io.f90:286-290)."""
    return truncation_order(k * max(Nx, Ny, Nz) * delta / 2.0)


def nm_of(Nmax: int) -> int:
    return (Nmax + 1) ** 2 - 1


def T_size(Nmaxs) -> int:
    return sum(nm_of(int(n)) ** 2 for n in Nmaxs)


def offsets(Nmaxs):
    off, out = 0, []
    for n in Nmaxs:
        out.append(off)
        off += nm_of(int(n)) ** 2
    return out


def split_T(T):
    """(Taa, Tab, Tba, Tbb) of the 2nm x 2nm T returned by compute_T_matrix
    (src/T_matrix.f90:270-275; the i k^3 factor is already applied)."""
    nm = T.shape[0] // 2
    return T[:nm, :nm], T[:nm, nm:], T[nm:, :nm], T[nm:, nm:]


def _pack(blk):
    return np.asarray(blk, np.complex128).reshape(-1, order="F")


def _save(path, d):
    tmp = path + ".tmp.npz"
    np.savez(tmp, **d)
    os.replace(tmp, path)


def _load(path):
    with np.load(path) as z:
        return {k: z[k].copy() for k in z.files}


def _header(Nmaxs, wavelengths, ref_a):
    if len(Nmaxs) != len(wavelengths):
        raise ValueError("one Nmax per wavelength")
    ra = np.asarray(ref_a, np.float64)
    if ra.shape != (3,):
        raise ValueError("T-ref-a is [Re eps(1), Im eps(1), a]")
    return {"T-ref-a": ra, "T-wavlens": np.asarray(wavelengths, np.float64),
            "Nmaxs": np.asarray(Nmaxs, np.int32)}


def write_T(path, Ts, Nmaxs, wavelengths, ref_a):
    """T_write2file: Ts[i] is wavelength i's 2nm x 2nm T or its four blocks."""
    d = _header(Nmaxs, wavelengths, ref_a)
    size = T_size(Nmaxs)
    full = {b: np.zeros(size, np.complex128) for b in BLOCKS}
    for i, (T, off) in enumerate(zip(Ts, offsets(Nmaxs))):
        blocks = split_T(T) if not isinstance(T, (tuple, list)) else T
        nm = nm_of(int(Nmaxs[i]))
        for b, blk in zip(BLOCKS, blocks):
            if np.shape(blk) != (nm, nm):
                raise ValueError(f"wavelength {i}: {b} is not {nm} x {nm}")
            full[b][off:off + nm * nm] = _pack(blk)
    for b in BLOCKS:
        d[f"{b}i_r"], d[f"{b}i_i"] = full[b].real.copy(), full[b].imag.copy()
    _save(path, d)


def T_empty(path, Nmaxs, wavelengths, ref_a):
    """Create a zero T file for all wavelengths; an existing file is left as
    it is (src/h5io.f90:598).  Returns True when it created one."""
    if os.path.exists(path):
        return False
    d = _header(Nmaxs, wavelengths, ref_a)
    z = np.zeros(T_size(Nmaxs), np.float64)
    for name in DATASETS:
        d[name] = z
    _save(path, d)
    return True


def write_single_T(path, which, T, Nmaxs=None):
    """singleT_write2file: replace wavelength `which`'s slice (0-based here,
    1-based ``whichbar`` in the reference) and keep the others."""
    d = _load(path)
    Nm = [int(n) for n in (Nmaxs if Nmaxs is not None else d["Nmaxs"])]
    if not 0 <= which < len(Nm):
        raise IndexError(f"wavelength {which} of {len(Nm)}")
    if len(d["Taai_r"]) != T_size(Nm):
        raise ValueError("file size does not match the Nmaxs")
    nm, off = nm_of(Nm[which]), offsets(Nm)[which]
    blocks = split_T(T) if not isinstance(T, (tuple, list)) else T
    for b, blk in zip(BLOCKS, blocks):
        if np.shape(blk) != (nm, nm):
            raise ValueError(f"{b} is not {nm} x {nm}")
        v = _pack(blk)
        d[f"{b}i_r"][off:off + nm * nm] = v.real
        d[f"{b}i_i"][off:off + nm * nm] = v.imag
    _save(path, d)


def read_T(path, Nmaxs=None):
    """read_T: returns (list of (Taa, Tab, Tba, Tbb) per wavelength,
    wavelengths, ref_a, Nmaxs)."""
    d = _load(path)
    Nm = [int(n) for n in (Nmaxs if Nmaxs is not None else d["Nmaxs"])]
    if len(d["Taai_r"]) != T_size(Nm):
        raise ValueError("file size does not match the Nmaxs")
    out = []
    for n, off in zip(Nm, offsets(Nm)):
        nm = nm_of(n)
        blk = []
        for b in BLOCKS:
            v = d[f"{b}i_r"][off:off + nm * nm] + 1j * d[f"{b}i_i"][off:off + nm * nm]
            blk.append(v.reshape(nm, nm, order="F"))
        out.append(tuple(blk))
    return out, d["T-wavlens"], d["T-ref-a"], Nm


def wavelengths_missing(path):
    """Indices of wavelengths whose slice is still all zero (what T_empty
    wrote), i.e. the ones a resumed single-T run still has to solve."""
    d = _load(path)
    Nm = [int(n) for n in d["Nmaxs"]]
    miss = []
    for i, (n, off) in enumerate(zip(Nm, offsets(Nm))):
        s = slice(off, off + nm_of(n) ** 2)
        if not any(np.any(d[name][s]) for name in DATASETS):
            miss.append(i)
    return miss
