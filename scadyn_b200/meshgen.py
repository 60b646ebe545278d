"""Seeded synthetic tetrahedral meshes in the layout scadyn reads.

scadyn reads a tetrahedral mesh from HDF5 (``src/h5io.f90:16-136``): vertex
coordinates ``coord(3, Nv)``, 1-based connectivity ``etopol(4, T)`` and the
per-tet relative permittivity ``param`` (``param_r``/``param_i`` datasets), and
rescales the coordinates so that the volume-equivalent radius equals ``a``
(``src/h5io.f90:129-131``).  The reference builds its meshes with pymesh/tetgen
(``other/scadyn_mesh.py``); those tools are not available here, so meshes are
generated from a cube lattice instead:

* a cube lattice of spacing ``h`` is clipped to the body (a cube is kept when
  its centre is inside the body);
* every kept cube is split into the 6 Kuhn tetrahedra along its main diagonal;
* vertices whose 8 surrounding cubes are all kept ("interior" vertices) are
  jittered by U(-0.1h, 0.1h) per coordinate from a seeded generator;
* every tet is positively oriented, so the outward-normal checks of
  ``tetra_n_vectors`` (``src/common.f90:343-362``) and ``gradshape``
  (``src/common.f90:454-492``) hold.

Arrays are returned C-contiguous with the Fortran shapes reversed:
``coord`` is ``(Nv, 3)`` (memory of Fortran ``coord(3, Nv)``), ``etopol`` is
``(T, 4)`` int32 1-based (memory of ``etopol(4, T)``), ``param`` is ``(T,)``
complex128.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

# the six Kuhn tetrahedra of the unit cube: paths (0,0,0) -> (1,1,1) that
# add one unit vector per step, one per permutation of the axes
_KUHN_PERMS = list(itertools.permutations(range(3)))


@dataclass
class Mesh:
    coord: np.ndarray      # (Nv, 3) float64
    etopol: np.ndarray     # (T, 4) int32, 1-based vertex ids
    param: np.ndarray      # (T,) complex128 relative permittivity
    a: float               # volume-equivalent radius after rescaling
    info: dict = field(default_factory=dict)

    @property
    def n_tet(self) -> int:
        return int(self.etopol.shape[0])

    @property
    def n_vert(self) -> int:
        return int(self.coord.shape[0])


def _inside(body: str, axes, p):
    ax = np.asarray(axes, dtype=np.float64)
    q = p / ax
    return np.einsum("...i,...i->...", q, q) < 1.0


def tet_volumes(coord: np.ndarray, etopol: np.ndarray) -> np.ndarray:
    """Unsigned tet volumes, as ``tetra_volume`` (``src/common.f90:255-267``)."""
    P = coord[etopol - 1]                      # (T, 4, 3)
    p41 = P[:, 3] - P[:, 0]
    p21 = P[:, 1] - P[:, 0]
    p31 = P[:, 2] - P[:, 0]
    dt = np.einsum("ti,ti->t", p41, np.cross(p21, p31))
    return np.abs(dt) / 6.0


def lattice_body(n_major: float, axes=(1.0, 1.0, 1.0), *, seed: int = 0,
                 jitter: float = 0.1, a: float = 1e-7,
                 eps=2.25 + 0.01j, eps_sampler=None,
                 core_scale: float | None = None, core_eps=None,
                 body: str = "ellipsoid") -> Mesh:
    """Cube-lattice tet mesh of an ellipsoid with semi-axes ``n_major*axes``
    (in units of the lattice spacing h = 1 before rescaling).

    ``eps`` is the uniform permittivity; ``eps_sampler(rng, T)`` overrides it
    with per-tet values; ``core_scale``/``core_eps`` make a two-layer body
    whose core is the same ellipsoid scaled by ``core_scale`` (a tet belongs to
    the core when its centroid is inside it).
    """
    rng = np.random.default_rng(seed)
    semi = np.asarray(axes, dtype=np.float64) * float(n_major)
    lim = np.ceil(semi).astype(int) + 1
    ii = [np.arange(-l, l) for l in lim]
    # cube (i,j,k) occupies [i, i+1] x [j, j+1] x [k, k+1]; keep it when its
    # centre is inside the body
    K, J, I = np.meshgrid(ii[2], ii[1], ii[0], indexing="ij")
    centres = np.stack([I + 0.5, J + 0.5, K + 0.5], axis=-1)
    keep = _inside(body, semi, centres)
    cubes = np.stack([I[keep], J[keep], K[keep]], axis=-1)   # z-major order
    if cubes.shape[0] == 0:
        raise ValueError("body contains no lattice cube")

    # occupancy lookup for the interior-vertex test
    off = lim  # shift so that indices are non-negative
    shape = tuple(int(2 * l + 1) for l in lim)
    occ = np.zeros(shape, dtype=bool)
    occ[cubes[:, 0] + off[0], cubes[:, 1] + off[1], cubes[:, 2] + off[2]] = True

    # vertices used by kept cubes, numbered z-major / x-fastest
    corners = np.array(list(itertools.product((0, 1), repeat=3)))[:, ::-1]
    allv = (cubes[:, None, :] + corners[None, :, :]).reshape(-1, 3)
    key = ((allv[:, 2] + off[2]) * (shape[1] + 1) + (allv[:, 1] + off[1])) * (shape[0] + 1) \
        + (allv[:, 0] + off[0])
    ukey, inv = np.unique(key, return_inverse=True)
    verts = np.zeros((ukey.shape[0], 3), dtype=np.int64)
    verts[inv] = allv
    vid = inv.reshape(-1, 8)                         # per cube, 8 corner ids

    # interior vertices: all 8 incident cubes kept
    interior = np.ones(verts.shape[0], dtype=bool)
    for d in itertools.product((-1, 0), repeat=3):
        c = verts + np.asarray(d)
        ok = np.all((c + off >= 0) & (c + off < np.asarray(shape)), axis=1)
        o = np.zeros(verts.shape[0], dtype=bool)
        cc = c[ok] + off
        o[ok] = occ[cc[:, 0], cc[:, 1], cc[:, 2]]
        interior &= o
    coord = verts.astype(np.float64)
    jit = rng.uniform(-jitter, jitter, size=coord.shape)
    coord[interior] += jit[interior]

    # corner index of (dx,dy,dz) within the 8-corner list above
    cidx = {tuple(c): n for n, c in enumerate(corners)}
    tets = []
    for perm in _KUHN_PERMS:
        p = [0, 0, 0]
        path = [cidx[tuple(p)]]
        for ax in perm:
            p[ax] = 1
            path.append(cidx[tuple(p)])
        tets.append(path)
    tets = np.asarray(tets)                          # (6, 4) corner slots
    et = vid[:, tets].reshape(-1, 4)                 # (6*Ncubes, 4), 0-based

    # positive orientation: det[p2-p1, p3-p1, p4-p1] > 0
    P = coord[et]
    det = np.einsum("ti,ti->t", P[:, 3] - P[:, 0], np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]))
    neg = det < 0
    et[neg] = et[neg][:, [0, 2, 1, 3]]
    P = coord[et]
    det = np.einsum("ti,ti->t", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))
    if np.any(det <= 0):
        raise RuntimeError("degenerate tetrahedron after jitter")

    T = et.shape[0]
    centroid = P.mean(axis=1)
    if eps_sampler is not None:
        param = np.asarray(eps_sampler(rng, T), dtype=np.complex128)
    else:
        param = np.full(T, complex(eps), dtype=np.complex128)
    if core_scale is not None:
        incore = _inside(body, semi * core_scale, centroid)
        param = param.copy()
        param[incore] = complex(core_eps)

    etopol = (et + 1).astype(np.int32)
    # volume-equivalent rescale (src/h5io.f90:129-131)
    vol = tet_volumes(coord, etopol).sum()
    a_eff = (3.0 * vol / 4.0 / np.pi) ** (1.0 / 3.0)
    coord = coord * (a / a_eff)
    return Mesh(coord=np.ascontiguousarray(coord), etopol=np.ascontiguousarray(etopol),
                param=param, a=a,
                info={"h": a / a_eff, "n_cubes": int(cubes.shape[0]), "seed": seed,
                      "semi_axes_h": semi.tolist()})


def sphere(n_radius: float, **kw) -> Mesh:
    """Sphere of radius ``n_radius`` lattice spacings (h = a/n_radius)."""
    return lattice_body(n_radius, (1.0, 1.0, 1.0), **kw)


def ellipsoid(n_major: float, ratios=(1.0, 0.8, 0.6), **kw) -> Mesh:
    return lattice_body(n_major, ratios, **kw)


def core_mantle(n_major: float, ratios=(1.0, 1.0, 1.0), core_scale=0.6,
                core_eps=3.5 + 0.1j, mantle_eps=1.8 + 0.01j, **kw) -> Mesh:
    return lattice_body(n_major, ratios, eps=mantle_eps, core_scale=core_scale,
                        core_eps=core_eps, **kw)


def uniform_eps_sampler(re=(2.0, 3.0), im=(0.01, 0.1)):
    """Per-tet permittivity with Re ~ U(re), Im ~ U(im)."""
    def f(rng, T):
        return rng.uniform(*re, size=T) + 1j * rng.uniform(*im, size=T)
    return f


def save_npz(path: str, mesh: Mesh) -> None:
    """npz mirror of the reference's HDF5 mesh datasets ``coord``, ``etopol``,
    ``param_r``, ``param_i`` (``other/scadyn_mesh.py`` ``write_h5``)."""
    np.savez(path, coord=mesh.coord.T, etopol=mesh.etopol.T,
             param_r=mesh.param.real, param_i=mesh.param.imag, a=mesh.a)


def load_npz(path: str) -> Mesh:
    z = np.load(path)
    coord = np.ascontiguousarray(np.asarray(z["coord"]).T)
    etopol = np.ascontiguousarray(np.asarray(z["etopol"]).T.astype(np.int32))
    param = np.asarray(z["param_r"]) + 1j * np.asarray(z["param_i"])
    return Mesh(coord=coord, etopol=etopol, param=param, a=float(z["a"]))
