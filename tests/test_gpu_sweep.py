"""A wavelength sweep in one batched solve (scd_solve_sweep, calc_T's
wavelength loop, src/T_matrix.f90:36-79): three wavelengths of one mesh, each
with its own grid, operator and VSWF order, share the solver's slots; every
wavelength's T is bit-identical to scd_compute_T_matrix on its own context
(a column's arithmetic depends on its operator only), in both precision
forms, and the sweep rejects contexts of different meshes."""
import numpy as np
import pytest

from scadyn_b200 import api

pytestmark = pytest.mark.gpu

WAVES = [(0.6, 1.8, 1), (1.2, 2.4, 2), (2.0, 1.4, 3)]     # (ka, cell size, Nmax)


def _context(mesh, ka, gs):
    d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
    s = api.Solver.from_desc(d)
    s.set_wavenumber(ka / mesh.a)
    s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
    s.build_G()
    s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C64)
    return s


@pytest.fixture(scope="module")
def sweep_ctxs(small_sphere):
    ctxs = [_context(small_sphere, ka, gs) for ka, gs, _ in WAVES]
    grids = {(c.desc.Nx, c.desc.Ny, c.desc.Nz) for c in ctxs}
    assert len(grids) == 3                       # every wavelength has its own grid
    yield ctxs
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED])
def test_sweep_equals_per_wavelength_solves(sweep_ctxs, precision):
    kw = dict(tol=1e-8, m=30, cycles=40, block=8, precision=precision, inner_tol=1e-3, max_outer=20)
    nmax = [w[2] for w in WAVES]
    Ts, its, st, rc = api.solve_sweep(sweep_ctxs, nmax, **kw)
    assert rc == api.SCD_OK and list(st) == [api.SCD_OK] * 3
    for c, Nmax, T, it in zip(sweep_ctxs, nmax, Ts, its):
        Tw, itw = c.compute_T_matrix(Nmax, **kw)
        assert np.array_equal(it, itw)
        assert np.array_equal(T, Tw)


def test_sweep_rejects_other_meshes(sweep_ctxs, small_sphere):
    from scadyn_b200 import meshgen
    other = meshgen.sphere(3, seed=2, eps=2.25 + 0.01j)
    o = _context(other, 1.0, 1.8)
    try:
        with pytest.raises(api.ScadynError) as e:
            api.solve_sweep([sweep_ctxs[0], o], [1, 1])
        assert e.value.code == api.SCD_BAD_ARG
    finally:
        o.close()
