"""Request loop (include/scadyn_server.h): requests of different meshes,
wavelengths and precision forms give the same T-matrix alone and in a mix
(bit-identical: a request's arithmetic depends on its own data only), the HBM
budget bounds how many run at once, and an oversize request is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from scadyn_b200 import api, meshgen
    sph = meshgen.sphere(4, seed=1, eps=2.25 + 0.01j)
    cm = meshgen.core_mantle(4, seed=3)
    return [
        (sph, 1.5 / sph.a, 1.8, 3, dict(precision=api.PREC_FP64, tol=1e-8)),
        (sph, 2.5 / sph.a, 1.8, 3, dict(precision=api.PREC_MIXED, tol=1e-8, m=20)),
        (cm, 2.0 / cm.a, 1.8, 2, dict(precision=api.PREC_FP64, tol=1e-8)),
    ]


def _solve(srv, reqs, all_at_once):
    out = []
    if all_at_once:
        ids = [srv.submit(m, k, gs, nmax, **o) for m, k, gs, nmax, o in reqs]
        for i in ids:
            srv.wait(i, 600)
        return [srv.result(i)[0] for i in ids]
    for m, k, gs, nmax, o in reqs:
        i = srv.submit(m, k, gs, nmax, **o)
        srv.wait(i, 600)
        out.append(srv.result(i)[0])
    return out


def test_alone_equals_mix():
    from scadyn_b200.server import Server
    reqs = _requests()
    alone = Server(max_running=1)
    Ta = _solve(alone, reqs, all_at_once=False)
    alone.close()
    mix = Server(max_running=3)
    Tm = _solve(mix, reqs, all_at_once=True)
    st = mix.stats()
    mix.close()
    assert st["completed"] == 3 and st["peak_running"] == 3
    for a, b in zip(Ta, Tm):
        assert np.array_equal(a, b)


def test_server_T_equals_direct_solve():
    """A request's T equals the T of the same set-up driven through the
    per-context entry points."""
    from scadyn_b200 import api, geometry
    from scadyn_b200.server import Server
    mesh, k, gs, nmax, o = _requests()[0]
    srv = Server(max_running=1)
    i = srv.submit(mesh, k, gs, nmax, **o)
    srv.wait(i, 600)
    T_srv = srv.result(i)[0]
    srv.close()
    d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
    s = api.Solver.from_desc(d)
    s.set_wavenumber(k)
    s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
    s.build_G()
    s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C64)
    T_dir, _ = s.compute_T_matrix(nmax, tol=o["tol"], m=50, cycles=12, block=16)
    s.close()
    assert np.array_equal(T_srv, T_dir)


def test_budget_bounds_running_requests():
    from scadyn_b200.server import Server
    reqs = _requests()
    probe = Server(max_running=1)
    est = max(probe.estimate(m, k, gs, nmax, **o) for m, k, gs, nmax, o in reqs)
    probe.close()
    srv = Server(hbm_budget=int(est * 1.5), max_running=3)
    ids = [srv.submit(m, k, gs, nmax, **o) for m, k, gs, nmax, o in reqs]
    for i in ids:
        srv.wait(i, 600)
    st = srv.stats()
    srv.close()
    assert st["completed"] == 3
    assert st["peak_running"] == 1
    assert st["peak_bytes"] <= est * 1.5


def test_oversize_request_refused():
    from scadyn_b200 import api
    from scadyn_b200.server import Server
    mesh, k, gs, nmax, o = _requests()[0]
    srv = Server(hbm_budget=1 << 20, max_running=1)
    with pytest.raises(api.ScadynError) as e:
        srv.submit(mesh, k, gs, nmax, **o)
    srv.close()
    assert e.value.code == api.SCD_OOM


def test_same_key_requests_share_a_resident_pool():
    """Requests with one operator key share a pool: the second joins while the
    first is solving (its columns batch with the first's), a third after both
    finished finds the pool resident (no rebuild); each T is bit-identical to
    the same request served alone, and a result is read once."""
    from scadyn_b200 import api
    from scadyn_b200.server import Server
    mesh, k, gs, _, o = _requests()[0]
    alone = Server()
    ia = alone.submit(mesh, k, gs, 2, **o)
    alone.wait(ia, 600)
    T2_alone = alone.result(ia)[0]
    alone.close()

    srv = Server()
    i3 = srv.submit(mesh, k, gs, 3, **o)
    i2 = srv.submit(mesh, k, gs, 2, **o)
    srv.wait(i3, 600)
    srv.wait(i2, 600)
    st = srv.stats()
    assert st["pools_built"] == 1 and st["pool_reuses"] == 1 and st["pools_resident"] == 1
    T2 = srv.result(i2)[0]
    assert np.array_equal(T2, T2_alone)
    with pytest.raises(api.ScadynError) as e:       # released by the first read
        srv.result(i2)
    assert e.value.code == api.SCD_NOT_READY
    i2b = srv.submit(mesh, k, gs, 2, **o)
    srv.wait(i2b, 600)
    st = srv.stats()
    assert st["pools_built"] == 1 and st["pool_reuses"] == 2
    assert np.array_equal(srv.result(i2b)[0], T2_alone)
    srv.close()
