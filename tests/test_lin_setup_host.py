"""The device arithmetic of the linear-basis set-up, run on the host.

k_near_build_lin and k_projectors_lin (scadyn_b200/csrc/setup_device.cu) call
the phase functions of scadyn_b200/csrc/lin_setup.cuh; tests/lin_setup_check.cu
runs the same functions on the host, item by item, and this test compares them
with the oracle's compute_near_zone_interactions_lin blocks (self, same-box and
neighbouring-box pairs) and with pfft_projection_lin's node integrals.
tests/lin_tile_check.cu checks where the kernel writes the blocks in a tile.
"""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_linear_setup import FACE, QR, QRW, QT, QW, SHP_R, SHP_T, _box, _node, green, tri_points, vol6

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "scadyn_b200", "csrc")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = tmp_path_factory.mktemp("lin") / "lin_setup_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                           "-I", CSRC, os.path.join(HERE, "lin_setup_check.cu"), "-o", str(out)])
    return str(out)


@pytest.fixture(scope="module")
def setup():
    from scadyn_b200 import meshgen
    m = meshgen.sphere(3, seed=1, eps=2.25 + 0.01j)
    k = 1.0 / m.a
    g = O.Geometry(m.coord, m.etopol, m.param, k=k, grid_size=1.8)
    P = g.projectors_lin()
    sp, ind = g.nearzone_lin(*P[:4], fp64=True)
    return m, k, g, P, sp, ind


def _pair_request(m, k, g, P, tT, tB):
    Tc, Bc = m.coord[m.etopol[tT] - 1], m.coord[m.etopol[tB] - 1]
    nt = g.etopol_box[_box(g, Tc) - 1]
    nb = g.etopol_box[_box(g, Bc) - 1]
    G = np.zeros((27, 27), complex)
    for a in range(27):
        for b in range(27):
            if nt[a] != nb[b]:
                G[a, b] = green(_node(g, nt[a]), _node(g, nb[b]), k)
    kinds = P[:4]
    st = np.array([[kinds[s][4 * tT + n] for s in range(4)] for n in range(4)])          # [node][kind][27]
    gp = np.array([[G @ kinds[s][4 * tB + n] for s in range(4)] for n in range(4)])
    eps = m.param[tT]
    parts = [np.array([k, eps.real, eps.imag], np.float64).tobytes(), np.array([int(tT == tB)], np.int32).tobytes(),
             Tc.astype(np.float64).tobytes(), Bc.astype(np.float64).tobytes(),
             np.array([vol6(Tc) / 6, vol6(Bc) / 6], np.float64).tobytes(),
             st.astype(np.complex128).tobytes(), gp.astype(np.complex128).tobytes()]
    return b"".join(parts)


def test_block_arithmetic_matches_oracle(exe, setup):
    m, k, g, P, sp, ind = setup
    pairs = {(a - 1, b - 1): i for i, (a, b) in enumerate(ind)}
    boxes = [_box(g, m.coord[m.etopol[t] - 1]) for t in range(m.n_tet)]
    self_p = [(a, b) for (a, b) in pairs if a == b]
    same = [(a, b) for (a, b) in pairs if a != b and boxes[a] == boxes[b]]
    diff = [(a, b) for (a, b) in pairs if boxes[a] != boxes[b]]
    chosen = self_p[::97][:4] + same[::211][:4] + diff[::1013][:6]
    req = np.array([0, len(chosen)], np.int32).tobytes() + b"".join(_pair_request(m, k, g, P, a, b) for a, b in chosen)
    r = subprocess.run([exe], input=req, capture_output=True)
    assert r.returncode == 0, r.stderr
    out = np.frombuffer(r.stdout, np.complex128).reshape(len(chosen), 144)
    for (a, b), got in zip(chosen, out):
        want = sp[pairs[(a, b)]].reshape(144)       # memory (12,12,B): entry row + 12 col
        rel = np.abs(got - want).max() / np.abs(want).max()
        assert rel < 1e-11, ((a, b), rel)


def test_projector_sample_arithmetic(exe, setup):
    m, k, g, P, sp, ind = setup
    rng = np.random.default_rng(3)
    tets = rng.choice(m.n_tet, 6, replace=False)
    req = [np.array([1, 6 * 4], np.int32).tobytes()]
    want = []
    for t in tets:
        tc = m.coord[m.etopol[t] - 1]
        vol = vol6(tc) / 6
        for j in range(4):
            r = tc.mean(0) + g.box_delta * (rng.random(3) * 4 - 2)
            req.append(tc.astype(np.float64).tobytes() + np.array([vol, *r, k], np.float64).tobytes())
            Pb, wb = SHP_T @ tc, QW * 6 * vol
            q = (green(r, Pb, k) * wb) @ SHP_T
            q2 = np.zeros((3, 4), complex)
            for f in range(4):
                Pt, wt, n = tri_points(tc[list(FACE[f])])
                s = (green(r, Pt, k) * wt) @ SHP_R
                for l in range(3):
                    q2[:, FACE[f][l]] += n * s[l]
            want.append(np.concatenate([q, q2.reshape(12)]))
    r = subprocess.run([exe], input=b"".join(req), capture_output=True)
    assert r.returncode == 0, r.stderr
    got = np.frombuffer(r.stdout, np.complex128).reshape(len(want), 16)
    want = np.array(want)
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-12


def test_tile_positions_apply_as_matmul_Acorr(tmp_path):
    """lin_tile_positions puts every entry where the near-zone kernels' tile
    application reproduces matmul_Acorr, for diagonal and off-diagonal tiles
    with the test tet in either group; its first position reads the entry back."""
    out = tmp_path / "lin_tile_check"
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.check_call([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                           "-I", CSRC, os.path.join(HERE, "lin_tile_check.cu"), "-o", str(out)])
    r = subprocess.run([str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "6 of 6 tiles ok" in r.stdout
