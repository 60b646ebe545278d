#!/usr/bin/env python
"""T-matrix solve benchmark: columns/s and per-column solve latency.

Workload (default): a seeded synthetic ellipsoid with semi-axes 1:0.8:0.6 at
size parameter ka = 8 (~150k tetrahedra from a jittered cube-lattice mesh,
per-tet eps with Re ~ U(2,3), Im ~ U(0.01,0.1)), zero-padded pFFT grid 128^3
(64 nodes on the longest axis), Nmax = 14 (448 incident VSWF columns).
`--config c1` runs the 43k-tet sphere (ka = 2, Nmax = 6, grid 64^3).

A step solves `--block` consecutive T-matrix columns (cycling through the
448) in the mixed-precision form: complex64 inner GMRES(30) to 3e-4 and FP64
iterative refinement on the true residual to 1e-6, `--slots` columns in
flight.  `value` is columns/s over K timed steps with the operator and the
incident columns resident in HBM (device time from CUDA events on the
library's stream, max over ranks); `e2e` is the same through the C ABI call a
host makes (scd_solve_columns with host buffers: the whole incident matrix
copied in from page-locked memory and the step's T columns copied out, every
step, inside the timed region).  `forms` holds the plain FP64 GMRES(50) form
one column at a time and batched, on the same columns, and
`t_rel_err_vs_fp64` the Frobenius error of the mixed T against the FP64 T.
`--impl reference` runs the reference's algorithm on the host cores through
the CPU oracle (its C restatement), end to end: the oracle sets up its own
operator and solves `--ref-columns` columns with its FP64 GMRES; the metric
string, unit and direction are the same as this arm's.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c1": dict(workload="C1: sphere ka=2, h=a/12 (~43k tets), eps=2.25+0.01i, Nmax=6 (96 columns), "
                        "padded pFFT grid 64^3, GMRES(50) tol 1e-6",
               body="sphere", n_major=12.0, axes=(1.0, 1.0, 1.0), ka=2.0, eps=2.25 + 0.01j,
               Nmax=6, N=32, tol=1e-6, m=50, cycles=4, seed=1001, eps_seed=2001,
               inner_m=30, inner_tol=3e-4, max_outer=10),
    "c2": dict(workload="C2: ellipsoid 1:0.8:0.6, ka=8 (~150k tets), per-tet eps Re U(2,3) Im U(0.01,0.1), "
                        "Nmax=14 (448 columns), padded pFFT grid 128^3, GMRES(50) tol 1e-6",
               body="ellipsoid", n_major=23.2, axes=(1.0, 0.8, 0.6), ka=8.0, eps=None,
               Nmax=14, N=64, tol=1e-6, m=50, cycles=12, seed=1002, eps_seed=2002,
               inner_m=30, inner_tol=3e-4, max_outer=10),
    "c5": dict(workload="C5: core-mantle ellipsoid 1:0.7:0.5, core at 60% (eps 3.5+0.1i), mantle eps 1.8+0.01i, "
                        "ka=20, ~1.2M tets, Nmax=25 (1350 columns), padded pFFT grid 256^3",
               body="core_mantle", n_major=51.6, axes=(1.0, 0.7, 0.5), ka=20.0, eps=1.8 + 0.01j,
               core_scale=0.6, core_eps=3.5 + 0.1j,
               Nmax=25, N=128, tol=1e-6, m=50, cycles=12, seed=1005, eps_seed=2005,
               inner_m=30, inner_tol=3e-4, max_outer=10),
    # C2-shaped case at a third of the size (for ncu captures: ~1 GB of near-zone tiles)
    "c2s": dict(workload="C2-shaped ellipsoid 1:0.8:0.6 at n_major 16 (~49k tets), ka=8, per-tet eps Re U(2,3) "
                         "Im U(0.01,0.1), Nmax=14, padded pFFT grid 88^3",
                body="ellipsoid", n_major=16.0, axes=(1.0, 0.8, 0.6), ka=8.0, eps=None,
                Nmax=14, N=44, tol=1e-6, m=50, cycles=12, seed=1002, eps_seed=2002,
                inner_m=30, inner_tol=3e-4, max_outer=10),
}

L2_BYTES = 126 * 1024 * 1024

# the headline metric, the same string in both arms
METRIC = "T-matrix columns/sec & p50/p99 solve latency at \u22641e-5 rel err, mixed vs plain FP64"
# kernel choices of scd_grid_desc / scd_solve_opts (0 = the library's default)
NEAR_KERNELS = {"default": 0, "cuda": 1, "split": 2, "merged": 3, "wide": 4}
GRAM_SCHMIDT = {"default": 0, "modified": 1, "classical": 2}
FFT_LENGTHS = {"default": 0, "pow2": 1, "smooth": 2}
FFT_PASSES = {"default": 0, "fused": 1, "three": 2}
NEAR_SPLIT = {"default": 0, "one": 1, "two": 2}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_mesh(cfg):
    from scadyn_b200 import meshgen
    kw = dict(seed=cfg["seed"])
    if cfg["eps"] is None:
        sampler = meshgen.uniform_eps_sampler((2.0, 3.0), (0.01, 0.1))
        rng_eps = np.random.default_rng(cfg["eps_seed"])
        mesh = meshgen.lattice_body(cfg["n_major"], cfg["axes"], eps=2.5, **kw)
        mesh.param = sampler(rng_eps, mesh.n_tet)
    elif cfg.get("core_scale"):
        mesh = meshgen.core_mantle(cfg["n_major"], cfg["axes"], core_scale=cfg["core_scale"],
                                   core_eps=cfg["core_eps"], mantle_eps=cfg["eps"], **kw)
    else:
        mesh = meshgen.lattice_body(cfg["n_major"], cfg["axes"], eps=cfg["eps"], **kw)
    return mesh


def build_solver(cfg, mesh, device, order=0, choices=None):
    """The operator from the mesh on the device; order 1 = linear basis (4
    basis functions per tet); choices = kernel choices of scd_grid_desc."""
    from scadyn_b200 import api, geometry
    gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, cfg["N"])
    d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
    d.device = device
    d.order = order
    for key, v in (choices or {}).items():
        setattr(d, key, v)
    s = api.Solver.from_desc(d, device=device)
    k = cfg["ka"] / mesh.a
    t0 = time.time()
    s.set_wavenumber(k)
    s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
    s.build_G()
    s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C64)
    setup_s = time.time() - t0
    return s, d, gs, k, setup_s


class Clocks:
    """nvidia-smi sampler during the timed region."""

    def __init__(self, device):
        self.path = tempfile.mktemp(suffix=".csv")
        self.device = device
        self.p = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if not self.p or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """ncu DRAM bytes per launch from a committed summary (profiles/<name>.txt)."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def cpu_oracle_op(solver, mesh, grid_size, k):
    """The CPU oracle's operator on the same data as the device's
    (projectors and near-zone blocks copied back, Green spectrum rebuilt on
    the CPU); returns (operator, seconds spent)."""
    from oracle import oracle as O
    t0 = time.time()
    g = O.Geometry(mesh.coord, mesh.etopol, mesh.param, k=k, grid_size=grid_size)
    S, Sx, Sy, Sz, indS = solver.get_projectors()
    sp, ind = solver.get_nearzone()
    sp = sp.astype(np.complex64)
    Fg = g.build_G()
    op = O.Operator(g, S, Sx, Sy, Sz, indS, Fg, sp, ind, merged=False, nthreads=0)
    return op, time.time() - t0


def mgs_unit_s(n, nvec=8, reps=3):
    """Seconds per modified Gram-Schmidt term (one <v_k, w> and one w -= h v_k
    over n unknowns, all host threads) of the oracle's GMRES, timed directly
    on nvec random Krylov vectors."""
    from oracle import oracle as O
    rng = np.random.default_rng(11)
    V = rng.standard_normal((nvec, n)) + 1j * rng.standard_normal((nvec, n))
    w = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    O.mgs_terms(V, w.copy())                       # warm
    best = 1e30
    for _ in range(reps):
        ww = w.copy()
        t = time.time()
        O.mgs_terms(V, ww)
        best = min(best, (time.time() - t) / nvec)
    return best


def mgs_terms_of(it, m):
    """MGS terms of a restarted GMRES(m) column that took `it` Arnoldi steps."""
    terms, left = 0, it
    while left > 0:
        s = min(left, m)
        terms += s * (s + 1) // 2
        left -= s
    return terms


def cpu_baseline(solver, mesh, grid_size, k, cfg, iters, cycles_run, op=None):
    """A bounded CPU sample beside the GPU line (about half a minute): the
    oracle's compute_Ax2 (six convolutions, complex64 near zone widened, all
    host threads) on the device-built operator copied back, and its MGS term
    cost timed alone; columns/s extrapolated with the GPU FP64 form's
    per-column iteration counts of the same columns.  `bench.py --impl
    reference` is the measured end-to-end CPU run."""
    prep = 0.0
    if op is None:
        op, prep = cpu_oracle_op(solver, mesh, grid_size, k)
    g = op.geom
    ncores = os.cpu_count()
    rng = np.random.default_rng(7)
    x = rng.standard_normal(3 * g.T) + 1j * rng.standard_normal(3 * g.T)
    op.compute_Ax2(x)                      # warm
    t = time.time()
    for _ in range(3):
        op.compute_Ax2(x)
    t_mv = (time.time() - t) / 3
    t_unit = mgs_unit_s(3 * g.T)
    per_col = [(it + cy) * t_mv + t_unit * mgs_terms_of(it, cfg["m"]) for it, cy in zip(iters, cycles_run)]
    value = 1.0 / float(np.mean(per_col))
    sample = (f"extrapolated: oracle compute_Ax2 x3 ({t_mv:.3f} s each) and MGS terms timed alone "
              f"({t_unit * 1e3:.2f} ms each) on the device-built operator copied back; per column "
              f"(iters + cycles) matvecs + MGS terms with the GPU FP64 iteration counts of the same columns "
              f"(mean {np.mean(iters):.1f}); operator copy-back {prep:.1f} s")
    return {"value": value, "unit": "columns/s", "cores": ncores, "kind": "port", "sample": sample,
            "t_matvec_s": t_mv, "t_mgs_unit_s": t_unit}


def reference_arm(args, cfg):
    """The reference's algorithm on the host cores, end to end, through the
    oracle (its C restatement of the Fortran): the operator set up by the
    oracle itself (pfft_projection_const, build_G,
    compute_near_zone_interactions_const), then `--ref-columns` T-matrix
    columns spread over all 2nm solved one at a time with its restarted FP64
    GMRES(m) (src/T_matrix.f90:254-268, src/gmres_module.f90:180-325) and
    assembled as mat^H x.  Columns/s = columns / measured solve time."""
    from oracle import oracle as O
    from scadyn_b200 import geometry
    mesh = make_mesh(cfg)
    gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, cfg["N"])
    k = cfg["ka"] / mesh.a
    t0 = time.time()
    op = O.setup(mesh, k, grid_size=gs, nthreads=0)
    op.nthreads = 0
    setup_s = time.time() - t0
    mat = O.vswf2constant(mesh.coord, mesh.etopol, k, cfg["Nmax"])
    ncol_tot = mat.shape[0]
    log(f"[reference] T={mesh.n_tet} grid={op.geom.Nx}x{op.geom.Ny}x{op.geom.Nz} "
        f"near blocks={op.sp_ind.shape[0]} oracle set-up {setup_s:.0f}s")
    rng = np.random.default_rng(7)
    x = rng.standard_normal(3 * mesh.n_tet) + 1j * rng.standard_normal(3 * mesh.n_tet)
    for _ in range(args.warmup):
        op.compute_Ax2(x)
    nref = max(1, args.ref_columns)
    cols = [int(c) for c in np.unique(np.linspace(0, ncol_tot - 1, nref + 2).round().astype(int)[1:-1])]
    secs, iters, T_err = [], [], []
    for c in cols:
        t = time.time()
        xs, info = op.gmres(mat[c], tol=cfg["tol"], m=cfg["m"], cycles=cfg["cycles"])
        Tc = mat.conj() @ xs                       # T_mat(:, c) = mat^H x (src/T_matrix.f90:260)
        secs.append(time.time() - t)
        iters.append(int(info["iters"]))
        log(f"[reference] column {c}: {info['iters']} iterations, relres {info['relres']:.2e}, {secs[-1]:.1f}s")
    value = len(cols) / float(sum(secs))
    ncores = os.cpu_count()
    sample = (f"{len(cols)} columns {cols} of {ncol_tot} solved end to end (FP64 GMRES({cfg['m']}), tol {cfg['tol']:g}, "
              f"mean {np.mean(iters):.1f} iterations) on the oracle's own operator, all {ncores} host threads; "
              f"operator set-up {setup_s:.0f} s not timed")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "columns/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128 (near zone stored complex64, as the reference)",
            "data": "synthetic (seeded jittered cube-lattice mesh)",
            "config": {"workload": cfg["workload"], "tets": mesh.n_tet,
                       "grid_nodes": [op.geom.Nx, op.geom.Ny, op.geom.Nz], "near_blocks": int(op.sp_ind.shape[0]),
                       "form": "plain FP64 GMRES(%d), one column at a time (the reference's only form)" % cfg["m"]},
            "p50_ms": round(float(np.percentile(secs, 50)) * 1e3, 1),
            "p99_ms": round(float(np.percentile(secs, 99)) * 1e3, 1),
            "columns": cols, "iters": iters, "column_s": [round(v, 2) for v in secs], "setup_s": round(setup_s, 1),
            "cpu_baseline": {"value": value, "unit": "columns/s", "cores": ncores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "columns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def pinned_like(a):
    """A page-locked host copy of a numpy array (torch pin_memory), so that
    host->device copies run at full bus speed as a host application's would."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--block", type=int, default=64, help="columns per step")
    ap.add_argument("--slots", type=int, default=32, help="columns solved concurrently (batched GMRES slots)")
    ap.add_argument("--plain-sample", type=int, default=8, help="columns timed in the plain one-at-a-time form")
    ap.add_argument("--ref-columns", type=int, default=2, help="columns the CPU reference arm solves end to end")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream summary")
    ap.add_argument("--no-tune", action="store_true", help="keep the library's default matvec kernels")
    ap.add_argument("--tune-slots", action="store_true",
                    help="also choose slots and the inner Krylov dimension from a sample of columns")
    ap.add_argument("--serve", type=int, default=0,
                    help="run a served request stream of this many requests instead (C4-shaped, scaled)")
    ap.add_argument("--serve-scale", default="small", choices=["small", "c4"],
                    help="request sizes of the served stream: small (5k-60k tets) or c4 (5k-300k tets, Nmax 4-16)")
    ap.add_argument("--sweep", type=int, default=0,
                    help="run a C3-shaped wavelength sweep with this many wavelengths instead")
    ap.add_argument("--sweep-nmax", type=int, default=14, help="largest Nmax of the sweep (C3: 14)")
    ap.add_argument("--profile", default=None,
                    choices=["near1", "near16", "mixed16", "mixed32", "solve16", "near-compare", "linear"],
                    help="only build the operator and run profile_matvec (for ncu captures); near-compare times "
                         "the complex64 x16 matvec with the CUDA-core near zone and both tensor-core schedules; "
                         "linear times the linear-basis set-up and matvec against the constant basis")
    ap.add_argument("--near-kernel", default="default", choices=sorted(NEAR_KERNELS),
                    help="near zone of the complex64 matvec (scd_grid_desc.near_kernel)")
    ap.add_argument("--gram-schmidt", default="default", choices=sorted(GRAM_SCHMIDT),
                    help="orthogonalisation of the complex64 inner solves (scd_solve_opts.gram_schmidt)")
    ap.add_argument("--fft-lengths", default="default", choices=sorted(FFT_LENGTHS),
                    help="padded FFT lengths (scd_grid_desc.fft_lengths)")
    ap.add_argument("--fft-passes", default="default", choices=sorted(FFT_PASSES),
                    help="fused y-z FFT pass or three separate passes (scd_grid_desc.fft_passes)")
    ap.add_argument("--near-split", default="default", choices=sorted(NEAR_SPLIT),
                    help="partial sums per FP64 near-zone row and column sum (scd_grid_desc.near_split)")
    args = ap.parse_args()
    choices = dict(near_kernel=NEAR_KERNELS[args.near_kernel], fft_lengths=FFT_LENGTHS[args.fft_lengths],
                   near_split=NEAR_SPLIT[args.near_split], fft_passes=FFT_PASSES[args.fft_passes])
    gs_choice = GRAM_SCHMIDT[args.gram_schmidt]
    if args.serve:
        print(json.dumps(serve_bench(args.serve, args.serve_scale, check_err=args.serve_scale != "small")),
              flush=True)
        return
    if args.sweep:
        print(json.dumps(sweep_bench(args.sweep, args.sweep_nmax)), flush=True)
        return
    cfg = CONFIGS[args.config]

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        # the CPU arm: rank 0 alone, no GPU work and no collective
        if rank == 0:
            reference_arm(args, cfg)
        return
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from scadyn_b200 import api
    mesh = make_mesh(cfg)
    solver, desc, gs, k, setup_s = build_solver(cfg, mesh, local, choices=choices)
    Nmax = cfg["Nmax"]
    ncol_tot = 2 * ((Nmax + 1) ** 2 - 1)
    B = args.block
    log(f"[rank {rank}] T={mesh.n_tet} grid={desc.Nx}x{desc.Ny}x{desc.Nz} near blocks={solver.nearzone_count()} "
        f"setup {setup_s:.1f}s")
    mixed = dict(tol=cfg["tol"], m=cfg["inner_m"], cycles=60, precision=api.PREC_MIXED,
                 inner_tol=cfg["inner_tol"], max_outer=cfg["max_outer"], gram_schmidt=gs_choice)
    if args.profile == "solve16":
        # sixteen columns in the mixed batched form (large configs: a sample of the column loop)
        solver.timing(reset=True)
        _, it = solver.compute_T_matrix(Nmax, col0=0, ncol=16, block=16, **mixed)
        ms = solver.timing(reset=True)["accum_ms"]
        print(json.dumps({"config": args.config, "tets": mesh.n_tet, "grid_nodes": [desc.Nx, desc.Ny, desc.Nz],
                          "near_bytes": solver.nearzone_bytes(), "setup_s": round(setup_s, 2),
                          "columns": 16, "columns_per_s": round(16 / (ms / 1e3), 4),
                          "iters_mean": float(np.mean(it))}), flush=True)
        solver.close()
        return
    if args.profile == "linear":
        # linear basis (mesh%order = 1) on the same mesh and grid: set-up from
        # the mesh, then median FP64 and complex64 matvec times, beside the
        # constant basis already built
        out = {"config": args.config, "tets": mesh.n_tet, "setup_s": {"constant": round(setup_s, 2)}, "ms": {}}
        runs = [solver.profile_matvec(10, 1, api.PREC_FP64) for _ in range(5)]
        out["ms"]["constant_fp64_1rhs"] = round(float(np.median([r["matvec_ms"] for r in runs])), 4)
        solver.close()
        sv, _, _, _, lin_setup_s = build_solver(cfg, mesh, local, order=1, choices=choices)
        out["setup_s"]["linear"] = round(lin_setup_s, 2)
        out["near_blocks_12x12"] = sv.nearzone_count()
        for label, nrhs, prec in (("linear_fp64_1rhs", 1, api.PREC_FP64), ("linear_c64_16rhs", 16, api.PREC_MIXED)):
            runs = [sv.profile_matvec(10, nrhs, prec) for _ in range(5)]
            out["ms"][label] = {key: round(float(np.median([r[key] for r in runs])), 4)
                                for key in ("nearzone_ms", "fft_ms", "gather_ms", "matvec_ms")}
        sv.close()
        print(json.dumps(out), flush=True)
        return
    if args.profile == "near-compare":
        # one operator build per context (the kernel is fixed at creation); the
        # same mesh, 16 and 32 complex64 right-hand sides, median of 5 profiled loops
        solver.close()
        out = {"config": args.config, "tets": mesh.n_tet, "ms": {}}
        for label in ("cuda", "split", "merged", "wide"):
            sv, _, _, _, _ = build_solver(cfg, mesh, local, choices=dict(choices, near_kernel=NEAR_KERNELS[label]))
            for nrhs in (16, 32, 64):
                runs = [sv.profile_matvec(10, nrhs, api.PREC_MIXED) for _ in range(5)]
                out["ms"][f"{label}_{nrhs}"] = {key: round(float(np.median([r[key] for r in runs])), 4)
                                                for key in ("nearzone_ms", "near_kernel_ms", "fft_ms", "gather_ms",
                                                            "matvec_ms")}
            sv.close()
        print(json.dumps(out), flush=True)
        return
    if args.profile:
        nrhs, prec = {"near1": (1, api.PREC_FP64), "near16": (16, api.PREC_FP64),
                      "mixed16": (16, api.PREC_MIXED), "mixed32": (32, api.PREC_MIXED)}[args.profile]
        for _ in range(3):
            t = solver.profile_matvec(1, nrhs, prec)
            log(f"profile {args.profile}: " + ", ".join(f"{k} {t[k]:.4f}" for k in ("nearzone_ms", "near_kernel_ms",
                                                                                   "fft_ms", "gather_ms",
                                                                                   "matvec_ms")))
        solver.close()
        return

    def cols_for(step):
        c0 = ((rank * (args.warmup + args.steps) + step) * B) % ncol_tot
        return min(c0, ncol_tot - B)

    # ---------------------------------------------------------------- ours
    # headline form: mixed precision (complex64 inner GMRES(inner_m) to
    # inner_tol, FP64 iterative refinement on the true residual to tol),
    # `S` columns in flight as batched slots, continuous batching
    fp64 = dict(tol=cfg["tol"], m=cfg["m"], cycles=cfg["cycles"])
    S = min(args.slots, B)
    # autotuner: the matvec kernels for the timed region's shape (S complex64
    # right-hand sides), and on request the slots and inner Krylov dimension
    # from a short sample of columns (untimed, before the warm-up)
    tuning = None
    if not args.no_tune:
        from scadyn_b200 import autotune
        t_tune = time.time()
        mv, cached = autotune.tune_matvec(solver, S, api.PREC_MIXED)
        tuning = {"matvec": {k: (round(v, 4) if isinstance(v, float) else v) for k, v in mv.items()},
                  "cached": cached}
        if args.tune_slots:
            choice, rates, _ = autotune.tune_slots(solver, Nmax, sample_cols=B, slots=(16, 32, 64),
                                                   inner_m=(20, 30), col0=cols_for(0),
                                                   tol=cfg["tol"], cycles=60, inner_tol=cfg["inner_tol"],
                                                   max_outer=cfg["max_outer"])
            S = min(choice["slots"], B)
            mixed["m"] = choice["inner_m"]
            tuning["slots"] = {"choice": choice, "columns_per_s": rates}
        tuning["seconds"] = round(time.time() - t_tune, 2)
    for st in range(args.warmup):
        solver.compute_T_matrix(Nmax, col0=cols_for(st), ncol=B, block=S, **mixed)

    def barrier():
        if dist:
            import torch
            dist.barrier()
            torch.cuda.synchronize()

    def max_over_ranks(v):
        if not dist:
            return v
        import torch
        tt = torch.tensor([v], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    lat, iters, T_mixed0 = [], [], None
    barrier()
    solver.timing(reset=True)
    t_wall = time.time()
    with Clocks(local) as clk:
        for st in range(args.warmup, args.warmup + args.steps):
            c0 = cols_for(st)
            Tm, it = solver.compute_T_matrix(Nmax, col0=c0, ncol=B, block=S, **mixed)
            if T_mixed0 is None:
                T_mixed0 = Tm
            lat += list(solver.column_latency(B))
            iters += [int(v) for v in it]
    barrier()
    wall = time.time() - t_wall
    tm = solver.timing(reset=True)
    dev_ms = max_over_ranks(tm["accum_ms"])
    launches = int(tm["launches"])
    cols = args.steps * B
    value = world * cols / (dev_ms / 1e3)

    # the same columns in FP64 (the plain algorithm, batched): accuracy
    # reference for the mixed T and the batched-FP64 comparison form
    forms = {}
    c0 = cols_for(args.warmup)
    solver.timing(reset=True)
    T64, it64 = solver.compute_T_matrix(Nmax, col0=c0, ncol=B, block=S, **fp64)
    ms64 = solver.timing(reset=True)["accum_ms"]
    t_err = float(np.linalg.norm(T_mixed0 - T64) / np.linalg.norm(T64))
    forms["batched_fp64_%d_slots" % S] = round(B / (ms64 / 1e3), 4)
    fp64_iters, fp64_cycles = [int(v) for v in it64], [max(1, -(-int(v) // cfg["m"])) for v in it64]
    # plain form: one column at a time, FP64 GMRES(m) -- the reference's algorithm on the GPU
    if args.plain_sample > 0:
        solver.timing(reset=True)
        pick = np.unique(np.linspace(0, B - 1, args.plain_sample).round().astype(int))
        for j in pick:
            solver.compute_T_matrix(Nmax, col0=c0 + int(j), ncol=1, block=1, **fp64)
        pm = solver.timing(reset=True)["accum_ms"]
        forms["plain_fp64_one_column"] = round(len(pick) / (pm / 1e3), 4)
        forms["plain_fp64_columns_timed"] = int(len(pick))
    forms["mixed_batched_%d_slots" % S] = round(value / world, 4)
    if "plain_fp64_one_column" in forms:
        forms["mixed_batched_over_plain_fp64"] = round(forms["mixed_batched_%d_slots" % S] /
                                                       forms["plain_fp64_one_column"], 3)

    # e2e: the same columns through the C ABI a host calls, scd_solve_columns
    # with host buffers: every step copies the whole incident matrix mat
    # (3T, 2nm) in from page-locked memory (T_mat = mat^H x needs all of it)
    # and the step's T columns (2nm, B) out
    mat_all = solver.vswf2constant(Nmax)
    _keep, mat_pinned = pinned_like(mat_all)
    e2e_ms = 0.0
    h2d = d2h = 0
    T_e2e0 = None
    for st in range(args.warmup, args.warmup + args.steps):
        c0s = cols_for(st)
        t = time.time()
        Tc, its, _, _ = solver.solve_columns(mat_pinned, col0=c0s, ncol=B, block=S, **mixed)
        e2e_ms += (time.time() - t) * 1e3
        if T_e2e0 is None:
            T_e2e0 = Tc
        h2d = mat_pinned.nbytes
        d2h = Tc.nbytes + its.nbytes
    e2e_val = world * cols / (max_over_ranks(e2e_ms) / 1e3)
    # the e2e T columns are the unscaled T_mat = mat^H x; times i k^3 they are
    # the timed region's first T block
    k3 = k ** 3
    e2e_vs_device = float(np.linalg.norm(1j * k3 * T_e2e0.T - T_mixed0) / np.linalg.norm(T_mixed0))

    # per-kernel times of the batched complex64 matvec (the timed region's shape)
    profb = solver.profile_matvec(5, S, api.PREC_MIXED)
    batched = {"nrhs": S, "precision": "complex64", "matvec_ms": profb["matvec_ms"],
               "nearzone_ms": profb["nearzone_ms"], "fft_chain_ms": profb["fft_ms"],
               "gather_ms": profb["gather_ms"]}
    peak, kind = peaks()
    Bref = solver.nearzone_count()
    alg_bytes = Bref * (9 * 8 + 8)                 # complex64 blocks + index pair, per pass over the tiles
    # roofline of the headline's dominant kernel: the complex64 near-zone
    # kernel the timed steps used, at the right-hand sides of one of its
    # launches (one pass of the batched inner matvec), live CUDA events on the
    # library's stream
    nk = tuning["matvec"]["near_kernel"] if tuning else choices["near_kernel"]
    nk = nk or NEAR_KERNELS["merged"]
    per_launch = 32 if nk == NEAR_KERNELS["wide"] else 16
    kname = {NEAR_KERNELS["wide"]: "k_near_mma<2> (tensor-core near zone, wide schedule)",
             NEAR_KERNELS["merged"]: "k_near_mma<1> (tensor-core near zone, merged schedule)",
             NEAR_KERNELS["split"]: "k_near_mma<0> (tensor-core near zone, split schedule)",
             NEAR_KERNELS["cuda"]: "k_near_groups (near-zone block SpMV on the CUDA cores)"}[nk]
    profl = solver.profile_matvec(20, per_launch, api.PREC_MIXED)
    near_ms = profl["near_kernel_ms"]
    achieved = alg_bytes / (near_ms / 1e3) / 1e9
    traffic = {NEAR_KERNELS["merged"]: profile_traffic(f"near_mma_{args.config}.txt"),
               NEAR_KERNELS["wide"]: profile_traffic(f"near_mma_wide_{args.config}.txt")}.get(nk)
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": traffic, "peak_kind": kind,
            "kernel": f"{kname}, {per_launch} complex64 right-hand sides per launch",
            "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": near_ms,
            "flops_per_launch": Bref * 144 * per_launch * 2}
    if nk == NEAR_KERNELS["wide"]:
        # the 16-wide merged pass that takes the last 16 or fewer right-hand sides
        prof16 = solver.profile_matvec(20, 16, api.PREC_MIXED)
        roof["merged_16"] = {"kernel": "k_near_mma<1> (16 complex64 right-hand sides)",
                             "avg_launch_ms": prof16["near_kernel_ms"],
                             "achieved": round(alg_bytes / (prof16["near_kernel_ms"] / 1e3) / 1e9, 1),
                             "frac": round(alg_bytes / (prof16["near_kernel_ms"] / 1e3) / 1e9 / peak, 4),
                             "traffic": profile_traffic(f"near_mma_{args.config}.txt")}
    # secondary: the FP64 one-right-hand-side near zone of the plain form
    prof1 = solver.profile_matvec(20, 1)
    roof["fp64_one_rhs"] = {"kernel": "k_near_groups (FP64, one right-hand side)", "avg_launch_ms": prof1["near_kernel_ms"],
                            "achieved": round(alg_bytes / (prof1["near_kernel_ms"] / 1e3) / 1e9, 1),
                            "frac": round(alg_bytes / (prof1["near_kernel_ms"] / 1e3) / 1e9 / peak, 4),
                            "traffic": profile_traffic(f"near_groups_{args.config}.txt")}
    # whole pFFT matvec against HBM (algorithmic bytes per right-hand side,
    # four merged convolutions, operator reads shared by the batch)
    roof["matvec"] = matvec_roofline(solver, desc, mesh.n_tet, Bref, peak, prof1["matvec_ms"], profb["matvec_ms"], S)

    serving = None
    if rank == 0 and world == 1 and not args.no_serve:
        try:
            sv = serve_bench(8)
            serving = {k: sv[k] for k in ("value", "unit", "p50_ms", "p99_ms", "completed", "columns",
                                          "peak_running", "busy_s")}
            serving["workload"] = sv["config"]["workload"]
        except Exception as e:
            serving = {"error": str(e)[:200]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(solver, mesh, gs, k, cfg, fp64_iters, fp64_cycles)
        except Exception as e:   # the baseline is reported, never the headline
            cpu = {"value": None, "error": str(e)[:200]}

    if rank == 0:
        lat_s = sorted(lat)
        line = {
            "metric": METRIC,
            "value": round(value, 4), "unit": "columns/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 inner / f64 outer",
            "data": "synthetic (seeded jittered cube-lattice mesh)",
            "config": {"workload": cfg["workload"], "tets": mesh.n_tet,
                       "grid_nodes": [desc.Nx, desc.Ny, desc.Nz], "near_blocks": Bref,
                       "near_bytes": solver.nearzone_bytes(), "columns_per_step": B, "slots": S,
                       "form": "mixed precision, batched columns",
                       "precision": "complex64 inner GMRES(%d) to %g, FP64 outer refinement to %g (near zone "
                                    "stored complex64 as the reference)" % (cfg["inner_m"], cfg["inner_tol"],
                                                                            cfg["tol"]),
                       "l2": "inputs larger than L2 (near-zone tiles %.2f GB per matvec)" % (solver.nearzone_bytes() / 1e9),
                       "near_kernel": args.near_kernel, "gram_schmidt": args.gram_schmidt,
                       "fft_passes": args.fft_passes,
                       "near_split": args.near_split,
                       "fft_lengths": [fft_len(2 * v, FFT_LENGTHS[args.fft_lengths] != 1) for v in (desc.Nx, desc.Ny, desc.Nz)],
                       "parallelism": f"replicas x{world}"},
            "t_rel_err_vs_fp64": t_err,
            "p50_ms": round(float(np.percentile(lat_s, 50)), 3),
            "p99_ms": round(float(np.percentile(lat_s, 99)), 3),
            "iters_mean": float(np.mean(iters)),
            "forms": forms,
            "batched_matvec": batched,
            "serving": serving,
            "e2e": {"value": round(e2e_val, 4), "unit": "columns/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "T_rel_diff_vs_device_region": e2e_vs_device},
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "setup_s": round(setup_s, 2),
            "tuning": tuning,
            "wall_s": round(wall, 2),
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if dist:
        dist.destroy_process_group()


def _serve_stream(nreq, scale, seed=3000):
    """The requests of a served stream: (mesh, k, cell size, Nmax, body) with
    repeats -- nreq requests drawn from nreq // 2 distinct problems, so that
    some arrive while an earlier request of the same operator is resident."""
    from scadyn_b200 import geometry, meshgen
    rng = np.random.default_rng(seed)
    nm_range, ka_range, nmax_cap = ((6.0, 13.0), (1.0, 6.0), 8) if scale == "small" else ((6.0, 22.5), (1.0, 12.0), 16)
    problems = []
    for r in range(max(1, nreq // 2)):
        kind = rng.choice(["sphere", "ellipsoid", "core_mantle"])
        nm = float(rng.uniform(*nm_range))
        if kind == "sphere":
            eps = complex(rng.uniform(1.5, 3.0), rng.uniform(0.01, 0.1))
            mesh = meshgen.sphere(nm, seed=4000 + r, eps=eps)
        elif kind == "ellipsoid":
            ax = (1.0, float(rng.uniform(0.5, 1.0)), float(rng.uniform(0.5, 1.0)))
            eps = complex(rng.uniform(1.5, 3.0), rng.uniform(0.01, 0.1))
            mesh = meshgen.ellipsoid(nm, ax, seed=4000 + r, eps=eps)
        else:
            mesh = meshgen.core_mantle(nm, seed=4000 + r)
        ka = float(rng.uniform(*ka_range))
        nmax = int(np.clip(round(ka + 4 * ka ** (1 / 3) + 2) if scale != "small" else round(ka) + 2, 4, nmax_cap))
        N = int(min(128, max(16, int(round(mesh.n_tet ** (1 / 3) / 2)) * 2)))
        gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, N)
        problems.append((mesh, ka / mesh.a, gs, nmax, str(kind)))
    order = list(range(len(problems))) + list(rng.integers(0, len(problems), size=nreq - len(problems)))
    rng.shuffle(order[len(problems) // 2:])
    return [problems[i] for i in order[:nreq]], [int(i) for i in order[:nreq]], problems


def serve_bench(nreq, scale="small", check_err=False):
    """A served stream shaped like C4: Poisson arrivals (seed 3000) of T-matrix
    requests over seeded meshes -- spheres, ellipsoids with axis ratios
    U(0.5,1), core-mantle spheres (core eps 3.5+0.1i, mantle 1.8+0.01i) --
    mixed precision, under a 150 GB HBM budget.  scale "small": 5k-60k tets,
    ka U(1,6), Nmax 4-8 (minutes, the bench line's summary); "c4": 5k-300k
    tets, ka U(1,12), Nmax from the Wiscombe rule in 4-16.  Requests repeat
    problems (nreq // 2 distinct operators).  The stream runs twice on fresh
    servers: with resident pools shared by requests of one operator, and
    with every request isolated in its own pool (a per-request key), the
    one-context-per-request baseline.  Reports served columns/s (columns of
    completed requests over the time any request was running), request
    latency p50/p99 (submit -> T ready) of both, and with check_err the T
    error of four columns of every distinct problem against a separate FP64
    solve."""
    from scadyn_b200.server import Server
    from scadyn_b200 import api
    reqs, which, problems = _serve_stream(nreq, scale)
    gap_mean = 0.5 if scale == "small" else 4.0
    gaps = np.random.default_rng(3001).exponential(gap_mean, size=len(reqs))
    opts = dict(m=30, cycles=60, block=32, precision=api.PREC_MIXED, inner_tol=3e-4, max_outer=10)

    def run(isolated):
        srv = Server(hbm_budget=150e9)
        ids, t0 = [], time.time()
        for q, ((mesh, k, gs, nmax, kind), gap) in enumerate(zip(reqs, gaps)):
            time.sleep(float(gap))
            tol = 1e-6 * (1 + 1e-12 * q) if isolated else 1e-6      # a per-request key: no sharing
            ids.append(srv.submit(mesh, k, gs, nmax, tol=tol, **opts))
        for i in ids:
            srv.wait(i, 7200)
        wall = time.time() - t0
        st = srv.stats()
        lat = [srv.poll(i)[2] for i in ids]
        Ts = [srv.result(i)[0] for i in ids]
        srv.close()
        return {"value": round(st["columns"] / st["busy_s"], 4), "p50_ms": round(st["p50_ms"], 1),
                "p99_ms": round(st["p99_ms"], 1), "request_latency_ms": [round(v, 1) for v in lat],
                "completed": st["completed"], "columns": st["columns"], "peak_running": st["peak_running"],
                "peak_bytes": st["peak_bytes"], "pools_built": st["pools_built"], "pool_reuses": st["pool_reuses"],
                "busy_s": round(st["busy_s"], 2), "wall_s": round(wall, 2)}, Ts

    shared, Ts = run(False)
    isolated, _ = run(True)
    errs = None
    if check_err:
        errs = []
        for p_idx, (mesh, k, gs, nmax, kind) in enumerate(problems):
            q = which.index(p_idx)
            d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
            s = api.Solver.from_desc(d)
            s.set_wavenumber(k)
            s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
            s.build_G()
            s.pfft_projection_const()
            s.compute_near_zone_interactions_const(api.STORE_C64)
            T64, _ = s.compute_T_matrix(nmax, col0=0, ncol=4, tol=1e-8, m=50, cycles=60, block=4)
            s.close()
            errs.append(float(np.linalg.norm(Ts[q][:, :4] - T64) / np.linalg.norm(T64)))
    line = {"metric": "served T-matrix columns/s and request latency p50/p99 (mixed precision, resident pools)",
            "value": shared["value"], "unit": "columns/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "c64 inner / f64 outer", "data": "synthetic (seeded meshes)",
            "config": {"workload": "C4-shaped served stream (%s): %d requests over %d operators, %s, Poisson arrivals "
                                   "mean gap %.1f s, HBM budget 150 GB"
                                   % (scale, len(reqs), len(problems),
                                      "5k-60k tets, ka U(1,6), Nmax 4-8" if scale == "small" else
                                      "5k-300k tets, ka U(1,12), Nmax 4-16", gap_mean),
                       "tets": [int(m.n_tet) for m, *_ in reqs], "Nmax": [int(r[3]) for r in reqs],
                       "bodies": [r[4] for r in reqs], "problem_of_request": which},
            "p50_ms": shared["p50_ms"], "p99_ms": shared["p99_ms"], "shared": shared,
            "one_pool_per_request": isolated}
    for key in ("completed", "columns", "peak_running", "busy_s"):
        line[key] = shared[key]
    if errs is not None:
        line["t_rel_err_vs_fp64"] = {"max": max(errs), "per_problem": errs, "columns": "4 per problem"}
    return line


def sweep_bench(nw, nmax_cap):
    """C3-shaped wavelength sweep in one batched solve: one ellipsoid mesh
    (1:0.8:0.6, ~60k tets, eps 2.5+0.05i), nw wavelengths taken evenly from
    32 values of ka log-spaced in [1, 10], Nmax from the Wiscombe rule
    ka + 4 ka^(1/3) + 2 clipped to [4, nmax_cap], grid N = 16..64 nodes on the
    longest axis with ka (padded 32^3-128^3), raised to the mesh resolution
    where that is finer.  Every wavelength gets its own context (grid,
    operator); all columns of all wavelengths are slots of one batched solver
    (scd_solve_sweep), mixed precision.  Reports columns/s over the whole
    sweep (device time), set-up separately, and the T error of a sample of
    columns per wavelength against the FP64 form.

    The operators of all wavelengths together can exceed the device: the
    wavelengths are then taken in groups whose operators leave a third of the
    device free for the solve's work buffers, one scd_solve_sweep per group;
    the line reports the groups and the summed device time."""
    import torch
    from scadyn_b200 import api, geometry, meshgen
    mesh = meshgen.ellipsoid(17.1, (1.0, 0.8, 0.6), seed=1003, eps=2.5 + 0.05j)
    kas = np.logspace(0, 1, 32)
    pick = np.unique(np.round(np.linspace(0, 31, nw)).astype(int))
    slots = 64
    opts = dict(tol=1e-6, m=30, cycles=60, block=slots, precision=api.PREC_MIXED, inner_tol=3e-4, max_outer=10)
    torch.cuda.init()

    def build(i):
        ka = float(kas[i])
        nmax = int(np.clip(round(ka + 4 * ka ** (1 / 3) + 2), 4, nmax_cap))
        # grid: the ka rule (16..64), but never coarser than the mesh resolution
        # (about T^(1/3) nodes on the longest axis); coarser boxes would make
        # the near zone dominate
        N = int(np.clip(round((16 + 48 * (ka - 1) / 9) / 2) * 2, 16, 64))
        N = max(N, int(round(0.9 * mesh.n_tet ** (1 / 3) / 2)) * 2)
        gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, N)
        d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
        s = api.Solver.from_desc(d)
        s.set_wavenumber(ka / mesh.a)
        s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
        s.build_G()
        s.pfft_projection_const()
        s.compute_near_zone_interactions_const(api.STORE_C64)
        w = {"ka": round(ka, 3), "Nmax": nmax, "grid_nodes": [d.Nx, d.Ny, d.Nz],
             "columns": 2 * ((nmax + 1) ** 2 - 1)}
        return s, w

    # the solve builds each wavelength's work buffers and tile planes while it
    # has columns in flight (a few wavelengths at a time: columns are taken in
    # wavelength order) and releases them after; keep this much device memory
    # free for them and for the slots' Krylov bases
    reserve = 0.35 * torch.cuda.mem_get_info()[1]
    Ts_all, its_all, st_all, waves, groups = [], [], [], [], []
    setup_s = solve_ms = wall = 0.0
    errs = []
    queue = list(pick)
    carry = None
    while queue or carry:
        ctxs, ws = [], []
        while queue or carry:
            t0 = time.time()
            s, w = carry if carry else build(queue.pop(0))
            carry = None
            setup_s += time.time() - t0
            if ctxs and torch.cuda.mem_get_info()[0] < reserve:
                carry = (s, w)        # solve the group first, keep this operator for the next one
                break
            ctxs.append(s)
            ws.append(w)
        lead = ctxs[0]
        lead.timing(reset=True)
        t = time.time()
        Ts, its, st, rc = api.solve_sweep(ctxs, [w["Nmax"] for w in ws], **opts)
        wall += time.time() - t
        solve_ms += lead.timing(reset=True)["accum_ms"]
        groups.append(len(ctxs))
        # accuracy: four columns of every fourth wavelength in FP64 GMRES(50)
        for wi in range(len(ctxs)):
            if (len(waves) + wi) % 4 == 0:
                T64, _ = ctxs[wi].compute_T_matrix(ws[wi]["Nmax"], col0=0, ncol=4, tol=1e-8, m=50, cycles=40,
                                                   block=4)
                errs.append(float(np.linalg.norm(Ts[wi][:, :4] - T64) / np.linalg.norm(T64)))
        for w, it in zip(ws, its):
            w["iters_mean"] = round(float(np.mean(it)), 1)
        waves += ws
        st_all += [int(v) for v in st]
        for c in ctxs:
            c.close()
    cols = sum(w["columns"] for w in waves)
    return {"metric": "C3-shaped wavelength sweep: T-matrix columns/s over all wavelengths in one batched solve "
                      "(mixed precision)",
            "value": round(cols / (solve_ms / 1e3), 4), "unit": "columns/s", "n_gpus": 1,
            "higher_is_better": True, "dtype": "c64 inner / f64 outer", "data": "synthetic (seeded mesh)",
            "config": {"workload": "ellipsoid 1:0.8:0.6, %d tets, eps 2.5+0.05i, %d of 32 log-spaced ka in [1,10], "
                                   "Nmax Wiscombe clipped to [4,%d], N 16-64, scd_solve_sweep over groups that fit "
                                   "the device, %d slots" % (mesh.n_tet, len(pick), nmax_cap, slots)},
            "wavelengths": waves, "columns": cols, "groups": groups, "solve_ms": round(solve_ms, 1),
            "wall_s": round(wall, 2), "setup_s": round(setup_s, 2), "status": st_all,
            "t_rel_err_vs_fp64_sample": {"max": max(errs), "columns": "4 per wavelength, every 4th wavelength"}}


def fft_len(v, smooth):
    """Padded FFT length the library picks for 2N = v (power of two, or the
    shorter of 80, 96, 192 with 5-smooth lengths enabled)."""
    p2 = 8
    while p2 < v:
        p2 *= 2
    if smooth:
        for p in (80, 96, 192):
            if v <= p < p2:
                return p
    return p2


def matvec_roofline(solver, desc, T, Bref, peak, ms1, msb, nb):
    """Algorithmic HBM bytes of one pFFT matvec per right-hand side (read x,
    write Ax; four merged convolutions over the pruned grid, each spectrum
    written and read twice; projectors, index-free box nodes, Green octant and
    near-zone blocks read once per call and shared by the nb right-hand sides
    of a batch) against the measured matvec time."""
    n = 3 * T
    Nx, Ny, Nz = desc.Nx, desc.Ny, desc.Nz
    K = 4

    def bytes_per_rhs(c, cs, cf, b):
        own = 2 * n * c + K * 16 * Nx * Ny * Nz * c
        shared = 4 * 27 * T * cs + K * (Nx + 1) * (Ny + 1) * (Nz + 1) * cf + Bref * (9 * 8 + 8)
        return own + shared / b

    b1 = bytes_per_rhs(16, 16, 16, 1)
    bb = bytes_per_rhs(8, 8, 8, nb)
    a1 = b1 / (ms1 / 1e3) / 1e9
    ab = bb / (msb / nb / 1e3) / 1e9
    return {"fp64_one_rhs": {"alg_bytes": int(b1), "ms": round(ms1, 4), "achieved": round(a1, 1),
                             "frac": round(a1 / peak, 4)},
            "complex64_batched": {"nrhs": nb, "alg_bytes_per_rhs": int(bb), "ms_per_rhs": round(msb / nb, 4),
                                  "achieved": round(ab, 1), "frac": round(ab / peak, 4)}}


if __name__ == "__main__":
    main()
