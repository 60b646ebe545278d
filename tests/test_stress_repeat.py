"""Run-to-run determinism of the batched matvec: every kernel of the pFFT
matvec (anterpolation, the FFT passes with the Green product, interpolation,
the near-zone sums on CUDA cores or tensor cores) forms each output from the
same terms in a fixed order, so repeating a matvec on the same inputs gives
the same bits.  scd_check_matvec_repeat compares repetitions with the first
one on the device; a differing bit in any repetition is a race between the
threads or CTAs of a kernel.  Every kernel choice of the autotuner is checked
at the column counts the batched solver uses (1, 16, 32 and 40 complex64
columns: the 40 take one 32-wide and one 16-wide tensor-core pass), and the
FP64 matvec of the refinement at 1 and 4 columns."""
import pytest

from scadyn_b200 import api, geometry, meshgen

pytestmark = pytest.mark.gpu

REPS = 40


@pytest.fixture(scope="module")
def solver():
    mesh = meshgen.lattice_body(12.0, (1.0, 0.8, 0.6), seed=1002, eps=2.5 + 0.05j)
    gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, 32)
    d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=gs)
    s = api.Solver.from_desc(d)
    s.set_wavenumber(4.0 / mesh.a)
    s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
    s.build_G()
    s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C64)
    yield s
    s.close()


def _apply(s, nrhs, precision, near_kernel, fft_passes, scatter_span=0, gather_span=0):
    s.apply_tuning(dict(nrhs=nrhs, precision=precision, near_kernel=near_kernel, fft_passes=fft_passes,
                        scatter_span=scatter_span, gather_span=gather_span))


@pytest.mark.parametrize("near_kernel", [api.NEAR_CUDA_CORES, api.NEAR_TENSOR_SPLIT, api.NEAR_TENSOR_MERGED,
                                         api.NEAR_TENSOR_WIDE], ids=["cuda", "split", "merged", "wide"])
@pytest.mark.parametrize("fft_passes", [api.FFT_PASSES_FUSED_YZ, api.FFT_PASSES_THREE], ids=["yz", "three"])
def test_complex64_matvec_repeats_bit_for_bit(solver, near_kernel, fft_passes):
    for nrhs in (1, 16, 32, 40):
        _apply(solver, nrhs, api.PREC_MIXED, near_kernel, fft_passes)
        bad, words = solver.check_matvec_repeat(REPS, nrhs, api.PREC_MIXED)
        assert (bad, words) == (0, 0), f"{nrhs} columns: {bad} of {REPS} repetitions differ ({words} words)"


@pytest.mark.parametrize("spans", [(8, 4), (16, 16)], ids=["8-4", "16-16"])
def test_complex64_matvec_repeats_with_spans(solver, spans):
    _apply(solver, 32, api.PREC_MIXED, api.NEAR_TENSOR_WIDE, api.FFT_PASSES_FUSED_YZ, *spans)
    bad, words = solver.check_matvec_repeat(REPS, 32, api.PREC_MIXED)
    assert (bad, words) == (0, 0)


@pytest.mark.parametrize("fft_passes", [api.FFT_PASSES_FUSED_YZ, api.FFT_PASSES_THREE], ids=["yz", "three"])
def test_fp64_matvec_repeats_bit_for_bit(solver, fft_passes):
    for nrhs in (1, 4):
        _apply(solver, nrhs, api.PREC_FP64, api.NEAR_DEFAULT, fft_passes)
        bad, words = solver.check_matvec_repeat(REPS, nrhs, api.PREC_FP64)
        assert (bad, words) == (0, 0), f"{nrhs} columns: {bad} of {REPS} repetitions differ ({words} words)"


def test_repeat_check_refuses_bad_arguments(solver):
    with pytest.raises(api.ScadynError) as e:
        solver.check_matvec_repeat(4, 1, 7)
    assert e.value.code == api.SCD_BAD_ARG
