"""Batch width, autotuner cache and concurrent scene batches."""
import json

import numpy as np
import pytest

from ultrasound_solver_b200 import autotune


def test_autotune_cache_roundtrip(tmp_path):
    """The cache is read back and reused without measuring (no GPU needed)."""
    path = tmp_path / "tune.json"
    key = autotune.cache_key("B200", (64, 48, 40), "bf16", 40, 10, False)
    assert key == "B200|64x48x40|bf16|m40|k10|fwd"
    path.write_text(json.dumps({key: {"batch_width": 8}}))
    t = autotune.BatchTuner(cache_path=path)
    assert t.cache[key]["batch_width"] == 8
    t.cache["x"] = {"batch_width": 2}
    t._save()
    assert json.loads(path.read_text())["x"]["batch_width"] == 2


def test_config2_scene_batch_is_seeded_and_fits():
    from ultrasound_solver_b200 import workloads as W
    a = W.config2_scene_batch(count=6, seed=3)
    b = W.config2_scene_batch(count=6, seed=3)
    assert a == b
    for cfg in a:
        n = cfg["domain"]["grid_size"][0]
        assert n in (48, 64, 80, 96, 112)
        ob = cfg["obstacles"][0]
        L = cfg["domain"]["box_size"][0]
        pml = 10e-3
        assert all(pml + ob["radius"] < c < L - pml - ob["radius"] for c in ob["center"])
    basis = W.config2_basis_scene()
    assert basis["transducer_specs"]["array_n"] == 16


@pytest.mark.gpu
def test_batch_width_split_matches_single_launch(golden):
    from tests.helpers import golden_solver, rel
    s = golden_solver(golden, precision="mixed", gmres_rtol=1e-10, gmres_maxiter=20000)
    rhs = s.sources.column_rhs(s.transducers.amplitudes)
    x_all = s.solve_rhs_device(rhs).cpu().numpy()
    s.iterative_solver.batch_width = 2
    x_split = s.solve_rhs_device(rhs).cpu().numpy()
    assert len(s.iterative_solver.last_stats) == rhs.shape[0]
    for k in range(rhs.shape[0]):
        assert rel(x_split[k], x_all[k]) <= 1e-6


@pytest.mark.gpu
def test_batch_tuner_picks_a_feasible_width(golden, tmp_path):
    from tests.helpers import golden_solver
    s = golden_solver(golden, precision="bf16", gmres_rtol=1e-10, gmres_maxiter=20000,
                      gmres_recycle=8)
    rhs = s.sources.column_rhs(s.transducers.amplitudes)
    t = autotune.BatchTuner(cache_path=tmp_path / "t.json", candidates=(1, 2, 4), cycles=1)
    w = t.tune(s.iterative_solver, s.operator, rhs)
    assert w in (1, 2, 4) and s.iterative_solver.batch_width == w
    assert set(t.last_timings) <= {1, 2, 4} and all(v > 0 for v in t.last_timings.values())
    # the Arnoldi kernel forms were timed too and the fastest one is set
    entry = next(iter(t.cache.values()))
    assert set(entry["seconds_per_rhs_iteration_by_variant"]) == {"0", "1", "2"}
    assert s.iterative_solver.kernel_variant == entry["kernel_variant"]
    # cached: a second tuner reads the width and form without measuring
    t2 = autotune.BatchTuner(cache_path=tmp_path / "t.json")
    s.iterative_solver.batch_width = 0
    s.iterative_solver.kernel_variant = 0
    assert t2.tune(s.iterative_solver, s.operator, rhs) == w and t2.last_timings == {}
    assert s.iterative_solver.kernel_variant == entry["kernel_variant"]
    # solving with the tuned width still reaches the direct solution
    from tests.helpers import rel
    x = s.solve_rhs_device(rhs).cpu().numpy()
    for k in range(rhs.shape[0]):
        assert rel(x[k], golden["G"][:, k]) <= 1e-6


@pytest.mark.gpu
def test_concurrent_scenes_match_sequential():
    """Golden scenes of different shapes solved concurrently give their own solutions."""
    from tests.conftest import load_golden
    from tests.helpers import golden_solver, rel
    from ultrasound_solver_b200.scene_batch import solve_scenes
    gs = [load_golden(n) for n in ("mixed", "air_pml", "fields")]
    solvers = [golden_solver(g, precision="bf16", gmres_rtol=1e-10, gmres_maxiter=20000,
                             gmres_recycle=8) for g in gs]
    rhs = [s.update_rhs_device() for s in solvers]
    xs = solve_scenes(solvers, rhs)
    for g, x in zip(gs, xs):
        want = g["x_direct"]
        assert rel(x.cpu().numpy(), want) <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("nrhs", [3, 4, 9])
def test_mixed_apply_on_an_uneven_grid(nrhs):
    """Complex64 K on a grid whose x edge is not a multiple of the 32-node warp
    span (an uneven-batch scene) matches the FP64 rows per column."""
    import torch
    from tests.helpers import rel
    from ultrasound_solver_b200 import _native as N
    from ultrasound_solver_b200 import workloads as W
    cfg = W.config2_scene_batch(count=1, seed=5, sizes=(48, 80, 112))[0]
    s = W.build_solver(cfg, seed=0)
    s.assemble_matrix()
    op = s.operator
    assert op.shape[0] % 32 != 0 or op.shape[1] % 8 != 0
    rng = np.random.default_rng(nrhs)
    x = torch.from_numpy(rng.standard_normal((nrhs, op.n)) + 1j * rng.standard_normal((nrhs, op.n)))
    x = x.cuda()
    for var in (N.APPLY_K, N.APPLY_KH):
        got = op.apply(x.to(torch.complex64), var, N.PREC_MIXED).cpu().numpy()
        want = op.apply(x, var, N.PREC_FP64).cpu().numpy()
        for b in range(nrhs):
            assert rel(got[b], want[b]) < 2e-6


@pytest.mark.gpu
def test_stencil_tuner_picks_a_kernel(golden, tmp_path):
    """StencilTuner times both complex64 stencil kernels for a batch width,
    caches the faster one, and the operator then applies with it (same rows
    as the FP64 operator)."""
    import numpy as np
    import torch
    from tests.helpers import golden_solver, rel
    from ultrasound_solver_b200 import _native as N
    s = golden_solver(golden)
    op = s.operator
    t = autotune.StencilTuner(cache_path=tmp_path / "s.json", reps=3)
    k = t.tune(op, 4)
    assert k in (N.STENCIL_COEF_ROWS, N.STENCIL_RECORD_TILES) and op.stencil_kernel == k
    assert set(t.last_timings) == {N.STENCIL_COEF_ROWS, N.STENCIL_RECORD_TILES}
    op.stencil_kernel = N.STENCIL_AUTO
    assert autotune.StencilTuner(cache_path=tmp_path / "s.json").tune(op, 4) == k
    rng = np.random.default_rng(4)
    x = torch.from_numpy(rng.standard_normal((4, op.n)) + 1j * rng.standard_normal((4, op.n))).cuda()
    got = op.apply(x.to(torch.complex64), N.APPLY_K, N.PREC_MIXED).cpu().numpy()
    want = op.apply(x, N.APPLY_K, N.PREC_FP64).cpu().numpy()
    for b in range(4):
        assert rel(got[b], want[b]) < 2e-6
