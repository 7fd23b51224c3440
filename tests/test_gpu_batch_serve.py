"""Batched and served solves: every result is the same alone and in the mix.

A batch enqueues many instances' solves on a pool of streams; the server also
warm-starts each substep from the session's previous pressure.  Each
instance's computation is independent and deterministic, so its result in the
mix must equal its result alone BIT FOR BIT (the stated tolerance is 0).
"""
import numpy as np
import pytest
import torch

import mg_scenes

pytestmark = pytest.mark.gpu


def _small_batch_scenes():
    params = [(2, 64, 11), (2, 96, 12), (3, 32, 13), (2, 128, 14), (3, 48, 15), (3, 32, 16)]
    return [mg_scenes.instance_scene(d, s, seed, levels=3) for d, s, seed in params]


@pytest.mark.parametrize("storage", ["f32", "f16"])
def test_batch_equals_alone(storage):
    from mg_batch import BatchSolver
    scenes = _small_batch_scenes()
    batch = BatchSolver(scenes, storage=storage, streams=4)
    ms, stats = batch.solve()
    assert all(st.status == 0 for st in stats), [st.status for st in stats]
    xs = [inst.solver.x.clone() for inst in batch.instances]
    its = [st.iters for st in stats]
    # each instance alone, through the blocking drop-in API
    for inst, x, it in zip(batch.instances, xs, its):
        it_alone = inst.solve_blocking(500, 1e-12)
        assert it_alone == it
        assert torch.equal(inst.solver.x, x)


def test_batch_plain_matches_oracle():
    """Every instance of the 96-scene uneven batch (64 2D sides 64..512, 32 3D
    sides 32..160, level counts as the batch bench uses them), solved in one
    batch both ways (each instance's graph on a pool of streams, and the
    batched kernels with one launch per stage for all instances), against the
    float32 oracle: iterations +-1, pressure within 1e-5."""
    from helpers import oracle_for, rel_l2
    from mg_batch import BatchSolver
    from mg_serve import levels_for
    params = mg_scenes.batch_scene_params(seed=3)
    scenes = [mg_scenes.instance_scene(d, s, ss, levels=levels_for(d, s)) for d, s, ss in params]
    assert len(scenes) == 96
    batch = BatchSolver(scenes, storage="f32", streams=32)
    _, stats = batch.solve()
    xs = [inst.solver.x.cpu().numpy() for inst in batch.instances]
    _, stats_b = batch.solve_batched()
    xb = [inst.solver.x.cpu().numpy() for inst in batch.instances]
    worst = 0.0
    for inst, st, stb, x, x2 in zip(batch.instances, stats, stats_b, xs, xb):
        assert st.status == 0 and stb.status == 0, (inst.scene.name, st.status, stb.status)
        o = oracle_for(inst.scene)
        it_o = o.solve(500)
        for it, xx in ((st.iters, x), (stb.iters, x2)):
            assert abs(it - it_o) <= 1, (inst.scene.name, it, it_o)
            e = rel_l2(xx, o.get("x"))
            assert e < 1e-5, (inst.scene.name, e)
            worst = max(worst, e)
    print(f"96-instance batch vs oracle: worst rel L2 {worst:.2e}")


@pytest.mark.parametrize("storage", ["f32", "f16", "bf16"])
def test_batched_kernels_match_alone(storage):
    """The batched kernels (tables of blocks, one launch per stage for every
    instance, one graph) give each instance the solve it gets alone: the same
    V-cycle arithmetic and reduction blocks, the z.r sum in its own kernel
    rather than inside the level-0 sweep (so the FP64 sums may part by an
    ulp): iterations +-1 and x within 1e-5.  Repeated and warm-started batch
    solves converge too."""
    from helpers import rel_l2
    from mg_batch import BatchSolver
    scenes = _small_batch_scenes()
    batch = BatchSolver(scenes, storage=storage, streams=4)
    _, stats = batch.solve_batched()
    assert all(st.status == 0 for st in stats), [st.status for st in stats]
    xs = [inst.solver.x.clone() for inst in batch.instances]
    its = [st.iters for st in stats]
    batch.solve_batched(groups=1)
    pro, body = batch.batch_launch_counts()
    assert body < 4 * len(scenes)  # one launch per stage, not per instance
    _, one = batch.solve_batched(groups=1)  # one graph for all: the same solves
    assert [st.iters for st in one] == its
    for inst, x in zip(batch.instances, xs):
        assert torch.equal(inst.solver.x, x)
    _, again = batch.solve_batched()
    assert [st.iters for st in again] == its
    for inst, x in zip(batch.instances, xs):
        assert torch.equal(inst.solver.x, x)
    _, warm = batch.solve_batched(warm_start=True)
    assert all(st.status == 0 and st.iters <= 2 for st in warm), [(st.status, st.iters) for st in warm]
    for inst, x, it in zip(batch.instances, xs, its):
        it_alone = inst.solve_blocking(500, 1e-12)
        assert abs(it_alone - it) <= 1, (inst.scene.name, it_alone, it)
        assert rel_l2(inst.solver.x.cpu().numpy(), x.cpu().numpy()) < 1e-5, inst.scene.name


def _specs(n=6, substeps=4):
    return mg_scenes.serving_sessions(seed=4, n_sessions=n, substeps=substeps, rate_hz=1e4)


def test_served_results_equal_alone():
    """Each (session, substep) result in the served mix equals the same
    session solved alone with the same warm starts."""
    from mg_serve import SolveServer, DeviceScene, levels_for
    from mgpcg import MGPCGPoissonSolver
    specs = _specs(8, 4)
    assert any(s["dim"] == 2 and s["side"] > 160 for s in specs)
    got = {}
    srv = SolveServer(storage="f16", streams=4)
    recs, wall = srv.run(specs, on_complete=lambda sid, step, solver: got.__setitem__((sid, step), solver.x.clone()))
    assert len(recs) == sum(s["substeps"] for s in specs)
    assert all(r["status"] == "converged" for r in recs)
    ordered = sorted(specs, key=lambda s: s["t_arrive"])
    for sid, spec in enumerate(ordered):
        dev = torch.device("cuda")
        sc = DeviceScene(spec, dev)
        L = levels_for(spec["dim"], spec["side"])
        solver = MGPCGPoissonSolver(spec["dim"], sc.res, L, 2, 50, storage="f16", device=dev)
        for step in range(spec["substeps"]):
            sc.build(step)
            solver.pressure_solve_async(sc.ct, sc.vel, sc.phi, sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp,
                                        warm_start=step > 0)
            solver.stats()
            assert torch.equal(solver.x, got[(sid, step)]), (sid, step)


def test_warm_start_saves_iterations():
    from mg_serve import SolveServer
    specs = _specs(4, 5)
    srv = SolveServer(storage="f32", streams=4)
    warm, _ = srv.run(specs, warm_start=True)
    cold, _ = srv.run(specs, warm_start=False)
    later = lambda recs: sum(r["iters"] for r in recs if r["step"] > 0)
    assert later(warm) < later(cold)


def test_admission_respects_hbm_budget():
    from mg_serve import SolveServer, levels_for, plan_bytes
    specs = _specs(6, 2)
    biggest = max(plan_bytes(s["dim"], (s["side"],) * s["dim"], levels_for(s["dim"], s["side"]), "f16")
                  for s in specs)
    srv = SolveServer(storage="f16", streams=4, hbm_budget=2.2 * biggest)
    recs, _ = srv.run(specs)
    assert len(recs) == 12 and all(r["status"] == "converged" for r in recs)
    assert srv.peak_in_use <= 2.2 * biggest
    # pooled idle workspaces count too: what is resident never passes the budget
    assert srv.peak_resident <= 2.2 * biggest
    assert srv.in_use == 0
