"""The autotuner of sweeps per level, bottom sweeps and level count
(mg_tune): every candidate it times is a valid multigrid configuration whose
solve converges and matches the float32 oracle run with the same parameters
(iterations +-1, pressure within 1e-5), and it returns the fastest."""
import numpy as np
import pytest

import mg_scenes
from helpers import oracle_for, rel_l2

pytestmark = pytest.mark.gpu


def _gpu_solve(sc, L, pp, bot):
    import torch
    from mgpcg import MGPCGPoissonSolver
    dev = torch.device("cuda")
    s = MGPCGPoissonSolver(sc.dim, sc.res, L, pp, bot, device=dev)
    s.pressure_solve_async(torch.from_numpy(sc.cell_type).to(dev), [torch.from_numpy(v).to(dev) for v in sc.velocity],
                           torch.from_numpy(sc.phi).to(dev), sc.p0, sc.scale_A, sc.scale_b, True, sc.gfm_clamp)
    st = s.stats()
    return st, s.x.cpu().numpy()


@pytest.mark.parametrize("make", [lambda: mg_scenes.instance_scene(2, 128, 17, levels=4),
                                  lambda: mg_scenes.instance_scene(3, 48, 18, levels=3)])
def test_tuner_candidates_converge_and_match_oracle(make):
    import mg_tune
    sc = make()
    r = mg_tune.tune(sc, "f32", sweeps=(1, 2, 3), bottoms=(10, 50), reps=1)
    assert r["candidates"] and all(c["converged"] for c in r["candidates"])
    best = min(r["candidates"], key=lambda c: c["ms"])
    assert (r["levels"], r["pre_post"], r["bottom"]) == (best["levels"], best["pre_post"], best["bottom"])
    for c in r["candidates"]:
        st, x = _gpu_solve(sc, c["levels"], c["pre_post"], c["bottom"])
        assert st.status == 0
        o = oracle_for(sc, levels=c["levels"], pre_post=c["pre_post"], bottom=c["bottom"])
        it_o = o.solve(500)
        assert abs(st.iters - it_o) <= 1, (c, st.iters, it_o)
        assert rel_l2(x, o.get("x")) < 1e-5, c


def test_tune_classes_gives_valid_parameters_per_scene():
    import mg_tune
    params = mg_scenes.batch_scene_params(seed=3, n2d=4, n3d=3)
    scenes = [mg_scenes.instance_scene(d, s, ss, levels=mg_tune.rule_levels(d, s)) for d, s, ss in params]
    per_scene, classes = mg_tune.tune_classes(scenes, "f32", sweeps=(1, 2), bottoms=(10, 50), reps=1)
    assert len(per_scene) == len(scenes)
    for sc, (L, pp, bot) in zip(scenes, per_scene):
        assert L in mg_tune.level_choices(sc.res)
        assert pp in (1, 2) and bot in (10, 50)
    from mg_batch import BatchSolver
    b = BatchSolver(scenes, params=per_scene, streams=4)
    _, stats = b.solve()
    assert all(st.status == 0 for st in stats)
