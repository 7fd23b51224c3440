"""The autotuner's host logic on the CPU: the level-count rule and its
candidates, the size classes, and how one class's measured choice spreads to
every scene of the class (the timing itself, `tune`, is replaced by a stub
that returns a fixed winner per class)."""
import types

import pytest

import mg_tune


def test_rule_levels_bring_the_coarsest_grid_to_8_to_16_cells():
    for dim, side in ((2, 64), (2, 128), (2, 512), (3, 32), (3, 128), (3, 160)):
        L = mg_tune.rule_levels(dim, side)
        coarsest = side >> (L - 1)
        assert side % (1 << (L - 1)) == 0 and 8 <= coarsest <= 16, (side, L)
    assert mg_tune.rule_levels(2, 128) == 5 and mg_tune.rule_levels(3, 256) == 6


@pytest.mark.parametrize("res", [(128, 128), (64, 64, 64), (96, 96, 96), (160, 160, 160), (256, 128)])
def test_level_choices_halve_evenly_to_at_least_4_cells(res):
    choices = mg_tune.level_choices(res)
    L0 = mg_tune.rule_levels(len(res), min(res))
    assert L0 in choices and set(choices) <= {L0 - 1, L0, L0 + 1}
    for L in choices:
        assert L >= 2
        assert all(n % (1 << (L - 1)) == 0 and (n >> (L - 1)) >= 4 for n in res), (res, L)


def test_size_classes_cover_the_batch_range():
    assert mg_tune.size_class(2, 64) == mg_tune.size_class(2, 128) == (2, 0)
    assert mg_tune.size_class(2, 160) == mg_tune.size_class(2, 288) == (2, 1)
    assert mg_tune.size_class(2, 512) == (2, 2)
    assert mg_tune.size_class(3, 32) == (3, 0) and mg_tune.size_class(3, 96) == (3, 1)
    assert mg_tune.size_class(3, 160) == (3, 2)


def _scene(dim, side):
    return types.SimpleNamespace(dim=dim, res=(side,) * dim, cells=side ** dim, name=f"{dim}d_{side}")


def test_tune_classes_tunes_the_largest_scene_of_each_class(monkeypatch):
    tuned = []

    def fake_tune(scene, storage="f32", device=None, **kw):
        tuned.append(scene.name)
        # class winner: one level fewer than the rule, 1 sweep, 10 bottom sweeps
        return {"levels": mg_tune.rule_levels(scene.dim, min(scene.res)) - 1, "pre_post": 1, "bottom": 10,
                "ms": 1.0, "iters": 5, "candidates": []}

    monkeypatch.setattr(mg_tune, "tune", fake_tune)
    scenes = [_scene(2, 64), _scene(2, 128), _scene(2, 256), _scene(3, 32), _scene(3, 64)]
    per_scene, results = mg_tune.tune_classes(scenes)
    assert sorted(tuned) == sorted(["2d_128", "2d_256", "3d_64"])   # one run per class, its largest scene
    assert set(results) == {(2, 0), (2, 1), (3, 0)}
    for sc, (L, pp, bot) in zip(scenes, per_scene):
        assert (pp, bot) == (1, 10)
        assert L == mg_tune.rule_levels(sc.dim, sc.res[0]) - 1         # the class's offset from the rule
        assert L in mg_tune.level_choices(sc.res)


def test_class_params_fall_back_to_the_rule_for_untuned_classes():
    results = {(2, 0): {"offset": 1, "pre_post": 3, "bottom": 20}}
    params = mg_tune.class_params(results)
    assert params(2, 128) == (mg_tune.rule_levels(2, 128) + 1, 3, 20)
    assert params(3, 64) == (mg_tune.rule_levels(3, 64), 2, 50)
