"""The cluster-resident V-cycle (the levels from the first brick level down in
one launch of one thread-block cluster, each CTA's bricks in shared memory)
against the streamed V-cycle and the oracle: z of one V-cycle BIT-EXACT, and
the solve BIT-EXACT (x and iteration count) where level 0 stays streamed, on
cubic and non-cubic grids, with the brick levels starting at level 0, 1 and 2
below streamed levels."""
import numpy as np
import pytest

import mg_scenes
from helpers import box_3d as _box
from helpers import gpu_for, oracle_for, rel_l2, small_3d

pytestmark = pytest.mark.gpu


# scene, first level that allows bricks (-1: none)
SCENES = {
    "drop3d_32": lambda: (small_3d(32, levels=3), 0),
    "drop3d_48": lambda: (small_3d(48, levels=4), -1),
    "drop3d_64": lambda: (small_3d(64, levels=4), 0),
    "drop3d_128": lambda: (small_3d(128, levels=5), 1),
    "box_96x64x128": lambda: (_box((96, 64, 128), 4), 1),
    "box_128x128x256": lambda: (_box((128, 128, 256), 5), 2),
}
BRICKED = [k for k in SCENES if k != "drop3d_48"]


def _np(t):
    return t.detach().float().cpu().numpy()


def _brick_levels(g, lp_min):
    """Every level the cluster can start at (forced one by one)."""
    from mg_lib import MGError
    out = []
    for lp in range(lp_min, g.n_mg_levels - 1):
        try:
            on, first = g.resident(True, first_level=lp)
        except MGError:
            continue
        assert on and first == lp
        out.append(lp)
    return out


def test_first_brick_level():
    from mg_lib import MGError
    for name, make in SCENES.items():
        if name.startswith("box_128"):
            continue  # the largest scene is set up by the tests below
        sc, lp = make()
        g, _ = gpu_for(sc)
        on, first = g.resident()
        if lp < 0:
            assert (on, first) == (False, -1), name
            with pytest.raises(MGError):
                g.resident(True)
            continue
        assert first >= lp, name
        assert g.resident(True, first_level=lp) == (True, lp)
        if lp > 0:
            with pytest.raises(MGError):
                g.resident(True, first_level=lp - 1)


@pytest.mark.parametrize("name", BRICKED)
def test_resident_v_cycle_bit_exact(name):
    import torch
    sc, lp = SCENES[name]()
    g, _ = gpu_for(sc)
    g.r[0].copy_(g.b)
    g.resident(False)
    g.v_cycle()
    z_streamed = _np(g.z[0])
    levels = _brick_levels(g, lp)
    assert levels and levels[0] == lp
    for first in levels:
        g.z[0].fill_(7.0)
        g.resident(True, first_level=first)
        g.v_cycle()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(_np(g.z[0]), z_streamed, err_msg=f"cluster from level {first}")
    if max(sc.res) <= 64:
        o = oracle_for(sc)
        o.set("r", o.get("b"), 0)
        o.v_cycle()
        np.testing.assert_array_equal(z_streamed, o.get("z", 0))


@pytest.mark.parametrize("name", BRICKED)
def test_resident_solve_bit_exact(name):
    import torch
    sc, lp = SCENES[name]()
    g, st = gpu_for(sc)
    ct = torch.from_numpy(sc.cell_type).to(g.x.device)
    levels = _brick_levels(g, lp)
    g.reinitialize(ct, st)
    g.resident(False)
    it0 = g.solve(500)
    x0 = _np(g.x)
    for first in sorted({levels[0], levels[-1]}):
        # a fresh system: solve() starts from x, p and beta as the last solve
        # left them (mgpcg.py:150-209), reinitialize() clears them
        g.reinitialize(ct, st)
        g.resident(True, first_level=first)
        it1 = g.solve(500)
        assert g.last_status == "converged"
        if first > 0:  # level 0 streamed in both: the same kernels and sums
            assert it1 == it0
            np.testing.assert_array_equal(_np(g.x), x0)
        else:
            # level 0 inside the cluster: z.r is summed by k_zr4 instead of
            # inside the level-0 sweep, so the FP64 sum may differ in its last
            # bits (the V-cycle itself is bit-exact, above)
            assert abs(it1 - it0) <= 1
            assert rel_l2(_np(g.x), x0) < 1e-6


def test_resident_stage_and_pcg_counts():
    sc, _ = SCENES["drop3d_64"]()
    g, _ = gpu_for(sc)
    g.resident(True)
    g.r[0].copy_(g.b)
    g.launch_stage(6)
    p, b = g.launch_counts()
    g.resident(False)
    p2, b2 = g.launch_counts()
    assert b < b2  # one launch replaces the lower levels' kernels and the coarse block


def test_no_bricks_in_2d():
    sc = mg_scenes.dam_break_2d(n=64, levels=3)
    g, _ = gpu_for(sc)
    assert g.resident() == (False, -1)
    from mg_lib import MGError
    with pytest.raises(MGError):
        g.resident(True)


@pytest.mark.parametrize("n,levels", [(32, 4), (64, 5)])
def test_hierarchy_down_to_4_cells(n, levels):
    """A 3D hierarchy whose coarsest grid is 4^3 (the coarse block then holds
    several levels): every V-cycle the autotuner may choose (streamed or the
    cluster from a start level no deeper than the coarse block's first level)
    launches, and the solve matches the oracle."""
    sc = small_3d(n, levels=levels)
    g, _ = gpu_for(sc)
    it = g.solve(500)
    assert g.last_status == "converged"
    o = oracle_for(sc)
    it_o = o.solve(500)
    assert abs(it - it_o) <= 1
    assert rel_l2(g.x.cpu().numpy(), o.get("x")) < 1e-5
