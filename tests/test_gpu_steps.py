"""Launch shapes of the streamed level sweep that the autotuner chooses:
planes per pipeline step (one or the tile's two, per level and direction) and
the grid (blocks per SM the grid is sized for, per level).  Only the shared-
memory ring, the step loop, the prefetch and the chunks of planes per block
change, not the arithmetic.  z of one V-cycle is BIT-EXACT for every forced
choice; the solve is BIT-EXACT across planes per step and within tolerance
across grids (z.r is summed per block inside the level-0 sweep, so the FP64
sum follows the block count); 1, 2 and 3 smoothing sweeps, float32 and
float16 storage."""
import numpy as np
import pytest

import mg_scenes
from helpers import box_3d, gpu_for, rel_l2, small_3d

pytestmark = pytest.mark.gpu

# both have a level-0 chunk of more than 2 planes (a pipelined sweep)
SCENES = {
    "drop3d_128": lambda: small_3d(128, levels=5),
    "box_96x64x128": lambda: box_3d((96, 64, 128), 4),
}


def _np(t):
    return t.detach().float().cpu().numpy()


@pytest.mark.parametrize("name,pre_post", [("drop3d_128", 2), ("box_96x64x128", 1),
                                           ("box_96x64x128", 2), ("box_96x64x128", 3)])
def test_one_plane_steps_bit_exact(name, pre_post):
    import torch
    sc = SCENES[name]()
    g, st = gpu_for(sc, pre_post=pre_post)
    ct = torch.from_numpy(sc.cell_type).to(g.x.device)
    _, streamed = g.split_levels()
    tuned = g.step_planes()
    assert streamed >= 1 and tuned >> (2 * streamed) == 0
    out = []
    for bits in (0, (1 << (2 * streamed)) - 1, tuned):
        # reinitialize() prepares the plan again (re-applying the tuned
        # choice), so the forced bits are set after it
        g.reinitialize(ct, st)
        assert g.step_planes(bits) == bits
        g.r[0].copy_(g.b)
        g.z[0].fill_(7.0)
        g.v_cycle()
        z = _np(g.z[0])
        g.reinitialize(ct, st)
        g.step_planes(bits)
        it = g.solve(500)
        assert g.last_status == "converged"
        torch.cuda.synchronize()
        out.append((bits, z, it, _np(g.x)))
    _, z0, it0, x0 = out[0]
    for bits, z, it, x in out[1:]:
        np.testing.assert_array_equal(z, z0, err_msg=f"V-cycle, step bits {bits:#x}")
        assert it == it0, bits
        np.testing.assert_array_equal(x, x0, err_msg=f"solve, step bits {bits:#x}")


def test_step_bits_checked():
    from mg_lib import MGError
    g, _ = gpu_for(small_3d(32, levels=3))
    _, streamed = g.split_levels()
    with pytest.raises(MGError):
        g.step_planes(1 << (2 * streamed))  # beyond the streamed levels
    g2, _ = gpu_for(mg_scenes.dam_break_2d(n=64, levels=3))
    assert g2.step_planes() == 0
    with pytest.raises(MGError):
        g2.step_planes(1)  # 2D sweeps keep their tile


@pytest.mark.parametrize("name,pre_post,storage", [("drop3d_128", 2, None), ("box_96x64x128", 1, None),
                                                   ("box_96x64x128", 3, None), ("drop3d_128", 2, "f16")])
def test_grid_choices(name, pre_post, storage):
    import torch
    sc = SCENES[name]()
    g, st = gpu_for(sc, pre_post=pre_post, storage=storage)
    ct = torch.from_numpy(sc.cell_type).to(g.x.device)
    _, streamed = g.split_levels()
    tuned = g.grid_extra()
    assert tuned >> (2 * streamed) == 0
    every = sum(1 << (2 * l) for l in range(streamed))
    out = []
    for bits in (0, every, 2 * every, 3 * every, tuned):
        g.reinitialize(ct, st)
        assert g.grid_extra(bits) == bits
        g.r[0].copy_(g.b)
        g.z[0].fill_(7.0)
        g.v_cycle()
        z = _np(g.z[0])
        g.reinitialize(ct, st)
        g.grid_extra(bits)
        it = g.solve(500)
        assert g.last_status == "converged"
        torch.cuda.synchronize()
        out.append((bits, z, it, _np(g.x)))
    _, z0, it0, x0 = out[0]
    for bits, z, it, x in out[1:]:
        np.testing.assert_array_equal(z, z0, err_msg=f"V-cycle, grid bits {bits:#x}")
        assert abs(it - it0) <= 1, bits
        assert rel_l2(x, x0) < 1e-5, bits


def test_grid_bits_checked():
    from mg_lib import MGError
    g, _ = gpu_for(small_3d(32, levels=3))
    _, streamed = g.split_levels()
    with pytest.raises(MGError):
        g.grid_extra(1 << (2 * streamed))  # beyond the streamed levels
