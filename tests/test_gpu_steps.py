"""Planes per pipeline step of the streamed level sweep (the autotuner's choice
of one plane or the tile's two, per level and direction): only the shared-
memory ring, the step loop and the prefetch change, not the arithmetic.  z of
one V-cycle and the solve (x and iteration count) are BIT-EXACT with every
streamed PRE and POST sweep forced to one plane, forced to two, and as tuned,
for 1, 2 and 3 smoothing sweeps."""
import numpy as np
import pytest

import mg_scenes
from helpers import box_3d, gpu_for, small_3d

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
