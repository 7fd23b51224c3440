"""The column-register sweep (k_colsweep: TMA-staged planes, each thread's
y-pair of columns in registers, one block barrier per plane step) against the
shared-memory ring sweep (k_sweep) and the float32 oracle.

Both kernels evaluate the same float32 operations in the reference's order
(mgpcg.py:104-123), so one V-cycle's z is BIT-EXACT for every tile shape,
every level the column kernel can run, float32 and 16-bit storage, and
against the oracle.  A solve differs only through the order of the FP64 z.r
sum that the level-0 POST sweep accumulates per block: iterations +-1 and
x within 1e-5.
"""
import numpy as np
import pytest

import mg_scenes
from helpers import box_3d, gpu_for, oracle_for, rel_l2, small_3d

pytestmark = pytest.mark.gpu

SCENES = {
    "drop3d_128": lambda: small_3d(128, levels=5),
    "box_96x64x128": lambda: box_3d((96, 64, 128), 4),
}
SHAPES = (1, 2, 3)  # 32x16, 32x32, 64x16 column tiles


def _np(t):
    return t.detach().float().cpu().numpy()


def _every(streamed, shape):
    return sum(shape << (2 * l) for l in range(streamed))


def _vcycle(g, st, ct, bits):
    """z of one V-cycle on r = b with every level above the coarse block
    streamed and the given sweep kernels."""
    g.reinitialize(ct, st)
    g.resident(False)
    assert g.sweep_kernel(bits) == bits
    g.r[0].copy_(g.b)
    g.z[0].fill_(7.0)
    g.v_cycle()
    return _np(g.z[0])


@pytest.mark.parametrize("storage", [None, "f16", "bf16"])
@pytest.mark.parametrize("name", list(SCENES))
def test_col_vcycle_bit_exact(name, storage):
    import torch
    sc = SCENES[name]()
    g, st = gpu_for(sc, storage=storage)
    ct = torch.from_numpy(sc.cell_type).to(g.x.device)
    _, streamed = g.split_levels()
    assert streamed >= 2
    z_ring = _vcycle(g, st, ct, 0)
    for shape in SHAPES:
        z = _vcycle(g, st, ct, _every(streamed, shape))
        np.testing.assert_array_equal(z, z_ring, err_msg=f"{name} {storage} shape {shape}")
    # one level at a time in the column kernel (the two kernels meet in r[l+1], z[l+1])
    for l in range(streamed):
        z = _vcycle(g, st, ct, 1 << (2 * l))
        np.testing.assert_array_equal(z, z_ring, err_msg=f"{name} {storage} level {l}")
    if storage is None:
        o = oracle_for(sc)
        o.set("r", o.get("b"), 0)
        o.v_cycle()
        np.testing.assert_array_equal(z_ring, o.get("z", 0))


@pytest.mark.parametrize("storage", [None, "f16"])
def test_col_solve_matches_ring(storage):
    import torch
    sc = SCENES["drop3d_128"]()
    g, st = gpu_for(sc, storage=storage)
    ct = torch.from_numpy(sc.cell_type).to(g.x.device)
    _, streamed = g.split_levels()
    out = []
    for bits in (0, _every(streamed, 1), _every(streamed, 3)):
        g.reinitialize(ct, st)
        g.sweep_kernel(bits)
        it = g.solve(500)
        assert g.last_status == "converged", (bits, g.last_status)
        out.append((bits, it, _np(g.x)))
    _, it0, x0 = out[0]
    for bits, it, x in out[1:]:
        assert abs(it - it0) <= 1, (bits, it, it0)
        assert rel_l2(x, x0) < 1e-5, bits


def test_col_tuned_choice_reported():
    """The autotuner's choice is readable and the tuned solve converges."""
    sc = SCENES["drop3d_128"]()
    g, _ = gpu_for(sc)
    _, streamed = g.split_levels()
    bits = g.sweep_kernel()
    assert bits >> (2 * streamed) == 0
    g.solve(500)
    assert g.last_status == "converged"


def test_col_bits_checked():
    from mg_lib import MGError
    g, _ = gpu_for(small_3d(64, levels=4), pre_post=1)  # the column kernel needs pre_post 2
    _, streamed = g.split_levels()
    assert g.sweep_kernel() == 0
    with pytest.raises(MGError):
        g.sweep_kernel(1)
    g2, _ = gpu_for(mg_scenes.dam_break_2d(n=64, levels=3))  # 2D keeps the ring kernel
    with pytest.raises(MGError):
        g2.sweep_kernel(1)
    g3, _ = gpu_for(small_3d(64, levels=4))
    _, streamed3 = g3.split_levels()
    with pytest.raises(MGError):
        g3.sweep_kernel(1 << (2 * streamed3))  # beyond the streamed levels
