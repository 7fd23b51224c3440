"""The solve server's HBM admission and eviction rules on the CPU.

SolveServer admits a session only while the workspace bytes of the admitted
sessions stay within its HBM budget, reuses an idle workspace of the same
shape when one is pooled, frees idle workspaces of other shapes (largest
first) before it creates a new one that would pass the budget, and refuses a
session larger than the whole budget.  These rules are host bookkeeping: here
the solver is a stand-in that allocates nothing and a workspace of a 2D
session of side s weighs s * s bytes.
"""
import types

import pytest

import mg_serve


class FakeSolver:
    made = 0
    closed = 0

    def __init__(self, dim, res, levels, pre_post, bottom, storage=None, device=None):
        FakeSolver.made += 1
        self.res = res

    def close(self):
        FakeSolver.closed += 1


@pytest.fixture
def server(monkeypatch):
    monkeypatch.setattr(mg_serve, "MGPCGPoissonSolver", FakeSolver)
    monkeypatch.setattr(mg_serve, "plan_bytes", lambda dim, res, levels, storage: res[0] ** dim)
    FakeSolver.made = FakeSolver.closed = 0

    def make(budget):
        return mg_serve.SolveServer(storage="f32", streams=0, hbm_budget=budget, device="cpu",
                                    params=lambda dim, side: (3, 2, 50))
    return make


def _session(solver, key):
    return types.SimpleNamespace(solver=solver, key=key)


def test_admits_within_budget_and_reuses_idle_workspaces(server):
    s = server(250)
    a, ka = s._acquire(2, 10)            # 100 bytes
    b, kb = s._acquire(2, 10)            # 200
    assert a is not None and b is not None and s.in_use == 200
    c, _ = s._acquire(2, 10)             # 300 > 250: the session waits
    assert c is None and s.in_use == 200
    s._release(_session(a, ka))          # back to the pool as an idle workspace
    assert s.in_use == 100 and s.idle == 100
    d, _ = s._acquire(2, 10)             # the idle workspace of the same shape
    assert d is a and s.in_use == 200 and s.idle == 0
    assert FakeSolver.made == 2 and s.peak_in_use == 200


def test_new_shape_evicts_idle_workspaces_first(server):
    s = server(250)
    a, ka = s._acquire(2, 10)
    b, _ = s._acquire(2, 10)
    s._release(_session(a, ka))          # in use 100, idle 100
    c, _ = s._acquire(2, 12)             # 144 bytes: 100 + 100 + 144 > 250
    assert c is not None and FakeSolver.made == 3
    assert s.evictions == 1 and FakeSolver.closed == 1
    assert s.idle == 0 and s.in_use == 244 and s.peak_resident <= 250


def test_session_larger_than_the_budget_is_refused(server):
    s = server(250)
    with pytest.raises(ValueError, match="more than the whole HBM budget"):
        s._acquire(2, 16)                # 256 bytes
