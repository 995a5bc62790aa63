"""CPU checks of bench.py's host logic that needs no GPU: the warm-up choice of
the multigrid cycle shape (timers faked, solves faked)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


class _Event:
    """Stand-in for torch.cuda.Event: elapsed time = the fake clock's advance."""
    clock = [0.0]

    def __init__(self, **kw):
        self.t = None

    def record(self):
        self.t = _Event.clock[0]

    def elapsed_time(self, other):
        return other.t - self.t


def test_cycle_choice_keeps_fastest_converged_candidate(monkeypatch):
    import torch

    import bench
    from hicar_b200 import wind_iterative as wi
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda: None)
    applied = []
    monkeypatch.setattr(wi, "set_options", lambda o: applied.append(o))
    # per candidate (by its W levels): solve time, whether it converged with the multigrid preconditioner
    runs = {(): 500.0, (2, 3): 150.0, (2, 3, 4): 120.0}

    def step():
        o = applied[-1]
        key = tuple(o.mg_w_levels)
        ms = runs.get(key, 400.0) if not (key == () and o.mg_skip_fine_presmooth) else 300.0
        _Event.clock[0] += ms
        if key == (2, 3, 4):   # this one stalls and falls back to the reference solve
            return {"status": 3, "precond": 0}
        return {"status": 0, "precond": 1}

    base = bench.solver_kwargs("mg")
    opt, name, table = bench.pick_cycle(wi, step, base)
    assert table["V01-W24"] is None                  # fell back: never chosen although fastest
    assert name == "V01-W23" and table[name] == 150.0
    assert opt.mg_w_levels == (2, 3) and opt.mg_skip_fine_presmooth and opt.mg_omega == 1.0
    assert opt.precond == base["precond"] and opt.stall_iters == base["stall_iters"]
    assert applied[-1] is opt                             # the chosen options are left set
    # every candidate failing: the V-cycle preset itself
    def bad_step():
        _Event.clock[0] += 1.0
        return {"status": 3, "precond": 0}

    opt, name, table = bench.pick_cycle(wi, bad_step, base)
    assert name == "V11" and all(v is None for v in table.values())
    assert opt.mg_w_levels == () and not opt.mg_skip_fine_presmooth
