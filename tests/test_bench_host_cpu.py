"""CPU checks of bench.py's host logic that needs no GPU: the warm-up choice of
the multigrid cycle shape and of the Krylov vector precision (timers faked,
solves faked)."""
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


def _setup(monkeypatch):
    import torch

    from hicar_b200 import wind_iterative as wi
    monkeypatch.setattr(torch.cuda, "Event", _Event)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda: None)
    applied = []
    monkeypatch.setattr(wi, "set_options", lambda o: applied.append(o))
    return wi, applied


def _fake_step(applied, f32_ms_factor, f32_true_res):
    # per candidate (by its W levels): solve time; W on 2-4 stalls and falls back
    runs = {(): 500.0, (2, 3): 150.0, (2, 3, 4): 120.0}

    def step():
        o = applied[-1]
        key = tuple(o.mg_w_levels)
        ms = runs.get(key, 400.0) if not (key == () and o.mg_skip_fine_presmooth) else 300.0
        f32 = o.krylov_precision == 2
        _Event.clock[0] += ms * (f32_ms_factor if f32 else 1.0)
        if key == (2, 3, 4):
            return {"status": 3, "precond": 0, "true_res": 1e-7, "target": 1e-6}
        return {"status": 0, "precond": 1, "true_res": f32_true_res if f32 else 9e-7, "target": 1e-6}
    return step


def test_cycle_choice_keeps_fastest_converged_candidate(monkeypatch):
    import bench
    wi, applied = _setup(monkeypatch)
    base = bench.solver_kwargs("mg")
    opt, name, table = bench.pick_cycle(wi, _fake_step(applied, 1.0, 9e-7), base)
    assert table["V01-W24"] is None                       # fell back: never chosen although fastest
    assert name == "V01-W23" and table[name] == 150.0      # the FP32-vector trial was not faster
    assert table["V01-W23/f32-vectors"] == 150.0
    assert opt.mg_w_levels == (2, 3) and opt.mg_skip_fine_presmooth and opt.mg_omega == 1.0
    assert opt.krylov_precision == base["krylov_precision"]
    assert opt.precond == base["precond"] and opt.stall_iters == base["stall_iters"]
    assert applied[-1] is opt                              # the chosen options are left set


def test_fp32_vectors_kept_only_when_faster_and_accurate(monkeypatch):
    import bench
    wi, applied = _setup(monkeypatch)
    base = bench.solver_kwargs("mg")
    opt, name, table = bench.pick_cycle(wi, _fake_step(applied, 0.9, 9.5e-7), base)
    assert name == "V01-W23/f32-vectors" and opt.krylov_precision == 2 and opt.mg_w_levels == (2, 3)
    opt, name, table = bench.pick_cycle(wi, _fake_step(applied, 0.9, 3e-6), base)   # true residual too large
    assert name == "V01-W23" and table["V01-W23/f32-vectors"] is None and opt.krylov_precision == 0
    assert bench.krylov_desc(opt) == "f64"


def test_no_candidate_converges(monkeypatch):
    import bench
    wi, applied = _setup(monkeypatch)

    def bad_step():
        _Event.clock[0] += 1.0
        return {"status": 3, "precond": 0, "true_res": 1.0, "target": 1e-6}

    opt, name, table = bench.pick_cycle(wi, bad_step, bench.solver_kwargs("mg"))
    assert name == "V11" and all(v is None for v in table.values())
    assert opt.mg_w_levels == () and not opt.mg_skip_fine_presmooth


def test_shorter_graphs_kept_when_faster(monkeypatch):
    import bench
    wi, applied = _setup(monkeypatch)
    inner = _fake_step(applied, 0.9, 9.5e-7)

    def step():
        t0 = _Event.clock[0]
        st = inner()
        if applied[-1].check_every == 4:        # fewer iterations launched past convergence
            _Event.clock[0] = t0 + 0.95 * (_Event.clock[0] - t0)
        return st

    opt, name, table = bench.pick_cycle(wi, step, bench.solver_kwargs("mg"))
    assert name == "V01-W23/f32-vectors/chunk4"
    assert opt.check_every == 4 and opt.krylov_precision == 2 and opt.mg_w_levels == (2, 3)
    assert table[name] < table["V01-W23/f32-vectors"] < table["V01-W23"]
