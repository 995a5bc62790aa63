"""CPU check of the multigrid solve emulation (tests/mg_emulate.py) on a small
generated case: every cycle shape it offers converges, and the names parse."""
import pytest


def test_emulated_cycles_converge():
    import mg_emulate
    out = mg_emulate.main(["40", "36", "10", "--alpha", "smooth", "--hills", "6",
                           "--cycles", "V11,V01,V01-W23"])
    assert all(0 < it < 100 for it in out.values()), out


def test_cycle_names():
    import numpy as np

    import mg_emulate
    c = np.zeros((15, 4, 3, 4), np.float32)
    c[0] = -4.0
    assert mg_emulate.cycle("V01-W24", c).wlevels == {2, 3, 4}
    assert mg_emulate.cycle("V11", c).fine_presmooth and not mg_emulate.cycle("V01", c).fine_presmooth
    with pytest.raises(ValueError):
        mg_emulate.cycle("F", c)
