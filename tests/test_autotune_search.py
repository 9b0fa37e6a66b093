"""The autotuner's coordinate search (s2l_b200.autotune), on the CPU with a stand-in for the device
setup: it keeps the fastest candidate, closes every other one, never revisits an option once it has
moved on, tries the runtime options on the current best setup (and sets back the best value), and
reports the default's time and the gain."""
import pytest

from s2l_b200 import autotune


class FakeSetup:
    """Stands in for capi.GpuSetup: the measured times come from a table of the options."""
    built, closed = [], []

    def __init__(self, ctx, st, options=None):
        self.options = dict(options or {})
        self.n = 4
        FakeSetup.built.append(self)

    def close(self):
        FakeSetup.closed.append(self)

    def set_option(self, name, value):
        self.options[name] = value


def fake_measure(g, k, reps, rng):
    o = g.options
    t = 10.0
    t -= {0.25: 0.0, 0.1: 1.0, 0.5: -1.0, 1.0: 0.5}[o.get("hop_us", 0.25)]
    t -= {8: 0.0, 4: -2.0, 16: 0.7}[o.get("chain_block", 8)]
    t -= {16: 0.0, 32: -0.2, 8: 0.2}[o.get("sweep_group", 16)]
    t -= {8: 0.0, 16: 0.4, 24: 0.3}[o.get("sweep_prefetch", 8)]
    return {"local_solve_ms": t, "spmv_ms": {0: 0.5, 1: 0.3, 2: 0.6, 4: 0.7}[o.get("spmv_tpr", 0)]}


def test_coordinate_search_keeps_the_fastest(monkeypatch):
    monkeypatch.setattr(autotune.capi, "GpuSetup", FakeSetup)
    monkeypatch.setattr(autotune, "measure", fake_measure)
    FakeSetup.built, FakeSetup.closed = [], []
    g, rep = autotune.tune(None, None, k=4, reps=1, base={"refactor": 1})
    assert rep["chosen"] == {"hop_us": 0.1, "chain_block": 16, "sweep_group": 8, "spmv_tpr": 1, "sweep_prefetch": 16}
    assert g.options == dict(rep["chosen"], refactor=1)  # the runtime option set back to its best value
    # a new setup per candidate of the layout options, none for the runtime option
    assert len(FakeSetup.built) == 1 + sum(len(v) - 1 for q, v in autotune.SEARCH if q not in autotune.RUNTIME)
    assert g not in FakeSetup.closed and len(FakeSetup.closed) == len(FakeSetup.built) - 1
    assert rep["default_ms"] == pytest.approx(10.0 + 2 * 0.5)
    assert rep["ms"] == pytest.approx(10.0 - 1.0 - 0.7 - 0.2 - 0.4 + 2 * 0.3)
    assert rep["gain"] == pytest.approx(rep["default_ms"] / rep["ms"])
