"""Every wait of the sparse sweeps is bounded (setup option "spin_limit", 2^24 polls by default).

A sweep row waits on the ready flags of the rows it reads.  With a limit of a few polls some wait
runs out on a layout with long dependency chains: the CTA then raises the workspace's error word,
every warp leaves, and the call returns S2L_ERR_TIMEOUT.  Nothing faults or hangs: the wait is
a bounded loop that returns.  The context and the setup stay usable, and with the default limit
restored the same setup applies and solves as before.
"""
import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_a_sweep_wait_that_runs_out_returns_timeout():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    w, st = small_setup("bubbles3d", nx=20, nsub=4)
    # no dense tail and no chain blocks: the deepest sparse dependency chains
    g = capi.GpuSetup(ctx, st, options={"tail_max": 0, "chain_block": 1})
    assert g.stat("levels_max") >= 50
    r = np.random.default_rng(11).standard_normal(st.n)
    z0 = g.apply(r)
    x0, res0 = g.gmres(st.b, restart=w.restart, rtol=1e-8)
    g.set_option("spin_limit", 1)  # checked every 32 polls: a wait gives up after 32 polls
    with pytest.raises(capi.S2LError) as e:
        for _ in range(20):
            g.apply(r)
    assert e.value.code == 5 and "bounded wait" in str(e.value)
    with pytest.raises(capi.S2LError) as e:
        for _ in range(5):
            g.gmres(st.b, restart=w.restart, rtol=1e-8)
    assert e.value.code == 5
    g.set_option("spin_limit", 1 << 24)
    assert rel(g.apply(r), z0) == 0.0  # the apply is deterministic: bit-identical to before
    x1, res1 = g.gmres(st.b, restart=w.restart, rtol=1e-8)
    assert res1["converged"] and res1["iterations"] == res0["iterations"]
    assert rel(x1, x0) == 0.0
    g.close()
    ctx.close()


def test_spin_limit_is_validated():
    from s2l_b200 import capi
    ctx = capi.Context(0)
    _, st = small_setup("poisson2d")
    g = capi.GpuSetup(ctx, st)
    with pytest.raises(capi.S2LError) as e:
        g.set_option("spin_limit", 0)
    assert e.value.code == 1
    with pytest.raises(capi.S2LError) as e:
        g.set_option("tail_max", 10)  # layout options are fixed once the setup is uploaded
    assert e.value.code == 7
    g.close()
    ctx.close()
