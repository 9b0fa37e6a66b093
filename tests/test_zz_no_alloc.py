"""s2l_gpu_coarse_apply_noalloc: the coarse correction without any device allocation.

Some callers cannot allocate device memory when they call the solve phase: code whose device
memory belongs to its own pool or allocator (a framework's caching allocator, a memory-capped
serving process), or that must not allocate once its solve loop runs.  This entry point keeps its
scratch in a static device array of the library instead, so it allocates nothing.  These tests call
it through the C ABI, twice in a row on the same array, and check it against the allocating entry
point s2l_gpu_coarse_apply at the 1e-12 tolerance of the other parity tests; they also check that a
setup needing more scratch than the array holds is refused with a clear error.

This file is collected last on purpose: if it fails, every other test has already run.
"""
import numpy as np
import pytest

from conftest import small_setup

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("name,kw", [("bubbles3d", {}),
                                     ("poisson2d", {"nx": 24, "nsub": 4, "pou": "multiplicity", "coarse": "additive"}),
                                     ("convdiff3d", {})])
def test_noalloc_matches_coarse_apply_twice(name, kw):
    import torch
    from s2l_b200 import capi
    ctx = capi.Context(0)
    _, st = small_setup(name, **kw)
    g = capi.GpuSetup(ctx, st)
    rng = np.random.default_rng(99)
    for call in range(2):  # two calls in a row share the static scratch
        r = rng.standard_normal(st.n)
        ref = g.coarse_apply(r)  # the existing entry point (setup-owned scratch)
        rd = torch.tensor(r, device="cuda", dtype=torch.float64)
        xd = torch.full_like(rd, float("nan"))
        torch.cuda.synchronize()
        g.coarse_apply_noalloc(rd.data_ptr(), xd.data_ptr())
        torch.cuda.synchronize()
        x = xd.cpu().numpy()
        assert np.all(np.isfinite(x)), f"call {call}: output not fully written"
        assert rel(x, ref) <= 1e-12, f"call {call}: {rel(x, ref):.3e}"
    g.close()
    ctx.close()


def test_noalloc_on_the_callers_stream():
    """With s2l_gpu_set_stream the kernels go on the caller's stream: writing r on a side stream,
    calling the entry point and synchronizing only that stream gives the allocating path's result."""
    import torch
    from s2l_b200 import capi
    ctx = capi.Context(0)
    _, st = small_setup("bubbles3d")
    g = capi.GpuSetup(ctx, st)
    side = torch.cuda.Stream()
    g.set_stream(side.cuda_stream)
    rng = np.random.default_rng(7)
    for call in range(2):
        r = rng.standard_normal(st.n)
        ref = g.coarse_apply(r)
        r_host = torch.tensor(r, dtype=torch.float64).pin_memory()
        with torch.cuda.stream(side):
            rd = torch.empty(st.n, device="cuda", dtype=torch.float64)
            xd = torch.empty_like(rd)
            xd.fill_(float("nan"))
            rd.copy_(r_host, non_blocking=True)  # r is written on the side stream only
        g.coarse_apply_noalloc(rd.data_ptr(), xd.data_ptr())
        side.synchronize()  # only the caller's stream
        x = xd.cpu().numpy()
        assert np.all(np.isfinite(x)), f"call {call}: output not fully written"
        assert rel(x, ref) <= 1e-12, f"call {call}: {rel(x, ref):.3e}"
    g.set_stream(None)
    g.close()
    ctx.close()


def test_noalloc_refuses_setups_beyond_its_scratch():
    import torch
    from s2l_b200 import capi
    # the multiplicity partition of unity needs the whole local space (> 262144 doubles here)
    ctx = capi.Context(0)
    _, st = small_setup("poisson2d", nx=520, nsub=4, pou="multiplicity", coarse="additive")
    g = capi.GpuSetup(ctx, st)
    rd = torch.zeros(st.n, device="cuda", dtype=torch.float64)
    xd = torch.zeros_like(rd)
    with pytest.raises(capi.S2LError) as e:
        g.coarse_apply_noalloc(rd.data_ptr(), xd.data_ptr())
    assert e.value.code == 1 and "scratch" in str(e.value)
    g.close()
    ctx.close()
