"""dpa_advect_device_no_alloc against dpa_advect_device.

The no-alloc entry point serves callers that must not allocate device memory
while running (their device memory is reserved up front by another owner, or
a cudaMalloc's device-wide synchronization would stall their other streams).
It takes its ordering scratch from a fixed array inside the library. This
test calls it through the C ABI twice in a row, with different inputs, and
requires the same bit-exact results as the allocating entry point, no change
in free device memory across calls, and a clear error above the size limit.
It creates its own context, so it runs the same alone in a fresh process or
after the other tests."""
import ctypes as C

import numpy as np
import pytest
from bitwise import assert_same

pytestmark = pytest.mark.gpu


def test_no_alloc_matches_the_allocating_entry_point():
    import torch

    import dpa_b200
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds

    ctx = dpa_b200.Context(0)
    lib = ctx._lib
    grid = fields.curl_noise(64, 4.0, 5)
    field = ctx.field(grid)
    offset, size = seeds.seed_box(grid)
    opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, 1)

    counts = (50000, 20000)
    inputs = []
    for i, n in enumerate(counts):
        p = seeds.generate_random(offset, size, n, 300, seed=20 + i).position
        inputs.append((torch.from_numpy(p).cuda(), torch.full((n,), 300, dtype=torch.int64,
                                                               device="cuda")))
    biggest = max(counts)
    pos = torch.empty((biggest, 3), dtype=torch.float32, device="cuda")
    rem = torch.empty(biggest, dtype=torch.int64, device="cuda")
    term = torch.empty(biggest, dtype=torch.uint8, device="cuda")

    def run(entry, which):
        p0, r0 = inputs[which]
        n = p0.shape[0]
        pos[:n].copy_(p0)
        rem[:n].copy_(r0)
        term[:n].zero_()
        torch.cuda.synchronize()
        ctx.check(entry(ctx.handle, field.handle, C.byref(opts), n, C.c_void_p(pos.data_ptr()),
                        C.c_void_p(rem.data_ptr()), C.c_void_p(term.data_ptr()), None))
        ctx.synchronize()
        return pos[:n].cpu().numpy(), rem[:n].cpu().numpy(), term[:n].cpu().numpy()

    want = [run(lib.dpa_advect_device, i) for i in range(len(counts))]
    # Warm the allocating path's caches first so that only the no-alloc calls
    # remain between the two memory readings below.
    free_before = None
    for call in range(2):
        for i in range(len(counts)):
            got = run(lib.dpa_advect_device_no_alloc, i)
            for g, w in zip(got, want[i]):
                assert_same(g, w)
        if call == 0:
            free_before = torch.cuda.mem_get_info()[0]
    assert torch.cuda.mem_get_info()[0] == free_before

    too_many = N.NO_ALLOC_MAX_PARTICLES + 1
    status = lib.dpa_advect_device_no_alloc(ctx.handle, field.handle, C.byref(opts), too_many,
                                            C.c_void_p(pos.data_ptr()),
                                            C.c_void_p(rem.data_ptr()),
                                            C.c_void_p(term.data_ptr()), None)
    assert status == 1
    assert b"DPA_NO_ALLOC_MAX_PARTICLES" in lib.dpa_last_error(ctx.handle)
    field.close()
    ctx.close()


@pytest.mark.parametrize("morton_order", [0, 1])
@pytest.mark.parametrize("tuned", [False, True])
def test_no_alloc_small_counts_orders_and_resumption(morton_order, tuned):
    """The paths that use only the shared work counter (one particle, input
    order) and a step budget followed by a resume, against dpa_advect_device
    on one stream, with the context's default and a non-default tuning (which
    both entry points apply)."""
    import torch

    import dpa_b200
    from dpa_b200 import _native as N
    from dpa_b200 import fields, seeds

    ctx = dpa_b200.Context(0)
    lib = ctx._lib
    if tuned:
        t = N.Tuning(32, 2, 16, 0.0, 64, 2)
        ctx.check(lib.dpa_context_set_tuning(ctx.handle, C.byref(t)))
    grid = fields.curl_noise(48, 3.0, 6)
    field = ctx.field(grid)
    offset, size = seeds.seed_box(grid)
    stream = ctx.stream

    def call(entry, p0, steps, max_steps, resume_from=None):
        n = p0.shape[0]
        opts = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], 0.25, 0, 0, 0, morton_order,
                               max_steps)
        if resume_from is None:
            pos = torch.from_numpy(p0.copy()).cuda()
            rem = torch.full((n,), steps, dtype=torch.int64, device="cuda")
            term = torch.zeros(n, dtype=torch.uint8, device="cuda")
        else:
            pos, rem, term = resume_from
        torch.cuda.synchronize()
        ctx.check(entry(ctx.handle, field.handle, C.byref(opts), n, C.c_void_p(pos.data_ptr()),
                        C.c_void_p(rem.data_ptr()), C.c_void_p(term.data_ptr()),
                        C.c_void_p(stream)))
        ctx.synchronize()
        return pos, rem, term

    def host(state):
        return tuple(x.cpu().numpy() for x in state)

    for n in (1, 3000):
        p0 = seeds.generate_random(offset, size, n, 0, seed=40 + n).position
        for budget in (0, 37):
            want_state = call(lib.dpa_advect_device, p0, 200, budget)
            got_state = call(lib.dpa_advect_device_no_alloc, p0, 200, budget)
            for g, w in zip(host(got_state), host(want_state)):
                assert_same(g, w)
            if budget:
                # Resume both from their in-flight states, twice.
                for _ in range(2):
                    want_state = call(lib.dpa_advect_device, p0, 200, budget, want_state)
                    got_state = call(lib.dpa_advect_device_no_alloc, p0, 200, budget, got_state)
                    for g, w in zip(host(got_state), host(want_state)):
                        assert_same(g, w)

    # The same argument checks as dpa_advect_device: a non-finite step size.
    bad = N.AdvectOptions(N.INTEGRATORS["runge_kutta_4"], float("nan"), 0, 0, 0, 1, 0)
    pos = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    rem = torch.zeros(4, dtype=torch.int64, device="cuda")
    for entry in (lib.dpa_advect_device, lib.dpa_advect_device_no_alloc):
        status = entry(ctx.handle, field.handle, C.byref(bad), 4, C.c_void_p(pos.data_ptr()),
                       C.c_void_p(rem.data_ptr()), None, None)
        assert status == 1
        assert b"step_size" in lib.dpa_last_error(ctx.handle)
    field.close()
    ctx.close()
