"""pf_join_unique_hash_static (the unique hash join on the library's fixed
device scratch, no workspace, match count left on the device) against
pf_join_unique_hash through the C ABI: two calls in a row on different inputs,
one and two keys, equal outputs; sizes past the scratch are refused.  Named to
run last, after every other test file has used the device."""
from __future__ import annotations

import pytest
import torch

from pageflow_b200 import _native

pytestmark = pytest.mark.gpu

def _inputs(seed, n_build, n_probe, nkeys):
    g = torch.Generator().manual_seed(seed)
    # unique build tuples; probe rows draw from them and from keys that miss
    k0 = torch.randperm(4 * n_build, generator=g)[:n_build].to(torch.int64) * 7 - 3 * n_build
    k1 = torch.randint(-5, 5, (n_build,), generator=g, dtype=torch.int64)
    pick = torch.randint(0, n_build, (n_probe,), generator=g)
    p0 = k0[pick].clone()
    p1 = k1[pick].clone()
    miss = torch.rand(n_probe, generator=g) < 0.3
    p0[miss] += 1                               # k0 are multiples of 7 apart: a miss
    b = [k0.cuda(), k1.cuda() if nkeys == 2 else None]
    p = [p0.cuda(), p1.cuda() if nkeys == 2 else None]
    return b, p


def _with_workspace(b, p, nkeys):
    L = _native.lib()
    nb, npr = b[0].numel(), p[0].numel()
    ws = _native.workspace(L.pf_join_unique_hash_workspace(nb, npr), b[0].device)
    bi = torch.empty(npr, dtype=torch.int64, device="cuda")
    pi = torch.empty(npr, dtype=torch.int64, device="cuda")
    host = torch.zeros(2, dtype=torch.int64, pin_memory=True)
    _native.check(L.pf_join_unique_hash(
        _native.ptr(b[0]), _native.ptr(b[1]), nb, _native.ptr(p[0]), _native.ptr(p[1]), npr,
        nkeys, _native.ptr(bi), _native.ptr(pi), host.data_ptr(), _native.ptr(ws), ws.numel(),
        _native.stream_of(b[0].device)), "join_unique_hash")
    n = int(host[0])
    return bi[:n].cpu(), pi[:n].cpu()


def _static(b, p, nkeys, bi, pi, cnt):
    L = _native.lib()
    return L.pf_join_unique_hash_static(
        _native.ptr(b[0]), _native.ptr(b[1]), b[0].numel(), _native.ptr(p[0]), _native.ptr(p[1]),
        p[0].numel(), nkeys, _native.ptr(bi), _native.ptr(pi), _native.ptr(cnt),
        _native.stream_of(b[0].device))


@pytest.mark.parametrize("nkeys", [1, 2])
def test_static_scratch_matches_workspace_path_twice_in_a_row(nkeys):
    # the largest sizes the scratch holds, then a small call on other keys
    # right after it on the same stream: the second call must not see the
    # first call's table
    cases = [(11, 524288, 1048576), (12, 1000, 5000)]
    inputs = [_inputs(seed, nb, npr, nkeys) for seed, nb, npr in cases]
    wants = [_with_workspace(b, p, nkeys) for b, p in inputs]
    outs = []
    for b, p in inputs:
        npr = p[0].numel()
        outs.append((torch.full((npr,), -7, dtype=torch.int64, device="cuda"),
                     torch.full((npr,), -7, dtype=torch.int64, device="cuda"),
                     torch.full((1,), -1, dtype=torch.int64, device="cuda")))
    rcs = [_static(b, p, nkeys, *o) for (b, p), o in zip(inputs, outs)]
    torch.cuda.synchronize()
    for rc, (wb, wp), (bi, pi, cnt) in zip(rcs, wants, outs):
        _native.check(rc, "join_unique_hash_static")
        n = int(cnt.item())
        assert n == wb.numel() > 0
        assert torch.equal(bi[:n].cpu(), wb) and torch.equal(pi[:n].cpu(), wp)
        # nothing written past the matches
        assert bool((bi[n:] == -7).all()) and bool((pi[n:] == -7).all())


def test_static_scratch_refuses_sizes_past_its_limit():
    L = _native.lib()
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    for nb, npr in [(1100000, 1000), (1000, 4 * 1048576)]:
        # buffers of the sizes claimed, though the call must refuse them
        bk = torch.zeros(nb, dtype=torch.int64, device="cuda")
        pk = torch.zeros(npr, dtype=torch.int64, device="cuda")
        out = torch.empty(npr, dtype=torch.int64, device="cuda")
        rc = L.pf_join_unique_hash_static(_native.ptr(bk), None, nb, _native.ptr(pk), None,
                                          npr, 1, _native.ptr(out), _native.ptr(out),
                                          _native.ptr(cnt), _native.stream_of(bk.device))
        assert rc == _native.PF_EINVAL
        assert b"static scratch" in L.pf_last_error()
    b, p = _inputs(3, 1000, 1000, 1)
    # a refused call queued nothing: the stream still runs and a valid call works
    torch.cuda.synchronize()
    bi = torch.empty(1000, dtype=torch.int64, device="cuda")
    pi = torch.empty(1000, dtype=torch.int64, device="cuda")
    _native.check(_static(b, p, 1, bi, pi, cnt), "join_unique_hash_static")
    torch.cuda.synchronize()
    wb, wp = _with_workspace(b, p, 1)
    n = int(cnt.item())
    assert torch.equal(bi[:n].cpu(), wb) and torch.equal(pi[:n].cpu(), wp)


def test_static_calls_allocate_no_device_memory():
    """After one call has set the scratch up (and loaded the module's
    kernels), further calls leave both torch's allocator and the device's
    free memory exactly where they were: the join's scratch is the library's
    fixed array, its outputs are the caller's."""
    b, p = _inputs(21, 200_000, 400_000, 1)
    npr = p[0].numel()
    bi = torch.empty(npr, dtype=torch.int64, device="cuda")
    pi = torch.empty(npr, dtype=torch.int64, device="cuda")
    cnt = torch.empty(1, dtype=torch.int64, device="cuda")
    _native.check(_static(b, p, 1, bi, pi, cnt), "join_unique_hash_static")
    torch.cuda.synchronize()
    torch_before = torch.cuda.memory_allocated()
    free_before, _ = torch.cuda.mem_get_info()
    for seed in (22, 23, 24):
        b2, p2 = _inputs(seed, 200_000, 400_000, 1)
        torch.cuda.synchronize()
        torch_mid = torch.cuda.memory_allocated()
        free_mid, _ = torch.cuda.mem_get_info()
        for _ in range(3):
            _native.check(_static(b2, p2, 1, bi, pi, cnt), "join_unique_hash_static")
        torch.cuda.synchronize()
        assert torch.cuda.memory_allocated() == torch_mid
        assert torch.cuda.mem_get_info()[0] == free_mid
        del b2, p2
    assert torch.cuda.memory_allocated() == torch_before
    assert free_before > 0
