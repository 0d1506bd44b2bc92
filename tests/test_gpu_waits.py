"""Bounded device waits and the status word that reports them.

Every wait inside a kernel (bulk copies landing, tensor-core MMAs completing)
is bounded; one that gives up drains its block's copies and MMAs in flight,
sets LITHO_E_TIMEOUT in the call's status word and lets the block exit. These
tests make waits run out without faulting or hanging the GPU: a probe kernel
waits on a barrier nothing arrives at, and a short wait budget makes the
tensor-core synthesis give up. Each time the status readers must report it,
and the next normal call must succeed with the same images as before.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
LITHO_E_TIMEOUT = 1000001


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200 as lb
    from lithobat_b200 import _native as nat
    from lithobat_b200 import aerial
    return torch, lb, nat, aerial


def _plan(env, n_clips, n):
    torch, lb, nat, aerial = env
    px = 1e-9
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5, sigma_outer=0.9,
                        source_grid=5)
    v = lb.config.optics_view(o)
    pd = aerial.plan_abbe([v] * n_clips, n, px, [[(v.defocus, v.image_index)]] * n_clips, 1.0, False, False)
    dev = torch.device("cuda", torch.cuda.current_device())
    rng = np.random.default_rng(n_clips)
    one = lb.patterns.manhattan_clip(rng, n, px, (10, 20), (40.0, 120.0)).astype(np.float32)
    masks = torch.from_numpy(one).to(dev)[None].repeat(n_clips, 1, 1).contiguous()
    masks += torch.arange(n_clips, device=dev, dtype=torch.float32)[:, None, None] * 1e-3
    blob = torch.from_numpy(pd.blob).to(dev)
    ws_bytes = C.c_size_t(0)
    L = nat.lib()
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=dev)
    return pd, blob, masks, ws


def _run(env, pd, blob, masks, ws):
    torch, _, nat, _ = env
    L = nat.lib()
    n = pd.plan.n
    img = torch.empty((pd.n_out, n, n), dtype=torch.float32, device=masks.device)
    pk = torch.empty((pd.n_out,), dtype=torch.float32, device=masks.device)
    s = torch.cuda.current_stream().cuda_stream
    nat.check("litho_abbe", L.litho_abbe(C.byref(pd.plan), blob.data_ptr(), masks.data_ptr(), img.data_ptr(),
                                          pk.data_ptr(), ws.data_ptr(), ws.numel(), s))
    return img, pk, L.litho_abbe_status(C.byref(pd.plan), ws.data_ptr(), s)


def test_a_wait_that_runs_out_is_reported_and_the_next_call_is_clean(env):
    torch, _, nat, _ = env
    L = nat.lib()
    pd, blob, masks, ws = _plan(env, 3, 256)
    img0, pk0, st0 = _run(env, pd, blob, masks, ws)
    assert st0 == 0
    s = torch.cuda.current_stream().cuda_stream
    # a barrier nothing arrives at: the bounded wait gives up after ~50 us
    nat.check("litho_wait_probe", L.litho_wait_probe(ws.data_ptr(), 100_000, s))
    assert L.litho_abbe_status(C.byref(pd.plan), ws.data_ptr(), s) == LITHO_E_TIMEOUT
    assert b"bounded" in L.litho_status_string(LITHO_E_TIMEOUT)
    # the context is usable and every call clears the word before it starts
    img1, pk1, st1 = _run(env, pd, blob, masks, ws)
    assert st1 == 0
    assert torch.equal(img0, img1) and torch.equal(pk0, pk1)
    assert L.litho_wait_probe(None, 10, s) == -1
    assert L.litho_wait_probe(ws.data_ptr(), 0, s) == -2


def test_short_wait_budget_makes_the_tensor_core_synthesis_give_up(env):
    """80 clips of 1024^2 put the synthesis on the tcgen05 path (bulk-copied
    operand planes, MMAs into TMEM, drains by tcgen05.ld). With a one-cycle
    budget its waits give up; the kernel drains what it issued, frees TMEM,
    and the status reader reports LITHO_E_TIMEOUT. With the default budget
    restored the same call reproduces the first images bit for bit."""
    torch, _, nat, aerial = env
    L = nat.lib()
    pd, blob, masks, ws = _plan(env, 80, 1024)
    assert aerial.engine_info(pd)["synthesis"] == "tensor_cores"
    img0, pk0, st0 = _run(env, pd, blob, masks, ws)
    assert st0 == 0
    seen = []
    try:
        nat.check("litho_set_wait_limit", L.litho_set_wait_limit(1))
        for _ in range(5):
            _img, _pk, st = _run(env, pd, blob, masks, ws)
            seen.append(st)
            if st == LITHO_E_TIMEOUT:
                break
    finally:
        nat.check("litho_set_wait_limit", L.litho_set_wait_limit(0))
    assert seen[-1] == LITHO_E_TIMEOUT, seen
    assert all(st in (0, LITHO_E_TIMEOUT) for st in seen), seen
    img1, pk1, st1 = _run(env, pd, blob, masks, ws)
    assert st1 == 0
    assert torch.equal(img0, img1) and torch.equal(pk0, pk1)
    assert L.litho_set_wait_limit(-1) == -2


def test_python_entry_points_raise_on_a_timed_out_status(env):
    """compute_aerial_batch with host masks reads the status word and raises
    LithoError when a wait gave up (the probe stands in for the failure)."""
    torch, lb, nat, aerial = env
    L = nat.lib()
    g = lb.GridConfig(n_pixels=128, pixel_size=2e-9)
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_grid=5)
    m = lb.patterns.lines_and_spaces(128, 2e-9, 80e-9, 40e-9)
    lb.compute_aerial_batch(m, o, g)          # status 0: no error
    v = lb.config.optics_view(o)
    pd = aerial.plan_abbe([v], 128, 2e-9, [[(v.defocus, v.image_index)]], 1.0, False, False)
    dev = torch.device("cuda", torch.cuda.current_device())
    ws = nat.Workspace.get(torch, dev, 0, tag="fused")
    nat.check("litho_wait_probe", L.litho_wait_probe(ws.data_ptr(), 1000, torch.cuda.current_stream().cuda_stream))
    with pytest.raises(nat.LithoError) as e:
        aerial.check_status(pd, dev)
    assert e.value.status == LITHO_E_TIMEOUT
    lb.compute_aerial_batch(m, o, g)          # the next call clears the word
    aerial.check_status(pd, dev)
