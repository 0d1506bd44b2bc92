"""The allocation-free Abbe entry point, checked against the workspace one.

litho_abbe_noalloc() exists for callers that cannot hand the library a device
workspace: processes whose device memory is all owned by another allocator,
or loops that must not pay cudaMalloc's implicit synchronisation. It runs the
same kernels in a fixed 32 MiB scratch array compiled into the library. This
file is collected last so that a failure here comes after every other test.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200 as lb
    from lithobat_b200 import _native as nat
    from lithobat_b200.aerial import plan_abbe
    return torch, lb, nat, plan_abbe


def _case(env, n_clips, seed):
    torch, lb, nat, plan_abbe = env
    rng = np.random.default_rng(seed)
    n, px = 256, 2e-9
    masks = np.stack([lb.patterns.manhattan_clip(rng, n, px, (10, 20)) for _ in range(n_clips)])
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                        source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=15,
                        defocus=20e-9, zernike_coeffs={5: 0.01})
    v = lb.config.optics_view(o)
    pd = plan_abbe([v] * n_clips, n, px, [[(v.defocus, v.image_index)]] * n_clips, 1.0, False, False)
    dev = torch.device("cuda", torch.cuda.current_device())
    blob = torch.from_numpy(pd.blob).to(dev)
    m = torch.from_numpy(masks.astype(np.float32)).to(dev)
    return pd, blob, m


def _run_both(env, pd, blob, m):
    torch, lb, nat, _ = env
    L = nat.lib()
    dev = m.device
    n = pd.plan.n
    ws_bytes = C.c_size_t(0)
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    assert ws_bytes.value <= nat.NOALLOC_SCRATCH_BYTES
    ws = torch.empty(ws_bytes.value, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    img_a = torch.empty((pd.n_out, n, n), dtype=torch.float32, device=dev)
    pk_a = torch.empty(pd.n_out, dtype=torch.float32, device=dev)
    nat.check("litho_abbe", L.litho_abbe(C.byref(pd.plan), blob.data_ptr(), m.data_ptr(), img_a.data_ptr(),
                                          pk_a.data_ptr(), ws.data_ptr(), ws.numel(), s))
    img_b = torch.full((pd.n_out, n, n), float("nan"), dtype=torch.float32, device=dev)
    pk_b = torch.full((pd.n_out,), float("nan"), dtype=torch.float32, device=dev)
    nat.check("litho_abbe_noalloc", L.litho_abbe_noalloc(C.byref(pd.plan), blob.data_ptr(), m.data_ptr(),
                                                          img_b.data_ptr(), pk_b.data_ptr(), s))
    torch.cuda.synchronize()
    return img_a, pk_a, img_b, pk_b


def test_noalloc_matches_workspace_entry_point_on_two_calls_in_a_row(env):
    torch = env[0]
    for call, (clips, seed) in enumerate([(3, 1), (2, 2)]):
        pd, blob, m = _case(env, clips, seed)
        img_a, pk_a, img_b, pk_b = _run_both(env, pd, blob, m)
        assert torch.isfinite(img_b).all() and torch.isfinite(pk_b).all(), f"call {call}"
        err = float(((img_b.double() - img_a.double()).abs().amax() / img_a.double().abs().amax()))
        assert err <= TOL, f"call {call}: {err:.3e}"
        assert float(((pk_b - pk_a).abs() / pk_a.abs()).max()) <= TOL
        # the status reader of the fixed scratch: no bounded wait gave up
        L = env[2].lib()
        assert L.litho_abbe_noalloc_status(C.byref(pd.plan), torch.cuda.current_stream().cuda_stream) == 0


def test_noalloc_rejects_plans_beyond_its_scratch(env):
    torch, lb, nat, plan_abbe = env
    L = nat.lib()
    # 1024^2 vector clips: ~100 clips need more than 32 MiB of scratch
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, imaging_model="vector", polarisation="te",
                        source_type="annular", sigma_inner=0.5, sigma_outer=0.9, source_grid=31)
    v = lb.config.optics_view(o)
    pd = plan_abbe([v] * 128, 1024, 1e-9, [[(v.defocus, v.image_index)]] * 128, 1.0, False, True)
    ws_bytes = C.c_size_t(0)
    nat.check("litho_abbe_workspace", L.litho_abbe_workspace(C.byref(pd.plan), C.byref(ws_bytes)))
    assert ws_bytes.value > nat.NOALLOC_SCRATCH_BYTES
    # rejected on the host before anything is launched; the outputs stay untouched
    dev = torch.device("cuda", torch.cuda.current_device())
    blob = torch.from_numpy(pd.blob).to(dev)
    m = torch.zeros((128, 1024, 1024), dtype=torch.complex64, device=dev)
    img = torch.full((128, 1024, 1024), 7.0, dtype=torch.float32, device=dev)
    pk = torch.full((128,), 7.0, dtype=torch.float32, device=dev)
    st = L.litho_abbe_noalloc(C.byref(pd.plan), blob.data_ptr(), m.data_ptr(), img.data_ptr(), pk.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert st == -8
    assert bool((img == 7.0).all()) and bool((pk == 7.0).all())
    assert b"no-allocation" in L.litho_status_string(st)
