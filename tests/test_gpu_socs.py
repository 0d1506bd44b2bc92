"""SOCS decomposition and SOCS imaging on the GPU against the reference."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu
TOL = 1e-5


@pytest.fixture(scope="module")
def lb():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import lithobat_b200
    return lithobat_b200


def _optics(lb, od):
    od = dict(od)
    od["zernike_coeffs"] = {int(k): v for k, v in (od.get("zernike_coeffs") or {}).items()}
    keep = {k: od[k] for k in lb.OpticsConfig.__dataclass_fields__ if k in od}
    return lb.OpticsConfig(**keep)


def rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / np.abs(b).max())


def test_tensor_core_gram_matches_fp64(lb):
    """The tcgen05 Gram (TF32 hi/lo split) against the FP64 CUDA-core Gram."""
    import ctypes as C
    import torch
    from lithobat_b200 import _native as nat
    from lithobat_b200.hopkins import aperture_mask, band_bins
    o = lb.OpticsConfig(NA=1.35, n_immersion=1.44, source_type="annular", sigma_inner=0.5, sigma_outer=0.8,
                        defocus=30e-9, zernike_coeffs={7: 0.02})
    n, px = 256, 4e-9
    src = lb.source_points(o)
    kx, ky, fxb, fyb = band_bins(n, px, o.NA / o.wavelength)
    inside = aperture_mask(fxb, fyb, src, o.NA / o.wavelength)
    L = nat.lib()
    dev = torch.device("cuda", 0)
    pupil = np.zeros(1, dtype=nat.PUPIL_DTYPE)
    pupil["wavelength"], pupil["NA"], pupil["defocus"], pupil["n_image"] = o.wavelength, o.NA, o.defocus, 1.44
    z = np.zeros(21); z[6] = 0.02
    pupil["zernike"], pupil["has_zernike"] = z, 1
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    S, nb = len(src), kx.size
    grams = []
    for mode in (0, 1):
        ws_b = C.c_size_t(0)
        nat.check("ws", L.litho_socs_workspace(S, nb, C.byref(ws_b)))
        ws = torch.empty(ws_b.value, dtype=torch.uint8, device=dev)
        phi = torch.empty((S, nb), dtype=torch.complex128, device=dev)
        lam = torch.empty(S, dtype=torch.float64, device=dev)
        ldg = S + (S & 1)
        G = torch.empty((ldg, ldg), dtype=torch.complex128, device=dev)
        args = [t(pupil.view(np.uint8)), t(src.fx), t(src.fy), t(src.weight)]
        band = [t(kx), t(ky), t(inside)]
        nat.check("build", L.litho_socs_build(args[0].data_ptr(), args[1].data_ptr(), args[2].data_ptr(),
                                              args[3].data_ptr(), S, band[0].data_ptr(), band[1].data_ptr(), nb,
                                              band[2].data_ptr(), n, px, mode, phi.data_ptr(), lam.data_ptr(),
                                              G.data_ptr(), ws.data_ptr(), ws.numel(),
                                              torch.cuda.current_stream().cuda_stream))
        sw = C.c_int(0)
        assert L.litho_socs_status(S, nb, ws.data_ptr(), C.byref(sw), torch.cuda.current_stream().cuda_stream) == 0
        grams.append(G[:S, :S].cpu().numpy())
    tc, ref = grams
    err = np.abs(tc - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
    assert np.allclose(ref, ref.conj().T, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("name", ["conventional", "annular_aberrated", "dipole_exact_clear"])
@pytest.mark.parametrize("gram", ["tensor", "fp64"])
def test_socs_build_and_raw_match_reference(lb, name, gram):
    a, od, gd = load_golden(f"socs_{name}")
    o, g = _optics(lb, od), lb.GridConfig(**gd)
    full = lb.SOCSKernels.build(o, g, tol=0.0, gram=gram)
    tr = lb.SOCSKernels.build(o, g, gram=gram)
    cap = lb.SOCSKernels.build(o, g, max_kernels=3, gram=gram)
    assert full.n_band == int(a["n_band"]) and full.n_source == int(a["n_source"])
    # default tolerance and the cap select the same kernels as the reference
    np.testing.assert_allclose(tr.weights, a["weights_tol"], rtol=1e-9, atol=1e-12 * a["weights_tol"][0])
    np.testing.assert_allclose(cap.weights, a["weights_cap3"], rtol=1e-9)
    assert tr.clear == pytest.approx(float(a["clear_tol"]), rel=1e-9)
    assert tr.energy_kept == pytest.approx(float(a["energy_tol"]), rel=1e-9)
    # tol=0 keeps every non-round-off eigenvalue; the image is the Abbe sum
    assert len(full) <= min(full.n_band, full.n_source)
    mask = a["mask"]
    raw, peak, clear = full.raw(mask)
    assert rel(raw, a["raw_full"]) <= TOL
    assert peak == pytest.approx(float(a["peak_full"]), rel=TOL)
    assert rel(tr.raw(mask)[0], a["raw_tol"]) <= TOL
    assert rel(cap.raw(mask)[0], a["raw_cap3"]) <= TOL
    assert rel(tr.image(mask, 0.8), a["image_tol"]) <= TOL


def test_socs_k24_mid_size(lb):
    a, od, gd = load_golden("socs_imm_128_k24")
    k = lb.SOCSKernels.build(_optics(lb, od), lb.GridConfig(**gd), tol=0.0, max_kernels=24)
    np.testing.assert_allclose(k.weights, a["weights"], rtol=1e-8)
    assert k.clear == pytest.approx(float(a["clear"]), rel=1e-8)
    assert k.energy_kept == pytest.approx(float(a["energy"]), rel=1e-8)
    raw, peak, _ = k.raw(a["mask"].astype(np.float64))
    assert rel(raw, a["raw"]) <= TOL


def test_socs_full_size_weights(lb):
    """The fourth workload's decomposition at 1024^2 (band 657, 124 points)."""
    a, od, gd = load_golden("socs_imm_1024_weights")
    k = lb.SOCSKernels.build(_optics(lb, od), lb.GridConfig(**gd), tol=0.0, max_kernels=26)
    assert k.n_band == int(a["n_band"]) and k.n_source == int(a["n_source"])
    np.testing.assert_allclose(k.weights, a["weights"], rtol=1e-8)


def test_all_kernels_equal_abbe(lb):
    """SOCS with every kernel reproduces the Abbe sum (test_hopkins.py:104-118)."""
    a, od, gd = load_golden("abbe_annular_aberrated")
    o, g = _optics(lb, od), lb.GridConfig(**gd)
    k = lb.SOCSKernels.build(o, g, tol=0.0)
    ra = lb.compute_aerial_image(a["mask"], o, g, return_raw=True)
    rk = k.raw(a["mask"])
    assert rel(rk[0], ra[0]) <= TOL
    assert rk[2] == pytest.approx(ra[2], rel=1e-9)


def test_socs_refuses_vector_and_thick(lb):
    with pytest.raises(ValueError, match="scalar thin-mask"):
        lb.SOCSKernels.build(lb.OpticsConfig(imaging_model="vector"), lb.GridConfig(64, 4e-9))
    with pytest.raises(ValueError, match="scalar thin-mask"):
        lb.SOCSKernels.build(lb.OpticsConfig(mask_model="fdtd"), lb.GridConfig(64, 4e-9))


def test_wrong_mask_shape(lb):
    k = lb.SOCSKernels.build(lb.OpticsConfig(), lb.GridConfig(64, 4e-9))
    with pytest.raises(ValueError, match="mask must be"):
        k.raw(np.zeros((32, 32)))


def _socs_raw_build(lb, o, n, px, mode):
    import ctypes as C
    import torch
    from lithobat_b200 import _native as nat
    from lithobat_b200.hopkins import aperture_mask, band_bins
    v = lb.config.optics_view(o)
    src = lb.source_points(o)
    kx, ky, fxb, fyb = band_bins(n, px, v.NA / v.wavelength)
    inside = aperture_mask(fxb, fyb, src, v.NA / v.wavelength)
    L = nat.lib()
    dev = torch.device("cuda", 0)
    pupil = np.zeros(1, dtype=nat.PUPIL_DTYPE)
    pupil["wavelength"], pupil["NA"], pupil["defocus"], pupil["n_image"] = v.wavelength, v.NA, v.defocus, v.image_index
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    S, nb = len(src), kx.size
    ws_b = C.c_size_t(0)
    nat.check("ws", L.litho_socs_workspace(S, nb, C.byref(ws_b)))
    ws = torch.empty(ws_b.value, dtype=torch.uint8, device=dev)
    phi = torch.empty((S, nb), dtype=torch.complex128, device=dev)
    lam = torch.empty(S, dtype=torch.float64, device=dev)
    ldg = S + (S & 1)
    G = torch.empty((ldg, ldg), dtype=torch.complex128, device=dev)
    keep = [t(pupil.view(np.uint8)), t(src.fx), t(src.fy), t(src.weight), t(kx), t(ky), t(inside)]
    nat.check("build", L.litho_socs_build(*[k.data_ptr() for k in keep[:4]], S, keep[4].data_ptr(),
                                          keep[5].data_ptr(), nb, keep[6].data_ptr(), n, px, mode, phi.data_ptr(),
                                          lam.data_ptr(), G.data_ptr(), ws.data_ptr(), ws.numel(),
                                          torch.cuda.current_stream().cuda_stream))
    sw = C.c_int(0)
    st = L.litho_socs_status(S, nb, ws.data_ptr(), C.byref(sw), torch.cuda.current_stream().cuda_stream)
    H = torch.empty((ldg, ldg), dtype=torch.complex128, device=dev)
    V = torch.empty((ldg, ldg), dtype=torch.complex128, device=dev)
    E = torch.empty(ldg, dtype=torch.float64, device=dev)
    nat.check("debug", L.litho_socs_debug(S, nb, ws.data_ptr(), H.data_ptr(), V.data_ptr(), E.data_ptr(),
                                          torch.cuda.current_stream().cuda_stream))
    _socs_raw_build.last = (H.cpu().numpy(), V.cpu().numpy(), E.cpu().numpy())
    return G[:S, :S].cpu().numpy(), lam.cpu().numpy(), phi.cpu().numpy(), int(sw.value), st


@pytest.mark.parametrize("mode", [1, 0])
def test_eigensolver_on_a_degenerate_source(lb, mode):
    """Conventional source: many exactly degenerate eigenvalues."""
    from oracle import litho_oracle as O
    o = lb.OpticsConfig(NA=0.93, sigma_outer=0.8, source_grid=9)
    G, lam, phi, sweeps, st = _socs_raw_build(lb, o, 64, 4e-9, mode)
    assert st == 0
    A, band, src = O.socs_pupil_matrix(o, lb.GridConfig(64, 4e-9))
    G_ref = A.conj() @ A.T
    assert np.abs(G - G_ref).max() <= (1e-12 if mode == 1 else 2e-6) * np.abs(G_ref).max()
    ev = np.sort(np.linalg.eigvalsh(G_ref))[::-1]
    got = np.sort(lam)[::-1]
    H, V, E = _socs_raw_build.last
    S = G.shape[0]
    Vs = V[:S, :S]
    offd = np.abs(H - np.diag(np.diag(H))).max()
    assert offd < 1e-12 * ev[0]
    assert sweeps < 40, sweeps
    assert np.abs(V.conj().T @ V - np.eye(len(V))).max() < 1e-12          # V stays unitary
    assert np.abs(Vs.conj().T @ G @ Vs - H[:S, :S]).max() < 1e-12 * ev[0]  # V^H G V = H
    # Jacobi eigenvalues of the Gram as assembled (TF32 split: ~1e-7 of the largest)
    np.testing.assert_allclose(np.sort(E[:S])[::-1], ev, rtol=0, atol=(1e-12 if mode == 1 else 1e-6) * ev[0])
    # the Rayleigh quotients with the exact A are FP64-accurate in either mode
    np.testing.assert_allclose(got, ev, rtol=0, atol=1e-12 * ev[0])
