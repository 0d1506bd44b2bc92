"""The multi-GPU paths' host logic (one process per GPU), tested with gloo on CPU.

The imaging engine itself needs a GPU; these tests run what surrounds it,
with two processes, gloo and 127.0.0.1:

* clip sharding: the shard plan, the ordered tensor all-gather (uneven clip
  sizes) and the failure of a rank, with a stand-in per-clip function;
* one image split by source points: each rank's share of the Abbe sum comes
  from the FP64 oracle (the reference's algorithm over that rank's source
  points), the shares are all-reduced, and the result must be the whole sum;
* one ILT clip split by SOCS kernels: each rank's forward and adjoint parts
  come from the oracle's dense SOCS with that rank's kernels, and the split
  objective must equal the whole objective and gradient.
"""

from __future__ import annotations

import os
import socket
import tempfile

import numpy as np
import pytest

from lithobat_b200.distributed import (clip_cost, contiguous_ranges, gather_results, gather_tensors, kernel_ranges,
                                      run_sharded, shard_plan, source_ranges, split_abbe_image,
                                      split_socs_objective)


def test_shard_plan_covers_every_clip_once_and_balances_uneven_sizes():
    rng = np.random.default_rng(0)
    sizes = rng.choice([256, 512, 1024, 2048], size=256, p=[0.4, 0.3, 0.2, 0.1])
    costs = [clip_cost(int(n), 204) for n in sizes]
    for world in (1, 2, 4, 8):
        parts = shard_plan(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.05 * (sum(costs) / world) + max(costs)
        assert all(p == sorted(p) for p in parts)
    assert shard_plan(costs, 4) == shard_plan(list(costs), 4)   # deterministic


def test_shard_plan_with_more_ranks_than_clips():
    parts = shard_plan([1.0, 2.0], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir, fail_rank):
    from datetime import timedelta

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=10))
    try:
        rng = np.random.default_rng(1)
        clips = [rng.random((n, n)) for n in (8, 16, 8, 32, 16, 8, 24)]
        costs = [clip_cost(c.shape[0]) for c in clips]

        def fn(batch):
            if rank == fail_rank:
                raise RuntimeError("injected failure on this rank")
            return [float(c.sum()) * 2.0 for c in batch]

        try:
            mine, res = run_sharded(clips, costs, fn, rank, world)
            full = gather_results(len(clips), mine, res)
            np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array(full))
        except Exception as e:  # noqa: BLE001 — reported to the parent through a file
            with open(os.path.join(out_dir, f"rank{rank}.err"), "w") as f:
                f.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


def _spawn(world, fail_rank):
    import torch.multiprocessing as mp
    out = tempfile.mkdtemp()
    mp.start_processes(_worker, args=(world, _free_port(), out, fail_rank), nprocs=world, join=True,
                       start_method="spawn")
    return out


def test_two_ranks_gather_results_in_input_order():
    out = _spawn(2, fail_rank=-1)
    rng = np.random.default_rng(1)
    clips = [rng.random((n, n)) for n in (8, 16, 8, 32, 16, 8, 24)]
    want = np.array([float(c.sum()) * 2.0 for c in clips])
    for r in range(2):
        got = np.load(os.path.join(out, f"rank{r}.npy"))
        np.testing.assert_array_equal(got, want)


def test_a_failing_rank_is_reported_on_every_rank():
    """Rank 1 raises before the exchange: it reports its own error, and rank 0's
    gather ends with an error (peer gone / timeout) instead of hanging."""
    out = _spawn(2, fail_rank=1)
    errs = {r: open(os.path.join(out, f"rank{r}.err")).read() for r in range(2)
            if os.path.exists(os.path.join(out, f"rank{r}.err"))}
    assert "injected failure" in errs.get(1, "")
    assert 0 in errs, "rank 0 must see the failure of rank 1"
    assert not os.path.exists(os.path.join(out, "rank0.npy"))


def test_contiguous_ranges_partition_in_order():
    for count in (0, 1, 5, 24, 400):
        for world in (1, 2, 3, 8):
            r = contiguous_ranges(count, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == count
            assert all(a <= b for a, b in r) and all(r[i][1] == r[i + 1][0] for i in range(world - 1))
            lens = [b - a for a, b in r]
            assert max(lens) - min(lens) <= 1
    assert source_ranges(400, 3) == [(0, 134), (134, 267), (267, 400)]
    assert kernel_ranges(24, 5)[0] == (0, 5) and kernel_ranges(24, 5)[-1] == (20, 24)
    with pytest.raises(ValueError):
        contiguous_ranges(4, 0)


def _split_worker(rank, world, port, out_dir, case):
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=30))
    try:
        if case == "gather":
            sizes = [8, 16, 8, 32, 16, 8, 24]
            costs = [clip_cost(n) for n in sizes]
            mine = shard_plan(costs, world)[rank]
            res = [torch.full((sizes[i], sizes[i]), float(i), dtype=torch.complex64) * (1 + 2j) for i in mine]
            full = gather_tensors(len(sizes), mine, res)
            np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                    np.array([complex(t.sum()) / t.numel() for t in full]))
            np.save(os.path.join(out_dir, f"shapes{rank}.npy"), np.array([t.shape[0] for t in full]))
        elif case == "abbe":
            from conftest import ns_grid, ns_optics
            from oracle import litho_oracle as O
            od = dict(wavelength=193e-9, NA=1.35, n_immersion=1.44, n_image=None, source_type="annular",
                      sigma_inner=0.5, sigma_outer=0.9, source_grid=11, imaging_model="vector", polarisation="te",
                      defocus=20e-9, zernike_coeffs={7: 0.02}, normalisation="peak")
            o, g = ns_optics(od), ns_grid({"n_pixels": 64, "pixel_size": 4e-9})
            mask = O.to_attenuated_psm(1.0 - O.contact_array(64, 4e-9, 100e-9, 100e-9, 50e-9))
            planes = [(o.defocus, o.image_index)]
            S = len(O.source_points(o))

            def partial(rng):
                raw, _, _ = O.abbe_sum(mask, o, g, planes, source_subset=range(*rng))
                return torch.from_numpy(raw[0].copy())
            img = split_abbe_image(partial, lambda t: t, S, None)
            np.save(os.path.join(out_dir, f"rank{rank}.npy"), img.numpy())
        elif case == "socs":
            from conftest import ns_grid, ns_optics
            from oracle import litho_oracle as O
            od = dict(wavelength=193e-9, NA=1.35, n_immersion=1.44, n_image=None, source_type="annular",
                      sigma_inner=0.5, sigma_outer=0.8, source_grid=11, normalisation="clear")
            o, g = ns_optics(od), ns_grid({"n_pixels": 64, "pixel_size": 2e-9})
            full = O.socs_build(o, g, tol=0.0, max_kernels=12)
            a, b = kernel_ranges(len(full), world)[rank]
            part = O.SOCS(full.kernels[a:b], full.weights[a:b], full.clear, full.energy_kept, full.n_band,
                          full.n_source, full.band, full.n, full.normalisation)
            rng = np.random.default_rng(3)
            target = O.lines_and_spaces(64, 2e-9, 40e-9, 20e-9)
            mask = O.mask_of(0.5 * rng.standard_normal((64, 64)), 4.0, 0.0)
            np.save(os.path.join(out_dir, "inputs.npy"), np.stack([target, mask]))
            engine = _DenseSocsPart(O, part, target, 1.0 / full.clear, 0.3, 1.0, 15.0)
            cost, grad = split_socs_objective(engine, mask, None)
            np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.concatenate([[cost], grad.numpy().ravel()]))
    except Exception as e:  # noqa: BLE001 — reported to the parent through a file
        with open(os.path.join(out_dir, f"rank{rank}.err"), "w") as f:
            f.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:  # noqa: BLE001
            pass


class _DenseSocsPart:
    """The FP64 dense SOCS of some kernels (the oracle's socs_fields and
    socs_gradient) behind split_socs_objective's engine interface; the
    objective is opc/ilt.py:313-336 without blur (sigma 0)."""

    def __init__(self, O, part, target, scale, level, sign, steepness):
        self.O, self.k, self.t = O, part, target
        self.scale, self.level, self.sign, self.a = scale, level, sign, steepness / abs(level)

    def forward(self, mask):
        import torch
        self.fields, inten = self.O.socs_fields(self.k, mask)
        return torch.from_numpy(inten.copy())

    def objective(self, inten):
        import torch
        signed = self.sign * (inten.numpy() * self.scale - self.level)
        z = 1.0 / (1.0 + np.exp(-np.clip(self.a * signed, -60.0, 60.0)))
        resid = z - self.t
        npix = float(resid.size)
        dz = (2.0 / npix) * resid * (self.a * z * (1.0 - z))
        return float(np.sum(resid ** 2) / npix), self.sign * dz * self.scale

    def adjoint(self, sens):
        import torch
        return torch.from_numpy(self.O.socs_gradient(self.k, self.fields, sens).copy())

    def gradient(self, q):
        return q


def _spawn_case(world, case):
    import torch.multiprocessing as mp
    out = tempfile.mkdtemp()
    mp.start_processes(_split_worker, args=(world, _free_port(), out, case), nprocs=world, join=True,
                       start_method="spawn")
    errs = [open(os.path.join(out, f)).read() for f in os.listdir(out) if f.endswith(".err")]
    assert not errs, errs
    return out


def test_tensor_all_gather_of_uneven_complex_results_in_input_order():
    out = _spawn_case(2, "gather")
    sizes = [8, 16, 8, 32, 16, 8, 24]
    for r in range(2):
        np.testing.assert_array_equal(np.load(os.path.join(out, f"rank{r}.npy")),
                                      np.arange(7) * (1 + 2j))
        np.testing.assert_array_equal(np.load(os.path.join(out, f"shapes{r}.npy")), sizes)


def test_one_image_split_by_source_points_equals_the_whole_sum():
    """Vector TE with defocus and coma, 121-point grid: two ranks each sum
    their half of the source points; the all-reduced image is the oracle's
    whole Abbe sum (to FP64 summation order) on both ranks."""
    from conftest import ns_grid, ns_optics
    from oracle import litho_oracle as O
    out = _spawn_case(2, "abbe")
    od = dict(wavelength=193e-9, NA=1.35, n_immersion=1.44, n_image=None, source_type="annular",
              sigma_inner=0.5, sigma_outer=0.9, source_grid=11, imaging_model="vector", polarisation="te",
              defocus=20e-9, zernike_coeffs={7: 0.02}, normalisation="peak")
    o, g = ns_optics(od), ns_grid({"n_pixels": 64, "pixel_size": 4e-9})
    mask = O.to_attenuated_psm(1.0 - O.contact_array(64, 4e-9, 100e-9, 100e-9, 50e-9))
    whole = O.abbe_sum(mask, o, g, [(o.defocus, o.image_index)])[0][0]
    for r in range(2):
        img = np.load(os.path.join(out, f"rank{r}.npy"))
        assert np.abs(img - whole).max() <= 1e-12 * np.abs(whole).max()


def test_one_ilt_clip_split_by_kernels_equals_the_whole_objective():
    """K = 12 kernels over two ranks: the partial images and gradients are
    all-reduced; cost and gradient equal the oracle's whole objective."""
    from conftest import ns_grid, ns_optics
    from oracle import litho_oracle as O
    out = _spawn_case(2, "socs")
    target, mask = np.load(os.path.join(out, "inputs.npy"))
    od = dict(wavelength=193e-9, NA=1.35, n_immersion=1.44, n_image=None, source_type="annular",
              sigma_inner=0.5, sigma_outer=0.8, source_grid=11, normalisation="clear")
    o, g = ns_optics(od), ns_grid({"n_pixels": 64, "pixel_size": 2e-9})
    full = O.socs_build(o, g, tol=0.0, max_kernels=12)
    cost, grad, _, _ = O.objective(full, target, mask, 1.0 / full.clear, 0.3, 0.0, 1.0, 15.0)
    for r in range(2):
        got = np.load(os.path.join(out, f"rank{r}.npy"))
        assert abs(got[0] - cost) <= 1e-12 * abs(cost)
        assert np.abs(got[1:].reshape(64, 64) - grad).max() <= 1e-10 * np.abs(grad).max()
