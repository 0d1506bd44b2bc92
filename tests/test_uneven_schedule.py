"""The uneven work queue's schedule (litho_uneven_schedule, host only): every
dependency points to an earlier task, waits cover all the tasks they wait
for, pass A covers every job once, pass B every (work item, row block) once,
and no pass-A task can overwrite a buffer slot before the previous chunk's
pass-B tasks finished with it. Runs on the CPU (no device pointers needed)."""

from __future__ import annotations

import ctypes as C
import random

import numpy as np
import pytest

from lithobat_b200 import _native as nat
from lithobat_b200.aerial import plan_abbe
from lithobat_b200.config import OpticsConfig, optics_view
from lithobat_b200.source import Source
from lithobat_b200.uneven import queue_schedule


def _groups(sizes_counts, items=8, **tune):
    o = OpticsConfig(wavelength=13.5e-9, NA=0.33, source_grid=15,
                     source_spec=Source.dipole(0.9, 0.6, opening_deg=60).to_dict())
    v = optics_view(o)
    out, keep = [], []
    for n, count in sizes_counts:
        pd = plan_abbe([v] * count, n, 2e-9, [[(v.defocus, v.image_index)]] * count, 1.0, False, False,
                       items_per_job_group=items)
        keep.append(pd)
        out.append(nat.UnevenGroup(plan=pd.plan, blob_host=pd.blob.ctypes.data, **tune))
    return (nat.UnevenGroup * len(out))(*out), keep


def _items(pd):
    return pd.blob[pd.plan.off_items:pd.plan.off_items + pd.plan.n_items * 16].view(nat.ITEM_DTYPE)


@pytest.mark.parametrize("tune", [{}, {"slot_kib": 2048, "n_slots": 2, "b_rows": 2, "a_units": 48},
                                  {"slot_kib": 65536, "n_slots": 4, "b_rows": 4, "a_units": 192}])
def test_schedule_dependencies_and_coverage(tune):
    L = nat.lib()
    arr, pds = _groups([(256, 3), (512, 3), (1024, 2), (2048, 1)], **tune)
    tasks, n_ctr = queue_schedule(L, arr)
    assert tasks.size > 0 and n_ctr > 0
    # every wait refers to a counter all of whose signalling tasks come earlier,
    # and waits for all of them
    signals: dict = {}
    for k, t in enumerate(tasks):
        signals.setdefault(int(t["done_ctr"]), []).append(k)
    for k, t in enumerate(tasks):
        c = int(t["wait_ctr"])
        if c < 0:
            continue
        before = signals.get(c, [])
        assert int(t["wait_value"]) == len(before) > 0
        assert max(before) < k
    # the wide groups, largest coarse grid first (the 256^2 group runs on chip)
    wide = [pd for pd in pds if pd.plan.L > 64]
    order = sorted(range(len(wide)), key=lambda i: -wide[i].plan.L)
    assert sorted(set(int(g) for g in tasks["group"])) == list(range(len(wide)))
    for gq, gi in enumerate(order):
        pd = wide[gi]
        p = pd.plan
        mine = tasks[tasks["group"] == gq]
        a = mine[mine["kind"] == 0]
        covered = np.zeros(p.n_jobs, dtype=np.int32)
        for t in a:
            covered[t["first"]:t["first"] + t["count"]] += 1
            assert t["first"] >= t["base"]
        assert np.all(covered == 1)
        b = mine[mine["kind"] == 1]
        lpw = 1024 // p.L
        row_blocks = p.L // (8 * lpw)
        seen = np.zeros((p.n_items, row_blocks), dtype=np.int32)
        items = _items(pd)
        for t in b:
            seen[t["first"], t["count"]:t["count"] + t["rows"]] += 1
            it = items[t["first"]]
            # the item's jobs lie in the chunk that owns the slot
            chunk_a = a[(a["slot"] == t["slot"]) & (a["base"] == t["base"])]
            lo = int(chunk_a["first"].min())
            hi = int((chunk_a["first"] + chunk_a["count"]).max())
            assert lo == t["base"] and lo <= it["job_begin"] and it["job_end"] <= hi
        assert np.all(seen == 1)


def test_slot_reuse_waits_for_the_previous_chunk():
    L = nat.lib()
    arr, _ = _groups([(512, 4)], slot_kib=1024, n_slots=2)
    tasks, _ = queue_schedule(L, arr)
    chunks = sorted(set(int(b) for b in tasks["base"]))
    assert len(chunks) >= 3
    for ci, base in enumerate(chunks):
        a = tasks[(tasks["kind"] == 0) & (tasks["base"] == base)]
        assert len(set(int(s) for s in a["slot"])) == 1
        if ci < 2:
            assert np.all(a["wait_ctr"] == -1)
            continue
        prev_b = tasks[(tasks["kind"] == 1) & (tasks["base"] == chunks[ci - 2])]
        assert int(prev_b["slot"][0]) == int(a["slot"][0])
        assert np.all(a["wait_ctr"] == prev_b["done_ctr"][0])
        assert np.all(a["wait_value"] == len(prev_b))


def test_in_order_dequeue_never_deadlocks():
    """Blocks that take tasks in list order and wait on counters finish with
    any number of blocks and any completion order."""
    L = nat.lib()
    arr, _ = _groups([(512, 3), (1024, 2)], slot_kib=1024, n_slots=2)
    tasks, n_ctr = queue_schedule(L, arr)
    rng = random.Random(5)
    for blocks in (1, 2, 7):
        ctr = [0] * n_ctr
        head, running, done = 0, [], 0
        while done < len(tasks):
            while len(running) < blocks and head < len(tasks):
                running.append(head)
                head += 1
            ready = [k for k in running if tasks[k]["wait_ctr"] < 0 or
                     ctr[tasks[k]["wait_ctr"]] >= tasks[k]["wait_value"]]
            assert ready, "every running block waits: deadlock"
            k = rng.choice(ready)
            running.remove(k)
            ctr[tasks[k]["done_ctr"]] += 1
            done += 1


def test_group_workspace_and_rejections():
    L = nat.lib()
    arr, pds = _groups([(512, 2)])
    nb = C.c_size_t(0)
    assert L.litho_uneven_group_workspace(C.byref(arr[0]), C.byref(nb)) == 0 and nb.value > 0
    small = C.c_size_t(0)
    arr2, _ = _groups([(512, 2)], slot_kib=1024)
    assert L.litho_uneven_group_workspace(C.byref(arr2[0]), C.byref(small)) == 0 and small.value < nb.value
    bad, _ = _groups([(512, 2)], n_slots=1)
    nt, nc = C.c_int(0), C.c_int(0)
    assert L.litho_uneven_schedule(bad, 1, None, 0, C.byref(nt), C.byref(nc)) == -2   # LITHO_E_SIZE
    arr[0].blob_host = None
    assert L.litho_uneven_schedule(arr, 1, None, 0, C.byref(nt), C.byref(nc)) == -1   # LITHO_E_NULL
    # a buffer shorter than the schedule is refused
    tasks, _ = queue_schedule(L, arr2)
    buf = np.zeros(max(1, tasks.size - 1), dtype=nat.QUEUE_TASK_DTYPE)
    assert L.litho_uneven_schedule(arr2, 1, buf.ctypes.data, buf.size, C.byref(nt), C.byref(nc)) == -2
