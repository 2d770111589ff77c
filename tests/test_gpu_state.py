"""State snapshots (cfd_batch_get_state / cfd_batch_set_state).

The resident state of every case (u, v, p, T, up, vp and the reference's int time)
crosses PCIe as one packed copy per direction. Restoring a snapshot and stepping
reproduces the steps taken from it bit for bit, in the same batch and in a fresh batch
of the same cases.
"""
import numpy as np
import pytest
import torch

from cfd_solver_b200.grid import cavity, ogrid

pytestmark = pytest.mark.gpu
FIELDS = ("u", "v", "p", "T", "up", "vp")


def _cases():
    from cfd_solver_b200.solver import case_params
    gs = [ogrid(65, 33, skew=0.1), cavity(49, 49, skew=0.12), ogrid(33, 25)]
    ps = [case_params(gs[0], Re=200.0, Ri=1.0, dt=1e-3), case_params(gs[1], Re=150.0, Ri=0.5, dt=2e-3),
          case_params(gs[2], Re=80.0, dt=2e-3)]
    return gs, ps


def _fields(b, n):
    return [{k: b.plane(c, k) for k in FIELDS} for c in range(n)]


def test_snapshot_round_trip_is_exact():
    from cfd_solver_b200.solver import Batch
    gs, ps = _cases()
    with Batch(gs, ps) as a:
        a.step(3)
        snap = torch.empty(a.state_bytes(), dtype=torch.uint8, pin_memory=True)
        a.get_state(snap)
        before = _fields(a, len(gs))
        a.step(4)
        ref = _fields(a, len(gs))
        a.set_state(snap)
        for f0, f1 in zip(before, _fields(a, len(gs))):
            for k in FIELDS:
                np.testing.assert_array_equal(f1[k], f0[k], err_msg=k)
        a.step(4)
        again = _fields(a, len(gs))
    with Batch(gs, ps) as fresh:
        fresh.set_state(snap)
        fresh.step(4)
        other = _fields(fresh, len(gs))
    for r, x, y in zip(ref, again, other):
        for k in FIELDS:
            np.testing.assert_array_equal(x[k], r[k], err_msg=k)
            np.testing.assert_array_equal(y[k], r[k], err_msg=k)


def test_checkpoint_file_restart_is_exact(tmp_path):
    from cfd_solver_b200 import _lib
    from cfd_solver_b200.solver import Batch
    gs, ps = _cases()
    ck = tmp_path / "state.ckpt"
    with Batch(gs, ps) as a:
        a.step(5)
        a.save(ck)
        a.step(4)
        ref = _fields(a, len(gs))
        ref_st = [a.stats(c) for c in range(len(gs))]
    with Batch(gs, ps) as fresh:
        fresh.load(ck)
        fresh.step(4)
        got = _fields(fresh, len(gs))
        got_st = [fresh.stats(c) for c in range(len(gs))]
    for r, x, sr, sx in zip(ref, got, ref_st, got_st):
        for k in FIELDS:
            np.testing.assert_array_equal(x[k], r[k], err_msg=k)
        # counters and relative residuals continue where they were
        assert sx["steps"] == sr["steps"] == 9
        assert sx["steady_res_rel"] == sr["steady_res_rel"]
    # a corrupt file or another batch is rejected and leaves the batch untouched
    raw = bytearray(ck.read_bytes())
    raw[100] ^= 0xFF
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(bytes(raw))
    with Batch(gs, ps) as other:
        with pytest.raises(_lib.CfdError, match="corrupt"):
            other.load(bad)
    with Batch(gs[:2], ps[:2]) as other:
        with pytest.raises(_lib.CfdError, match="does not match"):
            other.load(ck)
    # the same sizes, profiles and precision on another grid (another skew) are rejected too
    moved = [ogrid(g.n0, g.n1, skew=0.17) if g.kind == "ogrid" else cavity(g.n0, g.n1, skew=0.17) for g in gs]
    with Batch(moved, ps) as other:
        with pytest.raises(_lib.CfdError, match="another grid"):
            other.load(ck)


def test_state_image_layout():
    """The image holds, per case, u, v, p, T, up, vp as n1 rows of the stored columns (n0 - 1
    for the periodic O-grid, n0 for the cavity), then 16 doubles of counters."""
    from cfd_solver_b200.solver import Batch
    gs, ps = _cases()
    with Batch(gs, ps) as a:
        a.step(3)
        img = np.empty(a.state_bytes(), dtype=np.uint8)
        a.get_state(img)
        fields = _fields(a, len(gs))
    words = img.view(np.float64)
    o = 0
    for g, f in zip(gs, fields):
        nc = g.n0 - 1 if g.kind == "ogrid" else g.n0
        for k in FIELDS:
            got = words[o:o + g.n1 * nc].reshape(g.n1, nc)
            np.testing.assert_array_equal(got, f[k][:, :nc], err_msg=k)
            o += g.n1 * nc
        counters = words[o:o + 16]
        assert counters[:1].view(np.int32)[1] == 3  # steps taken
        o += 16
    assert o * 8 == img.size
