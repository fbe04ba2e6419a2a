"""The input path to the device (ndb_b200_load_bin, ndb_b200_run_loaded): the
reference's .bin layout (magma_input.h:113-125) read through pinned chunks whose
copies overlap the reads and whose bounding box is reduced as they land.  The
loaded run must equal ndb_b200_run on the same coordinates, and bad files must give
statuses, not crashes.  Also the batched form on host buffers, whose copies to and
from the device overlap the other groups' compute: its outputs must equal the
device-buffer batch."""
import struct

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,n,full", [(1, 100_000, True), (2, 3_000_000, False), (3, 200_000, True)])
def test_loaded_run_equals_run(ctx, pkg, tmp_path, cfg, n, full):
    w = pkg.synthetic.make(cfg, n=n)
    p = tmp_path / "in.bin"
    pkg.inputs.write_bin(str(p), w.coords)
    nn1, ci1, r1 = ctx.run(w.coords, w.eps, w.min_pts, full_count=full)
    assert ctx.load_bin(str(p)) == (w.n, w.d)
    for _ in range(2):  # the loaded job stays for further runs
        nn, ci, r = ctx.run_loaded(w.eps, w.min_pts, full_count=full)
        np.testing.assert_array_equal(ci, ci1)
        if full:
            np.testing.assert_array_equal(nn, nn1)
        else:
            below = nn1 < w.min_pts
            np.testing.assert_array_equal(nn[below], nn1[below])
            np.testing.assert_array_equal(nn >= w.min_pts, nn1 >= w.min_pts)
        assert r == r1


def test_loaded_golden_fixtures(ctx, pkg, tmp_path):
    for name in ("specials_m1", "c1_n4000", "blobs_d16", "n1"):
        g = load_golden(name)
        p = tmp_path / f"{name}.bin"
        pkg.inputs.write_bin(str(p), g["coords"])
        ctx.load_bin(str(p))
        nn, ci, r = ctx.run_loaded(float(g["eps"]), int(g["min_pts"]), full_count=True)
        np.testing.assert_array_equal(nn, g["nn"], err_msg=name)
        np.testing.assert_array_equal(ci, g["cluster_index"], err_msg=name)


def test_load_errors(ctx, pkg, tmp_path):
    with pytest.raises(pkg.lib.NdbError) as ei:
        ctx.load_bin(str(tmp_path / "missing.bin"))
    assert ei.value.status == 11
    short = tmp_path / "short.bin"
    short.write_bytes(struct.pack("<ii", 10, 3) + b"\0" * 8)
    with pytest.raises(pkg.lib.NdbError) as ei:
        ctx.load_bin(str(short))
    assert ei.value.status == 11
    bad_d = tmp_path / "d17.bin"
    bad_d.write_bytes(struct.pack("<ii", 1, 17) + b"\0" * 68)
    with pytest.raises(pkg.lib.NdbError) as ei:
        ctx.load_bin(str(bad_d))
    assert ei.value.status == 2
    with pytest.raises(pkg.lib.NdbError) as ei:  # nothing loaded after a failed load
        ctx.run_loaded(1.0, 4)
    assert ei.value.status == 9
    # a host run overwrites the loaded copy
    g = load_golden("c1_n4000")
    p = tmp_path / "ok.bin"
    pkg.inputs.write_bin(str(p), g["coords"])
    ctx.load_bin(str(p))
    ctx.run(g["coords"], float(g["eps"]), int(g["min_pts"]))
    with pytest.raises(pkg.lib.NdbError):
        ctx.run_loaded(float(g["eps"]), int(g["min_pts"]))


def test_batched_host_buffers_overlap_equals_device_batch(ctx, pkg):
    import torch
    jobs = pkg.synthetic.config4(n_jobs=96, seed=21, n_min=1000, n_max=30000)
    host = ctx.run_batched([(j.coords, j.eps, j.min_pts) for j in jobs])
    for j, (nn, ci, res) in zip(jobs, host):
        x = torch.from_numpy(j.coords).cuda()
        nn_d = torch.empty(j.n, dtype=torch.int32, device="cuda")
        ci_d = torch.empty(j.n, dtype=torch.int32, device="cuda")
        r = ctx.run_device(x.data_ptr(), j.n, j.d, j.eps, j.min_pts, nn_d.data_ptr(), ci_d.data_ptr())
        torch.cuda.synchronize()
        np.testing.assert_array_equal(ci, ci_d.cpu().numpy())
        below = nn < j.min_pts
        np.testing.assert_array_equal(below, nn_d.cpu().numpy() < j.min_pts)
        np.testing.assert_array_equal(nn[below], nn_d.cpu().numpy()[below])
        assert res == r
