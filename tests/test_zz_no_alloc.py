"""ov_direct_points_noalloc, the point query for callers that cannot allocate
device memory (their device memory belongs to another framework's allocator,
or they run in a loop that must not allocate).  It must give the same
velocities as the allocating query, ov_state_eval_points with the direct
sum, within the FP64 tolerance of the other GPU tests, on consecutive calls
that share its fixed scratch array.  The test allocates the input and output
buffers itself (through torch); the entry point allocates nothing.

Kept in a file of its own that pytest collects last."""
import numpy as np
import pytest

from cases import load, rel_err

pytestmark = pytest.mark.gpu

TOL_V64 = 1e-12


def test_no_alloc_matches_direct_point_query():
    import torch

    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    t, p, _, _ = load("periodic26_direct")
    ov.configure(p, ov.OV_PREC_FP64)
    t.set_images_from_library(lib)
    st = ov.DeviceState(t.copy())
    dev = torch.device("cuda", 0)
    d_pos = torch.from_numpy(np.ascontiguousarray(t.pos)).to(dev)
    d_links = torch.from_numpy(np.ascontiguousarray(t.links)).to(dev)
    d_status = torch.from_numpy(np.ascontiguousarray(t.stat)).to(dev)
    rng = np.random.default_rng(3)
    nodes = rng.choice(t.n, 300, replace=False).astype(np.int32)
    calls = [(rng.uniform(0.0, 0.1, size=(257, 3)), None),       # arbitrary points
             (t.pos[nodes].copy(), nodes)]                       # nodes, skipping themselves
    for pts, skip in calls:
        want = st.eval_points(pts, skip, method=0)
        d_pts = torch.from_numpy(np.ascontiguousarray(pts)).to(dev)
        d_skip = None if skip is None else torch.from_numpy(skip).to(dev)
        d_out = torch.full_like(d_pts, float("nan"))
        torch.cuda.synchronize()
        rc = lib.ov_direct_points_noalloc(t.ptr(), d_pos.data_ptr(), d_links.data_ptr(),
                                          d_status.data_ptr(), len(pts), d_pts.data_ptr(),
                                          None if d_skip is None else d_skip.data_ptr(),
                                          d_out.data_ptr(), None)
        assert rc == 0, lib.ov_last_error_message()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < TOL_V64
    st.close()


def test_no_alloc_rejects_sizes_beyond_its_scratch(monkeypatch):
    """Sizes beyond the stated maximum are refused before any GPU work."""
    import torch

    import openvort_b200 as ov
    monkeypatch.setenv("OV_QUIET", "1")
    lib = ov.load()
    assert lib.ov_init(0) == 0
    t, p, _, _ = load("ring256")
    ov.configure(p, ov.OV_PREC_FP64)
    dev = torch.device("cuda", 0)
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    t.struct.N = 131072 + 1   # OV_NOALLOC_MAX_NODES + 1
    rc = lib.ov_direct_points_noalloc(t.ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 1,
                                      buf.data_ptr(), None, buf.data_ptr(), None)
    t.struct.N = t.n
    assert rc == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
    rc = lib.ov_direct_points_noalloc(t.ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                      131072 + 1, buf.data_ptr(), None, buf.data_ptr(), None)
    assert rc == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
