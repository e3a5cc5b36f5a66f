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


# OV_NOALLOC_MAX_POINT_IMAGES: points x (1 + images) the partial sums hold
MAX_POINT_IMAGES = 131072


def _setup(name="periodic26_direct"):
    import torch

    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    t, p, _, _ = load(name)
    ov.configure(p, ov.OV_PREC_FP64)
    t.set_images_from_library(lib)
    dev = torch.device("cuda", 0)
    d_tangle = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (t.pos, t.links, t.stat)]
    return ov, lib, t, dev, d_tangle


def _query(lib, t, d_tangle, d_pts, d_skip, d_out):
    d_pos, d_links, d_status = d_tangle
    return lib.ov_direct_points_noalloc(t.ptr(), d_pos.data_ptr(), d_links.data_ptr(),
                                        d_status.data_ptr(), d_pts.shape[0], d_pts.data_ptr(),
                                        None if d_skip is None else d_skip.data_ptr(),
                                        d_out.data_ptr(), None)


def test_no_alloc_matches_direct_point_query():
    import torch
    ov, lib, t, dev, d_tangle = _setup()
    st = ov.DeviceState(t.copy())
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
        rc = _query(lib, t, d_tangle, d_pts, d_skip, d_out)
        assert rc == 0, lib.ov_last_error_message()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < TOL_V64
    st.close()


def test_no_alloc_at_the_point_image_limit_allocates_nothing():
    """Periodic-26: the most points whose 27 partial sums fit the scratch,
    twice in a row, the second call with the device's free memory and
    torch's allocated bytes read on both sides."""
    import torch
    ov, lib, t, dev, d_tangle = _setup()
    st = ov.DeviceState(t.copy())
    npts = MAX_POINT_IMAGES // 27
    rng = np.random.default_rng(4)
    outs = []
    for call in range(2):
        pts = rng.uniform(0.0, 0.1, size=(npts, 3))
        want = st.eval_points(pts, None, method=0)
        d_pts = torch.from_numpy(pts).to(dev)
        d_out = torch.full_like(d_pts, float("nan"))
        torch.cuda.synchronize()
        free0, alloc0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
        rc = _query(lib, t, d_tangle, d_pts, None, d_out)
        torch.cuda.synchronize()
        free1, alloc1 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
        assert rc == 0, lib.ov_last_error_message()
        if call == 1:     # the first call may load kernels; the second must not change anything
            assert free1 == free0 and alloc1 == alloc0, (free0, free1, alloc0, alloc1)
        got = d_out.cpu().numpy()
        assert np.all(np.isfinite(got))
        assert rel_err(got, want) < TOL_V64
        outs.append(got)
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
    # periodic-26: one point more than the partial sums of 27 images hold
    t26, p26, _, _ = load("periodic26_direct")
    ov.configure(p26, ov.OV_PREC_FP64)
    t26.set_images_from_library(lib)
    rc = lib.ov_direct_points_noalloc(t26.ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                      MAX_POINT_IMAGES // 27 + 1, buf.data_ptr(), None, buf.data_ptr(),
                                      None)
    assert rc == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
