"""GPU: the reference's own C linked against libov_gpu.so.

oracle/_ref/ov_linked_gpu is the reference's main loop (reconnect,
eliminate_small_loops, update_tangle, rk4_step, update_tangents_normals,
remesh, enforce_boundaries; src/main.c:96-118) compiled from the reference's
sources with the hot-path functions renamed in src/tangle.c and
src/vortex_dynamics.c and src/octree.c left out, linked against the GPU
library: update_tangle, rk4_step and the single-node update_velocity of
reconnect (src/vortex_dynamics.c:275-276) resolve to the library.  The same
loop built from the unmodified sources (ov_linked_ref) is the reference.
5 steps of a 40-ring periodic tangle with Barnes-Hut theta 0.4, remeshing
and reconnections: the same reconnections, links and status, and positions
within 1e-12 of the box."""
import numpy as np
import pytest

from cases import pos_err
from linked import GPU_EXE, REF_EXE, run, write_input
from openvort_b200 import geometry as G

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not (REF_EXE.exists() and GPU_EXE.exists()),
                    reason="linked programs not built (they need the reference sources)")
def test_reference_main_loop_linked_against_the_gpu_library(tmp_path):
    t = G.random_ring_tangle(3, 40, 0.1, dl=5e-4, boundary="periodic-26")
    inp = tmp_path / "in.bin"
    write_input(inp, t, steps=5, use_bh=1, theta=0.4, dt=2e-5, rec_dist=1.5e-3, rec_angle=0.5,
                dl_min=0.6 * 5e-4, dl_max=2.5 * 5e-4, core_a=1e-8, alpha=0.098, alpha_p=0.016,
                vn=(0.5, 0.0, 0.0))
    ref = run(REF_EXE, inp, tmp_path / "ref.bin")
    gpu = run(GPU_EXE, inp, tmp_path / "gpu.bin")
    assert ref["recs"] > 0                 # the loop reconnected
    assert gpu["n"] == ref["n"] and gpu["recs"] == ref["recs"]
    for key in ("fwd", "rev", "status"):
        assert np.array_equal(gpu[key], ref[key]), key
    live = ref["status"] != -1
    assert pos_err(gpu["pos"], ref["pos"], live) < 1e-12
