"""The C-ABI boundary on CPU: libov_gpu.so builds, loads and exports every
symbol include/openvort_b200.h declares; struct layouts agree between the
header, the Python mirror and the reference; tables and globals carry the
reference's values; without a GPU every entry point fails loudly (error
status, no CPU fallback)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from openvort_b200 import _lib, geometry as G
from openvort_b200.tangle import (BOUNDARY_SYMBOLS, IMAGE_TABLES, BoundaryImages, NodeStatus,
                                  Neighbour, Params, TangleState, VConf, Vec3d)
from oracle.oracle import REF_SO, REF_SRC, have_ref

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "openvort_b200.h"


def _gpu_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():
        from openvort_b200 import build
        build.build()
    return _lib.load()


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = "\n".join(l for l in text.splitlines() if not l.lstrip().startswith("typedef"))
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", text, flags=re.M):
        name = m.group(1)
        if name not in ("typedef", "struct", "if", "sizeof") and not name.startswith("get_v_t"):
            names.add(name)
    names.discard("get_v_t")
    return sorted(names)


def declared_data():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"^extern\s+(?:const\s+)?[\w\s]+?\b(\w+);", text, flags=re.M)))


def test_header_symbols_exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    funcs = declared_functions()
    data = declared_data()
    assert len(funcs) >= 30 and len(data) >= 25
    missing = [s for s in funcs + data if s not in exported]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(funcs) <= set(_lib.FUNCTIONS) | {"get_v_t"}
    assert set(data) <= set(_lib.DATA)


LAYOUT_C = r"""
#include <stdio.h>
#include <stddef.h>
#include "openvort_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(struct tangle_state),
         offsetof(struct tangle_state, box), offsetof(struct tangle_state, bimg),
         offsetof(struct tangle_state, N), sizeof(struct domain_box), sizeof(struct vec3d),
         sizeof(node_status), sizeof(struct neighbour_t), sizeof(struct boundary_images),
         sizeof(struct v_conf_t), offsetof(struct v_conf_t, v_params));
  return 0;
}
"""


def test_struct_layouts(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(LAYOUT_C)
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    py = [C.sizeof(TangleState), TangleState.box.offset, TangleState.bimg.offset, TangleState.N.offset,
          C.sizeof(TangleState._fields_[10][1]), C.sizeof(Vec3d), C.sizeof(NodeStatus),
          C.sizeof(Neighbour), C.sizeof(BoundaryImages), C.sizeof(VConf), VConf.v_params.offset]
    assert vals == py


@pytest.mark.skipif(not (REF_SRC / "include" / "tangle.h").exists(),
                    reason="reference headers absent ($OPENVORT_REF)")
def test_header_interchangeable_with_reference(tmp_path):
    """The reference's headers and this one compile together in either order."""
    for order in (("tangle.h", "openvort_b200.h"), ("openvort_b200.h", "tangle.h")):
        src = tmp_path / "both.c"
        src.write_text("".join(f'#include "{h}"\n' for h in order) + "int main(void){return 0;}\n")
        subprocess.run(["gcc", "-fsyntax-only", "-I", str(ROOT / "include"),
                        "-I", str(REF_SRC / "include"), str(src)], check=True)


def _table(lib, sym):
    b = BoundaryImages.in_dll(lib, sym)
    return [(tuple(b.images[j].shift), b.images[j].reflect) for j in range(b.n)]


def test_image_tables(lib):
    for name, table in IMAGE_TABLES.items():
        assert _table(lib, BOUNDARY_SYMBOLS[name]) == table
    if have_ref():
        ref = C.CDLL(str(REF_SO))
        for name, sym in BOUNDARY_SYMBOLS.items():
            assert _table(lib, sym) == _table(ref, sym), name


def test_global_defaults(lib):
    """The library's globals start at the reference's defaults
    (src/vortex_constants.c:24-95)."""
    p = Params()
    for sym, attr, ctype in Params.GLOBALS:
        assert ctype.in_dll(lib, sym).value == getattr(p, attr), sym
    if have_ref():
        ref = C.CDLL(str(REF_SO))
        for sym, attr, ctype in Params.GLOBALS:
            assert ctype.in_dll(ref, sym).value == ctype.in_dll(lib, sym).value, sym
    # the colinearity cut-off of the segment formula (src/tangle.c:505-506)
    lib.ov_get_colinear_cutoff.restype = C.c_double
    assert lib.ov_get_colinear_cutoff() == 1e-8


def test_error_strings(lib):
    for code in range(9):
        assert lib.ov_error_string(code)


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly(lib, monkeypatch):
    """Without a device every entry point reports OV_ERR_NO_DEVICE and
    leaves outputs unwritten: there is no CPU fallback."""
    monkeypatch.setenv("OV_QUIET", "1")
    import openvort_b200 as ov
    t = G.single_ring(32, 1e-2)
    ov.configure(Params(use_mf=0, hyperfriction=0))
    t.vels[:] = 7.0
    with pytest.raises(ov.OVError) as e:
        ov.update_velocities(t, 0.0)
    assert e.value.code == _lib.OV_ERR_NO_DEVICE
    assert np.all(t.vels == 7.0)
    with pytest.raises(ov.OVError):
        ov.rk4_step(t, 0.0, 1e-6)
    with pytest.raises(ov.OVError):
        ov.update_tangents_normals(t)
    assert lib.ov_init(0) == _lib.OV_ERR_NO_DEVICE
    peak = C.c_double(0)
    assert lib.ov_measure_fma_peak(0, C.byref(peak)) != 0


@pytest.mark.parametrize("value", [np.nan, np.inf])
def test_nonfinite_position_is_refused_before_any_work(lib, monkeypatch, value):
    """A live node at a NaN or infinite position makes every reference-named
    call return OV_ERR_NONFINITE from the host-side check, before the device
    is touched, with every output array left as it was."""
    monkeypatch.setenv("OV_QUIET", "1")
    import openvort_b200 as ov
    t = G.single_ring(32, 1e-2)
    ov.configure(Params(use_mf=0, hyperfriction=0))
    t.pos[5, 1] = value
    for arr in (t.vels, t.tangents, t.normals):
        arr[:] = 7.0
    pos0 = t.pos.copy()
    for call in (lambda: ov.update_velocities(t, 0.0), lambda: ov.rk4_step(t, 0.0, 1e-6),
                 lambda: ov.update_tangents_normals(t), lambda: ov.update_tangle(t, 0.0)):
        with pytest.raises(ov.OVError) as e:
            call()
        assert e.value.code == _lib.OV_ERR_NONFINITE
        lib.ov_clear_error()
    assert np.all(t.vels == 7.0) and np.all(t.tangents == 7.0) and np.all(t.normals == 7.0)
    assert np.array_equal(t.pos, pos0, equal_nan=True)
    # an EMPTY slot may hold anything
    t2 = G.single_ring(32, 1e-2)
    t2.stat[31, 0] = -1   # EMPTY
    t2.links[30, 0] = 0
    t2.links[0, 1] = 30
    t2.pos[31] = value
    try:
        ov.update_tangents_normals(t2)
    except ov.OVError as e:
        assert e.code != _lib.OV_ERR_NONFINITE
