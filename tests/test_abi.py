"""The C ABI library: it loads without a GPU, exports every symbol that
include/raven_b200.h declares, its descriptor layout matches the header, and the
argument checks that run before any CUDA call return the documented statuses."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "raven_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(rb200_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol(rb):
    L = rb._lib.lib()
    names = declared_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(L, name), name
    assert set(names) == set(rb._lib.EXPORTED)


def test_descriptor_layout_matches_header(rb, tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "raven_b200.h"\n'
        "int main(void){printf(\"%zu\", sizeof(rb200_desc));"
        + "".join(
            f'printf(" %zu", offsetof(rb200_desc, {f}));'
            for f, _ in rb._lib.Desc._fields_
        )
        + "return 0;}\n"
    )
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = [int(v) for v in subprocess.check_output([str(exe)]).split()]
    assert out[0] == ctypes.sizeof(rb._lib.Desc)
    assert out[1:] == [getattr(rb._lib.Desc, f).offset for f, _ in rb._lib.Desc._fields_]


def _desc(rb, grid, law=0, **kw):
    import numpy as np

    keep = [np.asfortranarray(a) for a in (grid.cell.D, grid.cell.w, grid.volume_metrics, grid.surface_metrics,
                                            grid.vmapM, grid.vmapP, grid.boundarycodes)]
    d = rb._lib.Desc()
    d.abi_version = 1
    d.dim, d.nq, d.law, d.num_elements = grid.dim, grid.nq, law, grid.E
    d.volume_form, d.volume_flux, d.surface_flux, d.precision, d.gamma = 0, 0, 3, 0, 1.4
    (d.D, d.w, d.volume_metrics, d.surface_metrics, d.vmapM, d.vmapP, d.boundary_codes) = [
        k.ctypes.data_as(ctypes.c_void_p) for k in keep]
    for k, v in kw.items():
        setattr(d, k, v)
    return d, keep


def _create(rb, d):
    L = rb._lib.lib()
    h = ctypes.c_void_p()
    st = L.rb200_create(ctypes.byref(d), ctypes.byref(h))
    msg = L.rb200_last_error(h).decode() if h else ""
    if h:
        L.rb200_destroy(h)
    return st, msg


@pytest.fixture(scope="module")
def small_grid(rb):
    cell = rb.LobattoCell(3, 3)
    return rb.generate(rb.GridManager(cell, rb.brick((rb.jl_range(0, 1, 3), rb.jl_range(0, 1, 3)), (True, True))))


def test_create_rejects_bad_arguments_before_touching_the_device(rb, small_grid):
    L = rb._lib.lib()
    h = ctypes.c_void_p()
    assert L.rb200_create(None, ctypes.byref(h)) == 1
    d, keep = _desc(rb, small_grid, abi_version=99)
    assert _create(rb, d)[0] == 1
    d, keep = _desc(rb, small_grid, dim=4)
    assert _create(rb, d)[0] == 6
    d, keep = _desc(rb, small_grid, dim=1)  # 1-D is supported: a 2-D grid's face maps do not fit it
    assert _create(rb, d)[0] == 2
    d, keep = _desc(rb, small_grid, nq=9)
    assert _create(rb, d)[0] == 6
    d, keep = _desc(rb, small_grid, law=7)
    assert _create(rb, d)[0] == 1
    d, keep = _desc(rb, small_grid, volume_form=1, volume_flux=1)  # advection + KG
    assert _create(rb, d)[0] == 6
    d, keep = _desc(rb, small_grid, law=1, gamma=1.0)
    assert _create(rb, d)[0] == 1
    d, keep = _desc(rb, small_grid, vmapP=None)
    assert _create(rb, d)[0] == 1


def test_create_checks_face_maps_node_by_node(rb, small_grid):
    import numpy as np

    g = small_grid
    # a face node mapped to an interior node of the neighbour, or to a node of a third
    # element, is no face connectivity (a permutation within the neighbour's face is:
    # that is a rotated face, kept as a vmapP table, which needs a device to upload)
    ne = (g.vmapP[0, 0] - 1) // g.np
    interior = ne * g.np + (g.nq + 1) + (g.nq * g.nq if g.dim == 3 else 0) + 1
    third = [e for e in range(g.E) if e not in (0, ne)][0]
    for val in (interior, third * g.np + 1):
        bad = g.vmapP.copy()
        bad[1, 0] = val
        d, keep = _desc(rb, g)
        keep.append(np.asfortranarray(bad))
        d.vmapP = keep[-1].ctypes.data_as(ctypes.c_void_p)
        st, msg = _create(rb, d)
        assert st == 2 and "one face of one other element" in msg
    badM = g.vmapM.copy()
    badM[0, 0] += 1
    d, keep = _desc(rb, g)
    keep.append(np.asfortranarray(badM))
    d.vmapM = keep[-1].ctypes.data_as(ctypes.c_void_p)
    assert _create(rb, d)[0] == 2


def test_status_strings(rb):
    L = rb._lib.lib()
    assert L.rb200_status_string(0) == b"ok"
    assert L.rb200_status_string(6) == b"unsupported"
    assert L.rb200_last_error(None) == b"null handle"


def test_bounded_wait_probe_validates_before_the_device(rb):
    L = rb._lib.lib()
    assert L.rb200_probe_bounded_wait(0, None) == 1  # RB200_ERR_BAD_ARG, no device call
    assert L.rb200_probe_bounded_wait(1 << 31, None) == 1
