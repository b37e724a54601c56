"""Host-side checks of the reference pinning harness (oracle/ref_gpu.cu).

The harness hands this project's models and receptors to the reference's
own FP64 device library; before it uploads anything it converts them to the
reference's flat structures (baseline/ref_gpu/flatten.h, a restatement of
src/gpu/gpu_flatten.cpp shared with the reference GPU baseline) and checks
every index the reference's kernels read.  These tests run that
conversion and those checks on the CPU for every input the golden-record
script uses, and compare the conversion's counts with counts taken here
from the descriptors.  The harness is built only where the reference tree
is present (`make -C oracle ref`)."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_ref_golden as G  # noqa: E402
import smina_b200 as sb  # noqa: E402

pytestmark = pytest.mark.skipif(not os.path.exists(G.REF_SO),
                                reason="reference harness not built (make -C oracle ref needs the reference tree)")


@pytest.fixture(scope="module")
def lib():
    L = C.CDLL(G.REF_SO)
    L.refg_last_error.restype = C.c_char_p
    L.refg_check_model.argtypes = [C.POINTER(sb.ModelDesc), C.POINTER(C.c_int)]
    L.refg_check_receptor.argtypes = [C.POINTER(sb.TablesDesc), C.POINTER(sb.ReceptorDesc), C.POINTER(sb.GridDims),
                                      C.POINTER(C.c_longlong)]
    return L


def _expected_counts(m):
    d = m.desc
    parent = np.ctypeslib.as_array(d.frame_parent, shape=(d.num_frames,))
    kind = np.ctypeslib.as_array(d.frame_kind, shape=(d.num_frames,))
    depth = np.zeros(d.num_frames, int)
    for f in range(d.num_frames):
        depth[f] = 0 if parent[f] < 0 else depth[parent[f]] + 1
    pr = np.ctypeslib.as_array(d.pairs, shape=(2 * d.num_pairs,)) if d.num_pairs else np.zeros(0, np.int32)
    incidences = int(np.sum(pr < d.num_movable))  # a pair appears in the list of each movable atom it has
    roots = int(np.sum(parent < 0))
    assert roots == d.num_ligands + d.num_flex
    assert int(np.sum(kind == 0)) == d.num_ligands  # SG_FRAME_RIGID: one rigid root per ligand
    return [d.num_frames, roots, incidences, int(depth.max()) + 1]


def test_models_flatten_and_pass_the_index_checks(lib):
    for name, T, R, gd, models in G.cases():
        for m in models:
            out = (C.c_int * 4)()
            rc = lib.refg_check_model(C.byref(m.desc), out)
            assert rc == 0, (name, lib.refg_last_error().decode())
            assert list(out) == _expected_counts(m), name


def test_receptor_cell_lists_pass_the_index_checks(lib):
    for name, T, R, gd, models in G.cases():
        out = (C.c_longlong * 4)()
        rc = lib.refg_check_receptor(C.byref(T.desc), C.byref(R.desc), C.byref(gd), out)
        assert rc == 0, (name, lib.refg_last_error().decode())
        types = np.ctypeslib.as_array(R.desc.type, shape=(R.desc.num_atoms,))
        usable = int(np.sum((types > 1) & (types < 27)))
        grid_atoms, grid_entries, full_atoms, full_entries = list(out)
        assert full_atoms == usable  # non_cache keeps every usable heavy atom
        assert 0 < grid_atoms <= usable and grid_entries > 0 and full_entries > 0


def test_a_bad_model_is_refused_before_any_upload(lib):
    m = G.cases()[0][4][1]
    bad = sb.ModelDesc.from_buffer_copy(m.desc)
    pairs = np.ctypeslib.as_array(m.desc.pairs, shape=(2 * m.desc.num_pairs,)).copy()
    pairs[1] = m.desc.num_atoms  # a pair atom past the last atom
    bad.pairs = pairs.ctypes.data_as(sb._ip)
    assert lib.refg_check_model(C.byref(bad), None) != 0
    assert b"pair" in lib.refg_last_error()
