"""The oracle, and this engine's FP64 path, against the reference's own FP64
device library.

tests/golden/ref_fp64.npz holds what the reference's FP64 validation path
(src/gpu/gpu_device.cu, src/gpu/gpu_kernels_f64.cu, behind
oracle/ref_gpu.cu) computed on a GPU for seeded synthetic inputs; it was
written by tests/golden/make_ref_golden.py.  Here every case's inputs are
rebuilt from their seeds, checked against the recorded SHA-256 digest, and
the oracle's outputs are compared with the records: grid maps, eval at two
curl caps, direct eval, BFGS with both line searches, Monte Carlo chains and
refine_structure, for vina and ad4 tables (ad4 also with non-zero partial
charges), a model with flexible residues and a user grid.

The bar is the reference's own for its FP64 path (gpu_eval_test.cpp:173-210,
gpu_mc_test.cpp:44-81): relative differences of at most 1e-9 and identical
chain containers.  Beyond that bar every value must agree bit for bit, as
both sides follow CPU smina's operation order without fused multiply-adds."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_ref_golden as G  # noqa: E402

FIXTURE = os.path.join(HERE, "golden", "ref_fp64.npz")
REL = 1e-9  # the reference's FP64 tolerance

pytestmark = pytest.mark.skipif(not os.path.exists(FIXTURE), reason="reference records not generated yet")


@pytest.fixture(scope="module")
def records():
    with np.load(FIXTURE) as z:
        return {k: z[k] for k in z.files}


def _check(records, name, mine):
    ref = {k: v for k, v in records.items() if k.startswith(f"{name}/") and not k.endswith("/sha256")}
    assert set(ref) == set(mine)
    for k, a in ref.items():
        b = np.asarray(mine[k])
        assert a.shape == b.shape, k
        if a.dtype.kind == "f":
            rel = np.abs(a - b) / np.maximum(np.abs(a), 1.0)
            assert rel.max(initial=0.0) <= REL, f"{k}: relative difference {rel.max():.3g}"
        else:
            assert np.array_equal(a, b), k
    total, same, worst, key = G.compare(ref, mine)
    assert same == total, f"{total - same} of {total} values differ in the last bits (largest {worst:.3g} at {key})"


def _case(records, case):
    name, T, R, gd, models = next(c for c in G.cases() if c[0] == case)
    ug = G.user_grid_for(name, gd)
    assert str(records[f"{name}/sha256"]) == G.digest(T, R, gd, models, ug), "inputs differ from the recorded ones"
    return name, T, R, gd, models, ug


@pytest.mark.parametrize("case", ["vina", "ad4", "vina_ug", "ad4_q"])
def test_oracle_matches_the_reference_device_library(records, case):
    name, T, R, gd, models, _ = _case(records, case)
    _check(records, name, G.outputs(G.oracle_for(name, T, R, gd), T, gd, models, name))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["vina", "ad4", "vina_ug", "ad4_q"])
def test_engine_matches_the_reference_device_library(records, case):
    """This engine's FP64 path (grid maps, eval at both curl caps, direct
    eval, both line searches, 40-step chains, refine; the vina case includes
    a model with flexible residues, vina_ug a user grid) against the same
    records."""
    name, T, R, gd, models, ug = _case(records, case)
    side = G.EngineSide(T, R, gd, ug)
    try:
        _check(records, name, G.outputs(side, T, gd, models, name))
    finally:
        side.close()
