"""Writes the golden vectors that pin the oracle's scalar math.

Inputs are seeded; outputs come from the reference's own headers
(src/lib/portable_math.h, src/gpu/gpu_rng.cuh, src/gpu/gpu_math.cuh) compiled by
`make -C oracle ref` into oracle/_ref/libref_probe.so.  Run in a tree that
has the reference mounted:  python tests/golden/make_golden.py
"""
import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PROBE = os.path.join(ROOT, "oracle", "_ref", "libref_probe.so")

dp = C.POINTER(C.c_double)


def hexs(a):
    return [format(int(x), "016x") for x in np.ascontiguousarray(a, np.float64).view(np.uint64)]


def main():
    L = C.CDLL(PROBE)
    L.ref_pm_eval.argtypes = [C.c_int, dp, dp, C.c_int]
    rng = np.random.default_rng(20261203)
    cases = {
        "sin": (0, np.concatenate([rng.uniform(-np.pi / 4, np.pi / 4, 500), rng.uniform(-60, 60, 1000),
                                   [0.0, -0.0, 0.3, 0.78125, 0.7853981633974483, 1e-9, 3.0, -3.0, 1e3]])),
        "cos": (1, np.concatenate([rng.uniform(-np.pi / 4, np.pi / 4, 500), rng.uniform(-60, 60, 1000),
                                   [0.0, 0.29999, 0.3, 0.78, 0.79, 1.5707963267948966, 3.14159]])),
        "acos": (2, np.concatenate([rng.uniform(-1, 1, 1500), [-1.0, 1.0, 0.0, 0.5, -0.5, 0.4999, 0.99999999]])),
        "exp": (3, np.concatenate([rng.uniform(-20, 5, 1000), rng.uniform(-745, 709, 500),
                                   [0.0, 1e-10, -1e-10, 0.34657, 0.34658, -0.5, 709.78, -745.2]])),
    }
    out = {"source": "reference src/lib/portable_math.h via oracle/_ref/libref_probe.so", "functions": {}}
    for name, (fn, x) in cases.items():
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros_like(x)
        L.ref_pm_eval(fn, x.ctypes.data_as(dp), y.ctypes.data_as(dp), len(x))
        out["functions"][name] = {"x": hexs(x), "y": hexs(y)}
    with open(os.path.join(HERE, "portable_math.json"), "w") as f:
        json.dump(out, f, indent=0)

    L.ref_mt_probe.argtypes = [C.c_uint32, C.c_int, C.POINTER(C.c_uint32), C.c_double, C.c_double, dp, C.c_int,
                               C.c_int, C.POINTER(C.c_int)]
    mt = {"source": "reference src/gpu/gpu_rng.cuh via oracle/_ref/libref_probe.so", "cases": []}
    for seed, a, b, lo, hi in [(5489, -1.0, 1.0, 0, 1000000), (0, -np.pi, np.pi, 0, 7), (123456789, 0.0, 1.0, -5, 5)]:
        n = 1500
        raw = np.zeros(n, np.uint32)
        fl = np.zeros(n)
        it = np.zeros(n, np.int32)
        L.ref_mt_probe(seed, n, raw.ctypes.data_as(C.POINTER(C.c_uint32)), a, b, fl.ctypes.data_as(dp), lo, hi,
                       it.ctypes.data_as(C.POINTER(C.c_int)))
        mt["cases"].append({"seed": seed, "a": a, "b": b, "lo": lo, "hi": hi, "raw": raw.tolist(),
                            "fl": hexs(fl), "int": it.tolist()})
    with open(os.path.join(HERE, "mt19937.json"), "w") as f:
        json.dump(mt, f)

    # quaternion / angle math: axis-angle, rotation vectors (some below epsilon),
    # angles over several turns, unit and slightly unnormalised quaternions
    L.ref_quat_probe.argtypes = [dp, dp, dp, C.c_int]
    n = 250
    axis = rng.normal(size=(n, 3))
    axis /= np.linalg.norm(axis, axis=1)[:, None]
    angle = np.concatenate([rng.uniform(-np.pi, np.pi, 120), rng.uniform(-40, 40, 120),
                            [np.pi, -np.pi, 3 * np.pi, -3 * np.pi, 0.0, 1e-12, 9.5, -9.5, 7 * np.pi, 2.5]])
    rot = rng.normal(size=(n, 3)) * rng.choice([1e-18, 1e-3, 0.5, 2.0, 6.0], size=n)[:, None]
    q0 = rng.normal(size=(n, 4))
    q0 /= np.linalg.norm(q0, axis=1)[:, None]
    q0[::7] *= 1 + rng.uniform(-1e-3, 1e-3, size=(len(q0[::7]), 1))
    inp = np.ascontiguousarray(np.concatenate([axis, angle[:, None], rot], axis=1))
    q0 = np.ascontiguousarray(q0)
    res = np.zeros((n, 22))
    L.ref_quat_probe(inp.ctypes.data_as(dp), q0.ctypes.data_as(dp), res.ctypes.data_as(dp), n)
    quat = {"source": "reference src/gpu/gpu_math.cuh (FP64, host-compiled) via oracle/_ref/libref_probe.so",
            "layout": "in[7] = axis xyz, angle, rotation xyz; out[22] = normalized_angle, angle_to_quaternion(axis, "
                      "angle), angle_to_quaternion(rotation), quaternion_increment(q0, rotation), "
                      "quaternion_to_r3(q0) column-major",
            "in": hexs(inp.ravel()), "q0": hexs(q0.ravel()), "out": hexs(res.ravel())}
    with open(os.path.join(HERE, "quaternion.json"), "w") as f:
        json.dump(quat, f)


if __name__ == "__main__":
    main()
