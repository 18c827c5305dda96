"""Pins oracle/extras.py — the CPU checker of the device extra observables (mcl_measure_extras, mcl_local_order) —
to the reference's own functions: Polarization, Splay_magnitude, Splay_divergence, Radial_order and
lattice_order_parameter from src/parameter_order.cpp, compiled from the reference sources with the GSL shim
(oracle/_ref/libref_extras.so, oracle/ref_extras.cpp). Same lattices as tests/test_gpu_extras.py plus a
cylinder-symmetric texture, a free slab and a lattice with scattered empty sites; the two must agree to FP32
rounding of the per-site terms (the sums are double on both sides)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import extras as X

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_extras.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref is built where the reference sources are")


def ref_lib():
    L = ctypes.CDLL(LIB)
    P = ctypes.POINTER
    L.mcr_extras.argtypes = [ctypes.c_int] * 3 + [P(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  P(ctypes.c_double)]
    L.mcr_local_order.argtypes = [ctypes.c_int] * 3 + [P(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p] + \
        [ctypes.c_int] * 3
    L.mcr_local_order.restype = ctypes.c_float
    return L


def ref_extras(ni, pt, shape, periodic, director):
    ni = np.ascontiguousarray(ni, np.float32).reshape(-1)
    pt = np.ascontiguousarray(pt, np.int32)
    d = np.ascontiguousarray(director, np.float32)
    per = (ctypes.c_int * 3)(*[int(p) for p in periodic])
    out = (ctypes.c_double * 7)()
    ref_lib().mcr_extras(*shape, per, ni.ctypes.data, pt.ctypes.data, d.ctypes.data, out)
    return dict(zip(["P", "dtheta", "divn", "Sr_sph", "Pr_sph", "Sr_cyl", "Pr_cyl"], list(out)))


def dirs(n, seed, bias):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3)) + np.asarray(bias)
    return (v / np.linalg.norm(v, axis=1)[:, None]).astype(np.float32)


def radial(nx, ny, nz, cylinder):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    r = np.stack([i - nx // 2, j - ny // 2, 0 * k if cylinder else k - nz // 2], -1).astype(np.float64)
    r = r.transpose(2, 1, 0, 3).reshape(-1, 3)
    r[np.linalg.norm(r, axis=1) == 0] = (0, 0, 1)
    return (r / np.linalg.norm(r, axis=1)[:, None]).astype(np.float32)


def sphere_pt(nx, ny, nz):
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    H = np.float32(nz // 2)
    r = np.sqrt(((i - np.float32(nx // 2)) ** 2 + (j - np.float32(ny // 2)) ** 2 + (k - H) ** 2).astype(np.float32))
    return np.where(r < H - 1, 1, np.where(r < H + 1, 2, 0)).transpose(2, 1, 0).reshape(-1)


def case(name):
    if name == "bulk_periodic":
        shape, per = (10, 8, 6), (1, 1, 1)
        return shape, per, dirs(480, 7, (0.3, -0.2, 1.0)), np.ones(480, int)
    if name == "bulk_free":
        shape, per = (9, 7, 5), (0, 0, 0)
        return shape, per, dirs(315, 8, (0.1, 0.4, 0.6)), np.ones(315, int)
    if name == "slab":
        shape, per = (8, 8, 7), (1, 1, 0)
        return shape, per, dirs(448, 9, (0.0, 0.0, 2.0)), np.ones(448, int)
    if name == "sphere_hedgehog":
        shape, per = (12, 12, 12), (0, 0, 0)
        return shape, per, radial(12, 12, 12, False), sphere_pt(12, 12, 12)
    if name == "cylinder_texture":
        shape, per = (11, 11, 6), (0, 0, 1)
        ni = radial(11, 11, 6, True)
        ni[::7] *= -1  # some inward sites: Pr below 1
        return shape, per, ni, np.ones(11 * 11 * 6, int)
    if name == "empty_sites":
        shape, per = (8, 6, 6), (1, 0, 1)
        rng = np.random.default_rng(4)
        pt = (rng.random(288) > 0.2).astype(int)
        return shape, per, dirs(288, 10, (0.5, 0.5, 0.5)), pt
    raise KeyError(name)


NAMES = ["bulk_periodic", "bulk_free", "slab", "sphere_hedgehog", "cylinder_texture", "empty_sites"]


@pytest.mark.parametrize("name", NAMES)
def test_extras_oracle_equals_reference(name):
    shape, per, ni, pt = case(name)
    director = np.array([0.2, -0.3, 0.93], np.float32)
    director /= np.linalg.norm(director)
    got = X.extras(ni, pt, shape, [bool(p) for p in per], director)
    ref = ref_extras(ni, pt, shape, per, director)
    for k in ref:
        # the reference rounds P, dtheta and divn to float on return; the radial orders stay double
        tol = 2e-7 * max(1.0, abs(ref[k])) if k in ("P", "dtheta", "divn") else 1e-12 + 1e-12 * abs(ref[k])
        assert abs(got[k] - ref[k]) <= tol, (name, k, got[k], ref[k])
    if name == "sphere_hedgehog":
        assert ref["Sr_sph"] > 0.99 and ref["Pr_sph"] > 0.99
    if name == "cylinder_texture":
        assert ref["Sr_cyl"] > 0.99 and 0.5 < ref["Pr_cyl"] < 0.9


def local_order_check(name):
    """Compares oracle/extras.py local_S with the reference at 40 random sites of one case. The reference keeps the
    lattice dimensions of its first call in function-local statics (one simulation per process), so every case runs
    in a process of its own (test_local_order_oracle_equals_reference)."""
    shape, per, ni, pt = case(name)
    nx, ny, nz = shape
    L = ref_lib()
    perc = (ctypes.c_int * 3)(*[int(p) for p in per])
    flat = np.ascontiguousarray(ni, np.float32).reshape(-1)
    pti = np.ascontiguousarray(pt, np.int32)
    rng = np.random.default_rng(1)
    for _ in range(40):
        i, j, k = int(rng.integers(nx)), int(rng.integers(ny)), int(rng.integers(nz))
        if not pti[i + nx * (j + ny * k)]:
            continue
        ref = L.mcr_local_order(nx, ny, nz, perc, flat.ctypes.data, pti.ctypes.data, i, j, k)
        got = X.local_S(ni, pt, shape, [bool(p) for p in per], i, j, k)
        assert abs(got - ref) <= 2e-7 * max(1.0, abs(ref)), (name, (i, j, k), got, ref)


@pytest.mark.parametrize("name", ["bulk_periodic", "bulk_free", "sphere_hedgehog", "empty_sites"])
def test_local_order_oracle_equals_reference(name):
    import subprocess
    import sys
    code = ("import sys; sys.path[:0] = [%r, %r]; import test_extras_pin as t; t.local_order_check(%r)"
            % (os.path.join(ROOT, "tests"), ROOT, name))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
