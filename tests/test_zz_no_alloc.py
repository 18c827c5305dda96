"""mcl_observe_device, the observables of a director field held in the caller's device memory with no allocation,
against the engine's mcl_measure on the same directors: same site energies, so the two agree to the rounding of
the FP64 sums. Two calls in a row must give identical records, and the second must leave the device's free
memory unchanged. The argument checks that turn a bad buffer into MCL_ERR_ARG run before any kernel launch.

This file is named to be collected last, so that it also runs after every other GPU test in one session."""
import ctypes

import numpy as np
import pytest

from helpers import M

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

P = ctypes.POINTER


def observe_fn():
    f = M.lib().mcl_observe_device
    f.argtypes = [P(M.CModel), P(M.CReplica), ctypes.c_void_p, P(M.CObservables), ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def observe(model, rep, ptr, stream=0):
    o = M.CObservables()
    rc = observe_fn()(ctypes.byref(model), ctypes.byref(rep), ctypes.c_void_p(ptr), ctypes.byref(o),
                      ctypes.c_void_p(stream))
    return rc, np.frombuffer(bytes(o), M.OBS_DTYPE)[0]


def ordered_dirs(n, seed, noise=0.35):
    rng = np.random.default_rng(seed)
    v = np.array([0.2, 0.1, 1.0]) + noise * rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    return v.astype(np.float32).reshape(-1)


CASES = {
    "ll_bulk": (lambda: M.Model("ll"), (24, 20, 16, "bulk", (1, 1, 1))),
    "ll_free_odd": (lambda: M.Model("ll"), (15, 9, 7, "bulk", (0, 0, 0))),
    "ghrl_chiral_slab": (lambda: M.Model("ghrl", k=(1.48, 1, 2.28, 12.0),
                                         surfaces=[("rp_ghrl", 1.0, 90, 30), ("fg_ghrl", 0.8, 0, 0)]),
                         (40, 36, 12, "slab", (1, 1, 0))),
    "pear_field_slab": (lambda: M.Model("pear", A=1.5, B1=0.09, C=0.3, field_dir=(0.3, 0, 1), elecP=0.7,
                                        elecA=0.1, surfaces=[("fg", 1.0, 0, 0), ("rp", 0.5, 40, 10)]),
                        (18, 22, 10, "slab", (0, 1, 0))),
    "ll_many_slots": (lambda: M.Model("ll", field_dir=(1, 0, 0), elecA=0.4),
                      (128, 96, 40, "bulk", (1, 1, 1))),   # 491,520 sites: 120 partial slots
    "ghrl_slab_256_cubed": (lambda: M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2),
                            (256, 256, 256, "slab", (1, 1, 0))),  # the bench lattice: 4096 partial slots
}


def engine_state(model, shape, seed):
    """Directors after a few engine sweeps, and the engine's own measurement of them."""
    nx, ny, nz, geo, per = shape
    rep = M.Replica(nx, ny, nz, geo, per, T=0.7, elecE=1.3, ang_var=0.3, seed=seed)
    e = M.Engine(model, [rep], M.SCHED_CHECKER2)
    try:
        e.upload(0, ordered_dirs(nx * ny * nz, seed))
        e.sweeps(3)
        ni = e.download(0)
        ref = e.measure(0)
    finally:
        e.close()
    return rep, ni, ref


@pytest.mark.parametrize("case", sorted(CASES))
def test_observe_device_matches_measure(case):
    make_model, shape = CASES[case]
    model = make_model()
    rep, ni, ref = engine_state(model, shape, seed=11)
    d_ni = torch.from_numpy(ni).cuda()
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    rc1, o1 = observe(model, rep, d_ni.data_ptr(), stream.cuda_stream)
    assert rc1 == 0, M.lib().mcl_last_error()
    free1 = torch.cuda.mem_get_info()[0]
    rc2, o2 = observe(model, rep, d_ni.data_ptr(), stream.cuda_stream)
    assert rc2 == 0, M.lib().mcl_last_error()
    free2 = torch.cuda.mem_get_info()[0]
    assert free2 == free1, "the second call changed the device's free memory"
    assert bytes(o1) == bytes(o2), "two calls on the same directors differ"

    nv = float(ref["n_valid"])
    assert o1["n_valid"] == nv
    # Same FP32 site energies on both paths; only the order of the FP64 sums differs.
    np.testing.assert_allclose(o1["energy"], ref["energy"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(o1["q"], ref["q"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(o1["nsum"], ref["nsum"], rtol=0, atol=1e-9 * np.sqrt(nv))
    np.testing.assert_allclose(o1["S"], ref["S"], rtol=0, atol=1e-11)
    sign = 1.0 if float(np.dot(o1["director"], ref["director"])) >= 0 else -1.0
    np.testing.assert_allclose(sign * o1["director"], ref["director"], rtol=0, atol=1e-8)
    assert o1["acceptance"] == 0.0 and o1["sweep"] == 0.0
    assert o1["ang_var"] == np.float32(rep.ang_var)


def test_observe_device_default_stream_and_repeat_after_other_work():
    make_model, shape = CASES["ghrl_chiral_slab"]
    model = make_model()
    rep, ni, ref = engine_state(model, shape, seed=5)
    d_ni = torch.from_numpy(ni).cuda()
    torch.cuda.synchronize()
    _, first = observe(model, rep, d_ni.data_ptr(), 0)
    # Another lattice in between overwrites the scratch; the next call must not depend on what it left there.
    model2, shape2 = CASES["ll_many_slots"]
    rep2, ni2, _ = engine_state(model2(), shape2, seed=6)
    d_ni2 = torch.from_numpy(ni2).cuda()
    torch.cuda.synchronize()
    rc, _ = observe(model2(), rep2, d_ni2.data_ptr(), 0)
    assert rc == 0, M.lib().mcl_last_error()
    rc, again = observe(model, rep, d_ni.data_ptr(), 0)
    assert rc == 0, M.lib().mcl_last_error()
    assert bytes(first) == bytes(again)
    np.testing.assert_allclose(again["energy"], ref["energy"], rtol=1e-10, atol=1e-12)


def test_observe_device_rejects_bad_requests_before_launching():
    model = M.Model("ll")
    small = torch.zeros(3 * 8 * 8 * 8, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    # lattice above the 2^26-site limit of the fixed scratch
    rc, _ = observe(model, M.Replica(512, 512, 257), small.data_ptr())
    assert rc == 1 and b"exceed the limit" in M.lib().mcl_last_error()
    # host memory
    host = np.zeros(3 * 512, np.float32)
    rc, _ = observe(model, M.Replica(8, 8, 8), host.ctypes.data)
    assert rc == 1 and b"not device memory" in M.lib().mcl_last_error()
    # the declared lattice runs past the end of the allocation holding the buffer (128^3 sites = 25 MB)
    rc, _ = observe(model, M.Replica(128, 128, 128), small.data_ptr())
    assert rc == 1 and b"allocation ends" in M.lib().mcl_last_error()
    # misaligned pointer
    rc, _ = observe(model, M.Replica(8, 8, 8), small.data_ptr() + 2)
    assert rc == 1 and b"aligned" in M.lib().mcl_last_error()
    # sphere needs the engine's point-type tables
    rc, _ = observe(M.Model("ll", surfaces=[("homeotropic", 1.0, 0, 0)]), M.Replica(8, 8, 8, "sphere"),
                    small.data_ptr())
    assert rc == 1 and b"sphere and custom" in M.lib().mcl_last_error()
    # the library still works afterwards
    rc, o = observe(model, M.Replica(8, 8, 8), small.data_ptr())
    assert rc == 0 and o["n_valid"] == 512


VMM_CHILD = r'''
import ctypes, sys
import numpy as np
import torch
sys.path[:0] = [{tests!r}, {root!r}]
import test_zz_no_alloc as t
from helpers import M
model = M.Model("ghrl", k=(1.0, 0.5, 1.5), surfaces=[("homeotropic", 1.5, 0, 0)] * 2)
rep, ni, ref = t.engine_state(model, (256, 128, 96, "slab", (1, 1, 0)), seed=9)
d_ni = torch.from_numpy(ni).cuda()  # 37.7 MB of directors: at least two of the allocator's 20 MiB mappings
torch.cuda.synchronize()
cuda = ctypes.CDLL("libcuda.so.1")
base, size = ctypes.c_uint64(), ctypes.c_size_t()
assert cuda.cuMemGetAddressRange_v2(ctypes.byref(base), ctypes.byref(size), ctypes.c_uint64(d_ni.data_ptr())) == 0
chunks = "one mapping" if base.value + size.value >= d_ni.data_ptr() + ni.nbytes else "several mappings"
rc, o = t.observe(model, rep, d_ni.data_ptr())
assert rc == 0, M.lib().mcl_last_error()
np.testing.assert_allclose(o["energy"], ref["energy"], rtol=1e-10, atol=1e-12)
np.testing.assert_allclose(o["q"], ref["q"], rtol=0, atol=1e-12)
print("ok", chunks)
'''


def test_observe_device_accepts_a_buffer_of_a_virtual_memory_pool():
    """Pool allocators built on the virtual-memory-management API map a large buffer as several physical chunks (torch's
    expandable segments: 20 MiB each). The call must accept such a buffer and measure it like any other."""
    import os
    import subprocess
    import sys
    tests = os.path.dirname(os.path.abspath(__file__))
    code = VMM_CHILD.format(tests=tests, root=os.path.dirname(tests))
    env = dict(os.environ, PYTORCH_CUDA_ALLOC_CONF="expandable_segments:True")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().startswith("ok"), r.stdout
    print(r.stdout.strip())
