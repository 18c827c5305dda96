"""ctypes front end of the CPU oracle (mc_oracle.c) and reader of the reference replay dumps.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker. The product (mclics_b200) never imports this module.
"""
import ctypes
import os
import struct
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
MAX_SURF = 16

POT = {"ll": 0, "lebwohl-lasher": 0, "ghrl": 1, "gruhn-hess": 1, "pear": 2}
ANCH = {"homeotropic": 0, "rp": 1, "rp_tangent": 2, "fg": 3, "homeotropic_ghrl": 4, "rp_ghrl": 5, "fg_ghrl": 6}
SCHED_REF8, SCHED_CHECKER2 = 0, 1


class Model(ctypes.Structure):
    _fields_ = [("potential", ctypes.c_int), ("A", ctypes.c_float), ("B1", ctypes.c_float), ("C", ctypes.c_float),
                ("ghrl_lambda", ctypes.c_float), ("ghrl_mu", ctypes.c_float), ("ghrl_nu", ctypes.c_float),
                ("ghrl_rho", ctypes.c_float), ("ghrl_sigma", ctypes.c_float), ("field_dir", ctypes.c_float * 3),
                ("elecA", ctypes.c_float), ("elecP", ctypes.c_float), ("elecE", ctypes.c_float),
                ("flip_move", ctypes.c_int), ("n_surfaces", ctypes.c_int), ("anch_type", ctypes.c_int * MAX_SURF),
                ("anch_W", ctypes.c_float * MAX_SURF), ("anch_theta", ctypes.c_float * MAX_SURF),
                ("anch_phi", ctypes.c_float * MAX_SURF)]


class Lattice(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("periodic", ctypes.c_int * 3),
                ("pt", ctypes.c_void_p), ("ns", ctypes.c_void_p)]


_lib = None


def lib():
    """Loads oracle/liboracle.so (building it with make when it is missing and a compiler is present)."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        L.mco_philox4x32_10.argtypes = [P(ctypes.c_uint32), P(ctypes.c_uint32), P(ctypes.c_uint32)]
        L.mco_site_uniforms.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_double)]
        L.mco_site_energy.argtypes = [P(Model), P(Lattice), ctypes.c_void_p, ctypes.c_int, P(ctypes.c_float)]
        L.mco_site_energy.restype = ctypes.c_float
        L.mco_sweep.argtypes = [P(Model), P(Lattice), ctypes.c_void_p, ctypes.c_float, P(ctypes.c_float),
                                ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.mco_sweep.restype = ctypes.c_int64
        L.mco_energy_ref.argtypes = [P(Model), P(Lattice), ctypes.c_void_p]
        L.mco_energy_ref.restype = ctypes.c_float
        L.mco_energy_fp64sum.argtypes = [P(Model), P(Lattice), ctypes.c_void_p]
        L.mco_energy_fp64sum.restype = ctypes.c_double
        L.mco_q_tensor_ref.argtypes = [P(Lattice), ctypes.c_void_p, P(ctypes.c_float)]
        L.mco_observables_fp64.argtypes = [P(Model), P(Lattice), ctypes.c_void_p, P(ctypes.c_double)]
        L.mco_largest_eigen.argtypes = [P(ctypes.c_double), P(ctypes.c_double)]
        L.mco_largest_eigen.restype = ctypes.c_double
        L.mco_ref8_stream.argtypes = [P(Model), P(Lattice), ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                                      ctypes.c_int64]
        L.mco_ref8_stream.restype = ctypes.c_int64
        L.mco_random_director.argtypes = [ctypes.c_uint64, ctypes.c_uint32, P(ctypes.c_float)]
        _lib = L
    return _lib


def philox(ctr, key):
    c = (ctypes.c_uint32 * 4)(*ctr)
    k = (ctypes.c_uint32 * 2)(*key)
    o = (ctypes.c_uint32 * 4)()
    lib().mco_philox4x32_10(c, k, o)
    return list(o)


def site_uniforms(seed, sweep, x, y, z, nx, ny, flip):
    u = (ctypes.c_double * 4)()
    lib().mco_site_uniforms(seed, sweep, x, y, z, nx, ny, flip, u)
    return list(u)


def random_directors(seed, n_sites):
    """Random initial directors of sites 0 .. n_sites - 1 (mco_random_director), float32 (n_sites, 3)."""
    out = np.empty((n_sites, 3), np.float32)
    f = (ctypes.c_float * 3)()
    for q in range(n_sites):
        lib().mco_random_director(seed, q, f)
        out[q] = f[:]
    return out


def make_model(potential="ll", A=1.0, B1=0.04, C=0.3, ghrl=(0, 0, 1, 0, 0), field_dir=(0, 0, 0), elecA=0.0,
               elecP=0.0, elecE=1.0, flip_move=None, surfaces=()):
    """surfaces: sequence of (anchoring name, W, theta_s, phi_s). ghrl = (lambda, mu, nu, rho, sigma)."""
    m = Model()
    m.potential = POT[potential] if isinstance(potential, str) else int(potential)
    m.A, m.B1, m.C = A, B1, C
    m.ghrl_lambda, m.ghrl_mu, m.ghrl_nu, m.ghrl_rho, m.ghrl_sigma = ghrl
    m.field_dir[:] = list(field_dir)
    m.elecA, m.elecP, m.elecE = elecA, elecP, elecE
    if flip_move is None:
        flip_move = 1 if (m.potential == 2 or elecP != 0) else 0
    m.flip_move = flip_move
    m.n_surfaces = len(surfaces)
    for s, (name, W, th, ph) in enumerate(surfaces):
        m.anch_type[s] = ANCH[name] if isinstance(name, str) else int(name)
        m.anch_W[s], m.anch_theta[s], m.anch_phi[s] = W, th, ph
    return m


def lattice_from_replay(d):
    return Lat(d["nx"], d["ny"], d["nz"], d["periodic"], d["pt"], d["ns"])


class Lat:
    """Lattice plus the numpy arrays it points to (kept alive together)."""

    def __init__(self, nx, ny, nz, periodic=(1, 1, 1), pt=None, ns=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.pt = None if pt is None else np.ascontiguousarray(pt, dtype=np.int32)
        self.ns = None if ns is None else np.ascontiguousarray(ns, dtype=np.float32)
        self.c = Lattice()
        self.c.nx, self.c.ny, self.c.nz = nx, ny, nz
        self.c.periodic[:] = list(periodic)
        self.c.pt = None if self.pt is None else self.pt.ctypes.data
        self.c.ns = None if self.ns is None else self.ns.ctypes.data

    @property
    def n(self):
        return self.nx * self.ny * self.nz


def ghrl_coefficients(k11, k22, k33, p0=0.0):
    """setGHRL (reference io.cpp:346-371) in the reference's float/double typing."""
    f = np.float32
    k11, k22, k33, p0 = f(k11), f(k22), f(k33), f(p0)
    scale = f(abs(9.0 / float(k11 - f(3) * k22 - k33)))
    sigma = f(-float(scale) * float(k22) * (2 * np.pi / float(p0))) if p0 else f(0)
    lam = f(float(scale / f(9)) * float(f(2) * k11 - f(3) * k22 + k33))
    mu = f(scale * (k22 - k11))
    rho = f(float(scale / f(9)) * float(k11 - k33))
    nu = f(float(scale / f(9)) * float(k11 - f(3) * k22 - k33))
    return (float(lam), float(mu), float(nu), float(rho), float(sigma))


def sweep(model, lat, ni, T, ang_var, seed, sweep_index, schedule=SCHED_CHECKER2, want_decisions=False):
    """One oracle sweep in place on ni (float32, AoS 3*N). Returns (acceptance, new ang_var, decisions, margin)."""
    assert ni.dtype == np.float32 and ni.flags.c_contiguous and ni.size == 3 * lat.n
    av = ctypes.c_float(ang_var)
    dec = np.zeros(lat.n, np.uint8) if want_decisions else None
    mar = np.zeros(lat.n, np.float32) if want_decisions else None
    acc = lib().mco_sweep(ctypes.byref(model), ctypes.byref(lat.c), ni.ctypes.data, T, ctypes.byref(av), seed,
                          sweep_index, schedule, None if dec is None else dec.ctypes.data,
                          None if mar is None else mar.ctypes.data)
    return acc, av.value, dec, mar


def site_energy(model, lat, ni, idx, n=None):
    v = ni[3 * idx:3 * idx + 3] if n is None else n
    arr = (ctypes.c_float * 3)(*[float(x) for x in v])
    return lib().mco_site_energy(ctypes.byref(model), ctypes.byref(lat.c), ni.ctypes.data, idx, arr)


def energy_ref(model, lat, ni):
    return lib().mco_energy_ref(ctypes.byref(model), ctypes.byref(lat.c), ni.ctypes.data)


def energy_fp64sum(model, lat, ni):
    return lib().mco_energy_fp64sum(ctypes.byref(model), ctypes.byref(lat.c), ni.ctypes.data)


def q_tensor_ref(lat, ni):
    q = (ctypes.c_float * 9)()
    lib().mco_q_tensor_ref(ctypes.byref(lat.c), ni.ctypes.data, q)
    return np.array(list(q), np.float32)


def observables_fp64(model, lat, ni):
    o = (ctypes.c_double * 11)()
    lib().mco_observables_fp64(ctypes.byref(model), ctypes.byref(lat.c), ni.ctypes.data, o)
    return np.array(list(o))


def largest_eigen(q6):
    q = (ctypes.c_double * 6)(*[float(x) for x in q6])
    v = (ctypes.c_double * 3)()
    s = lib().mco_largest_eigen(q, v)
    return s, np.array(list(v))


def ref8_stream(model, lat, seed, sweep_index):
    out = np.zeros(4 * lat.n + 16, np.float64)
    n = lib().mco_ref8_stream(ctypes.byref(model), ctypes.byref(lat.c), seed, sweep_index, out.ctypes.data,
                              out.size)
    return out[:n]


# ---- reference replay dumps (oracle/ref_replay.cpp) ----------------------------------------------------------

def ref_available():
    return os.path.exists(os.path.join(REF_DIR, "mclics_ref_replay"))


def run_ref_replay(input_text, n_sweeps, seed, workdir):
    """Runs the reference's own sweep (oracle/_ref/mclics_ref_replay) and parses its dump."""
    os.makedirs(workdir, exist_ok=True)
    inp = os.path.join(workdir, "input.txt")
    with open(inp, "w") as f:
        f.write(input_text)
    out = os.path.join(workdir, "replay.bin")
    env = dict(os.environ, OMP_NUM_THREADS="1")
    p = subprocess.run([os.path.join(REF_DIR, "mclics_ref_replay"), "input.txt", str(n_sweeps), str(seed),
                        "replay.bin"], cwd=workdir, env=env, capture_output=True, text=True, timeout=600)
    if p.returncode != 0:
        raise RuntimeError("mclics_ref_replay failed (%d): %s" % (p.returncode, p.stderr[-2000:]))
    return read_replay(out)


def read_replay(path):
    with open(path, "rb") as f:
        b = f.read()
    o = 0

    def take(fmt):
        nonlocal o
        v = struct.unpack_from(fmt, b, o)
        o += struct.calcsize(fmt)
        return v

    assert b[:4] == b"MCLR"
    o = 4
    (ver, nx, ny, nz, nsw, pot, flip, nsurf) = take("<8i")
    periodic = take("<3i")
    hdr = take("<15f")
    keys = ["A", "B1", "C", "lambda", "mu", "nu", "rho", "sigma", "elecX", "elecY", "elecZ", "elecA", "elecP",
            "elecE", "T"]
    d = dict(zip(keys, hdr))
    d.update(nx=nx, ny=ny, nz=nz, n_sweeps=nsw, potential=pot, flip_move=flip, periodic=periodic)
    surf = []
    for _ in range(nsurf):
        t, = take("<i")
        W, th, ph = take("<3f")
        surf.append((t, W, th, ph))
    d["surfaces"] = surf
    N = nx * ny * nz
    d["pt"] = np.frombuffer(b, np.int32, N, o).copy()
    o += 4 * N
    d["ns"] = np.frombuffer(b, np.float32, 3 * N, o).copy()
    o += 12 * N
    sweeps = []
    for _ in range(nsw):
        av, = take("<f")
        ni = np.frombuffer(b, np.float32, 3 * N, o).copy()
        o += 12 * N
        nd, = take("<i")
        E, av2 = take("<2f")
        sweeps.append(dict(ang_var=av, ni=ni, n_draws=nd, E_after=E, ang_var_after=av2))
    d["sweeps"] = sweeps
    d["final"] = np.frombuffer(b, np.float32, 3 * N, o).copy()
    return d


def model_from_replay(d):
    m = make_model(d["potential"], d["A"], d["B1"], d["C"],
                   (d["lambda"], d["mu"], d["nu"], d["rho"], d["sigma"]),
                   (d["elecX"], d["elecY"], d["elecZ"]), d["elecA"], d["elecP"], d["elecE"], d["flip_move"],
                   [(t, W, th, ph) for (t, W, th, ph) in d["surfaces"]])
    return m


def lattice_from_replay(d):
    return Lat(d["nx"], d["ny"], d["nz"], d["periodic"], d["pt"], d["ns"])
