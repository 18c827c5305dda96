"""mclics_b200 — B200-native checkerboard Metropolis sweep for McLics, Python front end.

Thin ctypes layer over the C ABI of libmclics_b200.so (include/mclics_b200.h). The library is loaded from this
package folder only; when it is missing the import of `lib()` raises (there is no CPU fallback).

    from mclics_b200 import Engine, Model, Replica
    e = Engine(Model(potential="ll"), [Replica(32, 32, 32, T=1.1, seed=1)])
    e.upload(0, ni)            # float32, 3 per site, reference layout (x fastest)
    e.sweeps(100)              # thermalisation
    e.sweeps(200, measure=True)
    E = e.series(0)["energy"]
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmclics_b200.so")
MAX_SURFACES = 16

POTENTIALS = {"ll": 0, "lebwohl-lasher": 0, "ghrl": 1, "gruhn-hess": 1, "pear": 2}
GEOMETRIES = {"bulk": 0, "slab": 1, "sphere": 2, "custom": 3}
ANCHORINGS = {"homeotropic": 0, "rp": 1, "rp_tangent": 2, "fg": 3, "homeotropic_ghrl": 4, "rp_ghrl": 5,
              "fg_ghrl": 6}
SCHED_REF8, SCHED_CHECKER2, SCHED_CHECKER2_SIMPLE = 0, 1, 2
N_MLP_PARAMS = 64 * 7 + 64 + 64 * 64 + 64 + 4 * 64 + 4  # learned proposal network 7 -> 64 -> 64 -> 4
KAPPA_MAX = 500.0
STATUS = {0: "MCL_OK", 1: "MCL_ERR_ARG", 2: "MCL_ERR_CUDA", 3: "MCL_ERR_NOMEM", 4: "MCL_ERR_STATE",
          5: "MCL_ERR_INPUT", 6: "MCL_ERR_IO", 7: "MCL_ERR_NONFINITE", 8: "MCL_ERR_NO_DEVICE"}


class McLicsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (STATUS.get(code, str(code)), msg))
        self.code = code


class CModel(ctypes.Structure):
    _fields_ = [("potential", ctypes.c_int), ("A", ctypes.c_float), ("B1", ctypes.c_float), ("C", ctypes.c_float),
                ("ghrl_lambda", ctypes.c_float), ("ghrl_mu", ctypes.c_float), ("ghrl_nu", ctypes.c_float),
                ("ghrl_rho", ctypes.c_float), ("ghrl_sigma", ctypes.c_float), ("field_dir", ctypes.c_float * 3),
                ("elecA", ctypes.c_float), ("elecP", ctypes.c_float), ("flip_move", ctypes.c_int),
                ("n_surfaces", ctypes.c_int), ("anch_type", ctypes.c_int * MAX_SURFACES),
                ("anch_W", ctypes.c_float * MAX_SURFACES), ("anch_theta", ctypes.c_float * MAX_SURFACES),
                ("anch_phi", ctypes.c_float * MAX_SURFACES)]


class CReplica(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("geometry", ctypes.c_int),
                ("periodic", ctypes.c_int * 3), ("T", ctypes.c_float), ("elecE", ctypes.c_float),
                ("ang_var", ctypes.c_float), ("seed", ctypes.c_ulonglong)]


class CObservables(ctypes.Structure):
    _fields_ = [("energy", ctypes.c_double), ("q", ctypes.c_double * 6), ("S", ctypes.c_double),
                ("director", ctypes.c_double * 3), ("nsum", ctypes.c_double * 3), ("n_valid", ctypes.c_double),
                ("acceptance", ctypes.c_double), ("ang_var", ctypes.c_double), ("sweep", ctypes.c_double)]


OBS_DTYPE = np.dtype([("energy", "f8"), ("q", "f8", 6), ("S", "f8"), ("director", "f8", 3), ("nsum", "f8", 3),
                      ("n_valid", "f8"), ("acceptance", "f8"), ("ang_var", "f8"), ("sweep", "f8")])
assert OBS_DTYPE.itemsize == ctypes.sizeof(CObservables)

_lib = None


def lib():
    """The loaded libmclics_b200.so. Raises if it has not been built (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libmclics_b200.so is not built; run `python -m mclics_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        P, vp, i, f = ctypes.POINTER, ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        sig = {
            "mcl_create": [P(CModel), P(CReplica), i, i, P(vp)],
            "mcl_destroy": [vp],
            "mcl_set_geometry": [vp, i, vp, vp],
            "mcl_upload_directors": [vp, i, vp],
            "mcl_download_directors": [vp, i, vp],
            "mcl_random_directors": [vp, i, ctypes.c_ulonglong],
            "mcl_set_temperature": [vp, i, f],
            "mcl_set_field": [vp, i, f],
            "mcl_set_ang_var": [vp, i, f],
            "mcl_get_ang_var": [vp, i, P(f)],
            "mcl_set_sweep_counter": [vp, ctypes.c_ulonglong],
            "mcl_get_sweep_counter": [vp, P(ctypes.c_ulonglong)],
            "mcl_sweeps": [vp, i, i],
            "mcl_sweeps_io": [vp, i, vp, vp],
            "mcl_series_length": [vp, P(i)],
            "mcl_read_series": [vp, i, i, i, vp],
            "mcl_reserve_series": [vp, i],
            "mcl_clear_series": [vp],
            "mcl_measure": [vp, i, P(CObservables)],
            "mcl_synchronize": [vp],
            "mcl_record_decisions": [vp, i],
            "mcl_read_decisions": [vp, i, vp],
            "mcl_run_input_file": [ctypes.c_char_p],
            "mcl_set_stream": [vp, vp],
            "mcl_profile": [vp, i],
            "mcl_debug_wait_limit": [vp, ctypes.c_longlong, i],
            "mcl_profile_read": [vp, P(ctypes.c_double), P(ctypes.c_longlong), P(ctypes.c_longlong)],
            "mcl_set_proposal": [vp, vp, f],
            "mcl_set_proposal_mix": [vp, i],
            "mcl_autotune": [vp, i, P(CTuning)],
            "mcl_measure_extras": [vp, i, P(ctypes.c_double * 3), P(CExtras)],
            "mcl_local_order": [vp, i, vp],
            "mcl_set_graphs": [vp, i],
            "mcl_set_plan": [vp, i, i],
            "mcl_zslab_init": [vp, i, i, i, P(ctypes.c_longlong)],
            "mcl_zslab_pass": [vp, i, i],
            "mcl_zslab_pack": [vp, vp, vp],
            "mcl_zslab_unpack": [vp, vp, vp],
            "mcl_zslab_sums": [vp, i, vp],
            "mcl_zslab_finalize": [vp, vp, i],
            "mcl_get_plan": [vp, P(CTuning)],
            "mcl_set_adaptation": [vp, i],
            "mcl_extract_samples": [vp, i, ctypes.c_longlong, ctypes.c_ulonglong, vp, vp],
            "mcl_mlp_forward": [vp, vp, ctypes.c_longlong, vp, vp],
            "mcl_mlp_forward_tcgen05": [vp, vp, ctypes.c_longlong, vp, vp],
            "mcl_trainer_create": [vp, ctypes.c_longlong, f, P(vp)],
            "mcl_trainer_gradient": [vp, vp, vp, ctypes.c_longlong, vp, P(ctypes.c_double)],
            "mcl_trainer_step": [vp, vp, vp, ctypes.c_longlong, f, P(ctypes.c_double)],
            "mcl_trainer_get": [vp, vp],
            "mcl_trainer_destroy": [vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        L.mcl_last_error.restype = ctypes.c_char_p
        L.mcl_last_error.argtypes = []
        L.mcl_version.restype = ctypes.c_char_p
        L.mcl_version.argtypes = []
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise McLicsError(rc, lib().mcl_last_error().decode(errors="replace"))
    return rc


def ghrl_coefficients(k11, k22, k33, p0=0.0):
    """GHRL coefficients (lambda, mu, nu, rho, sigma) from the Frank constants, with the float/double typing of
    the reference's setGHRL (src/io.cpp:346-371)."""
    f = np.float32
    k11, k22, k33, p0 = f(k11), f(k22), f(k33), f(p0)
    scale = f(abs(9.0 / float(k11 - f(3) * k22 - k33)))
    sigma = f(-float(scale) * float(k22) * (2 * np.pi / float(p0))) if p0 else f(0)
    lam = f(float(scale / f(9)) * float(f(2) * k11 - f(3) * k22 + k33))
    mu = f(scale * (k22 - k11))
    rho = f(float(scale / f(9)) * float(k11 - k33))
    nu = f(float(scale / f(9)) * float(k11 - f(3) * k22 - k33))
    return (float(lam), float(mu), float(nu), float(rho), float(sigma))


def Model(potential="ll", A=1.0, B1=0.04, C=0.3, ghrl=None, k=None, field_dir=(0.0, 0.0, 0.0), elecA=0.0,
          elecP=0.0, flip_move=None, surfaces=()):
    """Builds the C model struct. ghrl = (lambda, mu, nu, rho, sigma) or k = (k11, k22, k33[, p0]);
    surfaces = [(anchoring, W, theta_s, phi_s), ...]; field_dir is normalised here as src/main.cpp:97-106 does."""
    m = CModel()
    m.potential = POTENTIALS[potential] if isinstance(potential, str) else int(potential)
    m.A, m.B1, m.C = A, B1, C
    if k is not None:
        ghrl = ghrl_coefficients(*k)
    if ghrl is None:
        ghrl = (0.0, 0.0, 1.0, 0.0, 0.0)
    m.ghrl_lambda, m.ghrl_mu, m.ghrl_nu, m.ghrl_rho, m.ghrl_sigma = ghrl
    fd = np.asarray(field_dir, np.float32)
    if elecA != 0 or elecP != 0:
        nrm = np.float32(np.sqrt(np.float32(fd[0] * fd[0] + fd[1] * fd[1] + fd[2] * fd[2])))
        if nrm == 0:
            raise ValueError("elecA or elecP is set but the field direction is zero")
        fd = (fd / nrm).astype(np.float32)
    m.field_dir[:] = [float(x) for x in fd]
    m.elecA, m.elecP = elecA, elecP
    if flip_move is None:
        flip_move = 1 if (m.potential == 2 or elecP != 0) else 0
    m.flip_move = int(flip_move)
    if len(surfaces) > MAX_SURFACES:
        raise ValueError("at most %d surfaces" % MAX_SURFACES)
    m.n_surfaces = len(surfaces)
    for s, (name, W, th, ph) in enumerate(surfaces):
        m.anch_type[s] = ANCHORINGS[name] if isinstance(name, str) else int(name)
        m.anch_W[s], m.anch_theta[s], m.anch_phi[s] = W, th, ph
    return m


def Replica(nx, ny, nz, geometry="bulk", periodic=(1, 1, 1), T=1.0, elecE=1.0, ang_var=0.5, seed=1):
    r = CReplica()
    r.nx, r.ny, r.nz = nx, ny, nz
    r.geometry = GEOMETRIES[geometry] if isinstance(geometry, str) else int(geometry)
    r.periodic[:] = [int(bool(p)) for p in periodic]
    r.T, r.elecE, r.ang_var, r.seed = T, elecE, ang_var, seed
    return r


class CExtras(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("P", "dtheta", "divn", "Sr_sph", "Pr_sph", "Sr_cyl", "Pr_cyl")]


class CTuning(ctypes.Structure):
    _fields_ = [("tile_config", ctypes.c_int), ("rows_per_tile", ctypes.c_int), ("threads_per_cta", ctypes.c_int),
                ("planes_per_segment", ctypes.c_int), ("work_items", ctypes.c_int), ("candidates", ctypes.c_int),
                ("ms_per_sweep", ctypes.c_double), ("ms_default", ctypes.c_double)]


class Engine:
    """One engine = a batch of replicas sharing a model, swept together on the current CUDA device."""

    def __init__(self, model, replicas, schedule=SCHED_CHECKER2):
        self._h = ctypes.c_void_p()
        arr = (CReplica * len(replicas))(*replicas)
        check(lib().mcl_create(ctypes.byref(model), arr, len(replicas), schedule, ctypes.byref(self._h)))
        self.model = model
        self.replicas = [(r.nx, r.ny, r.nz) for r in replicas]
        self.n = len(replicas)

    def close(self):
        if self._h:
            lib().mcl_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sites(self, r):
        nx, ny, nz = self.replicas[r]
        return nx * ny * nz

    def set_geometry(self, r, pt, normals):
        pt = np.ascontiguousarray(pt, np.int32)
        nrm = np.ascontiguousarray(normals, np.float32)
        assert pt.size == self.sites(r) and nrm.size == 3 * self.sites(r)
        check(lib().mcl_set_geometry(self._h, r, pt.ctypes.data, nrm.ctypes.data))

    def upload(self, r, ni):
        ni = np.ascontiguousarray(ni, np.float32).reshape(-1)
        assert ni.size == 3 * self.sites(r)
        check(lib().mcl_upload_directors(self._h, r, ni.ctypes.data))

    def download(self, r):
        out = np.empty(3 * self.sites(r), np.float32)
        check(lib().mcl_download_directors(self._h, r, out.ctypes.data))
        return out

    def random_directors(self, r, seed):
        """Random initial condition of replica r on the device (Philox stream 2 keyed by seed)."""
        check(lib().mcl_random_directors(self._h, r, seed))

    def set_temperature(self, T, r=-1):
        check(lib().mcl_set_temperature(self._h, r, T))

    def set_field(self, E, r=-1):
        check(lib().mcl_set_field(self._h, r, E))

    def set_ang_var(self, v, r=-1):
        check(lib().mcl_set_ang_var(self._h, r, v))

    def ang_var(self, r=0):
        v = ctypes.c_float()
        check(lib().mcl_get_ang_var(self._h, r, ctypes.byref(v)))
        return v.value

    def set_sweep_counter(self, t):
        check(lib().mcl_set_sweep_counter(self._h, t))

    def sweep_counter(self):
        v = ctypes.c_ulonglong()
        check(lib().mcl_get_sweep_counter(self._h, ctypes.byref(v)))
        return v.value

    def sweeps(self, n, measure=False):
        check(lib().mcl_sweeps(self._h, n, 1 if measure else 0))

    def sweeps_io(self, n, T=None, out=None):
        """n measured sweeps in one call: T (one float32 per replica, or None to keep the temperatures) goes up, the
        n x replicas observables records come back (in `out` when given, an OBS_DTYPE array of that size).
        The data addresses of the last T and out arrays are cached while this engine holds them (numpy refuses to
        resize an array that another object references, so the addresses stay valid)."""
        n_rep = self.n
        if out is None:
            out = np.zeros(n * n_rep, OBS_DTYPE)
        elif out.dtype != OBS_DTYPE or out.size < n * n_rep or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous OBS_DTYPE array of at least {n * n_rep} records")
        cache = self.__dict__.setdefault("_io_cache", [None, 0, None, 0])
        tp = None
        if T is not None:
            if T is not cache[0]:
                if not (isinstance(T, np.ndarray) and T.dtype == np.float32 and T.flags.c_contiguous):
                    T = np.ascontiguousarray(T, dtype=np.float32)
                if T.size != n_rep:
                    raise ValueError(f"T needs {n_rep} values, got {T.size}")
                cache[0], cache[1] = T, T.ctypes.data
            tp = cache[1]
        if out is not cache[2]:
            cache[2], cache[3] = out, out.ctypes.data
        check(lib().mcl_sweeps_io(self._h, n, tp, cache[3]))
        return out

    def series_length(self):
        v = ctypes.c_int()
        check(lib().mcl_series_length(self._h, ctypes.byref(v)))
        return v.value

    def series(self, r=0, first=0, count=None):
        if count is None:
            count = self.series_length() - first
        out = np.zeros(count, OBS_DTYPE)
        if count:
            check(lib().mcl_read_series(self._h, r, first, count, out.ctypes.data))
        return out

    def reserve_series(self, rows):
        check(lib().mcl_reserve_series(self._h, rows))

    def clear_series(self):
        check(lib().mcl_clear_series(self._h))

    def measure(self, r=0):
        o = CObservables()
        check(lib().mcl_measure(self._h, r, ctypes.byref(o)))
        return np.frombuffer(bytes(o), OBS_DTYPE)[0]

    def synchronize(self):
        check(lib().mcl_synchronize(self._h))

    def set_stream(self, stream_handle):
        """Route the engine's work to an existing cudaStream_t (int handle, e.g. torch's stream.cuda_stream)."""
        check(lib().mcl_set_stream(self._h, ctypes.c_void_p(stream_handle or 0)))

    def profile(self, on=True):
        check(lib().mcl_profile(self._h, 1 if on else 0))

    def profile_read(self):
        """(total sweep-kernel ms, timed sweeps, kernels launched so far)."""
        ms, n, k = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().mcl_profile_read(self._h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(k)))
        return ms.value, n.value, k.value

    def debug_wait_limit(self, timeout_ns, withhold_first_load=False):
        check(lib().mcl_debug_wait_limit(self._h, timeout_ns, 1 if withhold_first_load else 0))

    def record_decisions(self, on=True):
        check(lib().mcl_record_decisions(self._h, 1 if on else 0))

    def decisions(self, r=0):
        out = np.empty(self.sites(r), np.uint8)
        check(lib().mcl_read_decisions(self._h, r, out.ctypes.data))
        return out

    def set_proposal(self, params=None, kappa_max=KAPPA_MAX):
        """Learned proposal with the flat MLP parameter vector `params` (N_MLP_PARAMS floats, mcl_mlp order);
        None returns to the plain proposal."""
        if params is None:
            check(lib().mcl_set_proposal(self._h, None, kappa_max))
            return
        p = mlp_params(params)
        check(lib().mcl_set_proposal(self._h, p.ctypes.data, kappa_max))

    def set_proposal_mix(self, period):
        """With a learned proposal set: one learned sweep after every period - 1 plain sweeps (1: all learned)."""
        check(lib().mcl_set_proposal_mix(self._h, period))

    def measure_extras(self, r, director):
        """P, dtheta, divn and the radial orders of replica r's current state (director: that state's Q director)."""
        d = (ctypes.c_double * 3)(*[float(v) for v in director])
        x = CExtras()
        check(lib().mcl_measure_extras(self._h, r, ctypes.byref(d), ctypes.byref(x)))
        return {k: getattr(x, k) for k, _ in CExtras._fields_}

    def local_order(self, r):
        """Local order parameter S of every site of replica r (NaN on empty sites), reference order."""
        out = np.empty(self.sites(r), np.float32)
        check(lib().mcl_local_order(self._h, r, out.ctypes.data))
        return out

    def autotune(self, trial_sweeps=3):
        """Times the candidate tile plans on this engine's replicas, keeps the fastest (state is restored)."""
        t = CTuning()
        check(lib().mcl_autotune(self._h, trial_sweeps, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in CTuning._fields_}

    def set_plan(self, tile_config, planes_per_segment=0):
        """Applies a plan without timing it (tile configuration 0..4, planes per z segment; 0: heuristic)."""
        check(lib().mcl_set_plan(self._h, tile_config, planes_per_segment))

    def plan(self):
        t = CTuning()
        check(lib().mcl_get_plan(self._h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in CTuning._fields_ if not k.startswith("ms_") and k != "candidates"}

    # z-slab of a lattice split over processes (mclics_b200.zslab drives these); pointers are device addresses
    def zslab_init(self, nz_global, z_offset, periodic_z):
        n = ctypes.c_longlong(0)
        check(lib().mcl_zslab_init(self._h, nz_global, z_offset, 1 if periodic_z else 0, ctypes.byref(n)))
        return n.value

    def zslab_pass(self, colour, measure):
        check(lib().mcl_zslab_pass(self._h, colour, 1 if measure else 0))

    def zslab_pack(self, send_lo, send_hi):
        check(lib().mcl_zslab_pack(self._h, send_lo or None, send_hi or None))

    def zslab_unpack(self, recv_lo, recv_hi):
        check(lib().mcl_zslab_unpack(self._h, recv_lo or None, recv_hi or None))

    def zslab_sums(self, measure, d_sums):
        check(lib().mcl_zslab_sums(self._h, 1 if measure else 0, d_sums))

    def zslab_finalize(self, d_sums, measure):
        check(lib().mcl_zslab_finalize(self._h, d_sums, 1 if measure else 0))

    def set_graphs(self, on=True):
        check(lib().mcl_set_graphs(self._h, 1 if on else 0))

    def set_adaptation(self, on=True):
        check(lib().mcl_set_adaptation(self._h, 1 if on else 0))

    def extract_samples(self, r, n, seed, features_ptr, directors_ptr):
        """n training samples of replica r into device buffers (n x 8 and n x 3 floats)."""
        check(lib().mcl_extract_samples(self._h, r, n, seed, ctypes.c_void_p(features_ptr),
                                        ctypes.c_void_p(directors_ptr)))


def mlp_params(params):
    p = np.ascontiguousarray(params, np.float32).reshape(-1)
    if p.size != N_MLP_PARAMS:
        raise ValueError("the MLP has %d parameters, got %d" % (N_MLP_PARAMS, p.size))
    return p


def mlp_forward(params, features_ptr, n, out_ptr, stream=0, tcgen05=False):
    """Raw network outputs (n x 4) of the tensor-core MLP for n device feature rows (n x 8): mma.sync warps, or
    with tcgen05=True the fifth-generation tensor cores."""
    p = mlp_params(params)
    fn = lib().mcl_mlp_forward_tcgen05 if tcgen05 else lib().mcl_mlp_forward
    check(fn(p.ctypes.data, ctypes.c_void_p(features_ptr), n, ctypes.c_void_p(out_ptr), ctypes.c_void_p(stream or 0)))


class Trainer:
    """GPU training of the proposal network (mcl_trainer_*): maximum likelihood, Adam."""

    def __init__(self, params, max_batch, kappa_max=KAPPA_MAX):
        self._h = ctypes.c_void_p()
        p = mlp_params(params)
        check(lib().mcl_trainer_create(p.ctypes.data, max_batch, kappa_max, ctypes.byref(self._h)))

    def gradient(self, features_ptr, directors_ptr, n):
        g = np.empty(N_MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        check(lib().mcl_trainer_gradient(self._h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(directors_ptr), n,
                                         g.ctypes.data, ctypes.byref(loss)))
        return loss.value, g

    def step(self, features_ptr, directors_ptr, n, lr):
        loss = ctypes.c_double()
        check(lib().mcl_trainer_step(self._h, ctypes.c_void_p(features_ptr), ctypes.c_void_p(directors_ptr), n, lr,
                                     ctypes.byref(loss)))
        return loss.value

    def params(self):
        p = np.empty(N_MLP_PARAMS, np.float32)
        check(lib().mcl_trainer_get(self._h, p.ctypes.data))
        return p

    def close(self):
        if self._h:
            lib().mcl_trainer_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_input_file(path):
    """Runs a McLics input file in the current directory (mcl_run_input_file); raises McLicsError on failure."""
    return check(lib().mcl_run_input_file(os.fsencode(path)))


def version():
    return lib().mcl_version().decode()
