"""One lattice split along z over several processes, one GPU each, for lattices larger than one GPU holds.

A process owns a contiguous range of planes plus one halo plane on each side. It sweeps its planes with the
in-place colour passes (`mcl_zslab_*` in include/mclics_b200.h), and after every colour pass it exchanges its
boundary planes with its neighbours, so the next pass reads current neighbours. After every sweep the processes
add up their observables and accepted rotations, and every process finalises the same global record (E, Q, S,
acceptance, ang_var adaptation). Site draws use global plane indices, so the processes together make the sweep one
engine would make on the whole lattice, bit for bit (tests/test_gpu_zslab.py).

    ex = TorchExchange()                                   # torch.distributed, NCCL between the GPUs
    slab = ZSlab(model, nx, ny, nz, rank, world, ex, periodic_z=True, T=1.0, seed=7)
    slab.upload_global(ni)                                 # the whole lattice, reference layout
    slab.sweeps(100, measure=True)
    E = slab.series()["energy"]                            # the global series, the same on every rank

The transfers per colour pass are one padded plane (3 x (ny + 4) x 2 hp floats, about 0.85 MB at 256^2) to each
neighbour, and one 11-double all-reduce per sweep; they are enqueued on the CUDA stream the engine sweeps on, so
no step waits for the host. LocalGroup runs several slabs in one process on one device, with device copies as the
exchange: it is how the decomposition is checked where only one GPU is available.
"""
import numpy as np
import torch

from . import Engine, Replica

N_SUMS = 11  # energy, Q xx xy xz yy yz zz, sum n x y z, accepted rotations


def partition(nz, world):
    """(first plane, number of planes) of each rank: contiguous ranges whose sizes differ by at most one, the
    larger ones first."""
    if world < 1 or nz < world:
        raise ValueError("cannot split %d planes over %d ranks" % (nz, world))
    base, extra = divmod(nz, world)
    out, z = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((z, n))
        z += n
    return out


def neighbours(rank, world, periodic_z):
    """(lower, upper) neighbour ranks of a rank; None beyond a free z boundary. With a periodic z axis the first
    and last ranks are neighbours (a single rank is its own)."""
    lo = rank - 1 if rank > 0 else (world - 1 if periodic_z else None)
    hi = rank + 1 if rank < world - 1 else (0 if periodic_z else None)
    return lo, hi


class TorchExchange:
    """Boundary planes and sums through torch.distributed (NCCL between GPUs, gloo on CPU). The point-to-point
    operations of one exchange form one batch, enqueued after the work already on the current CUDA stream."""

    def __init__(self, group=None):
        self.group = group

    def exchange(self, rank, lo, hi, send_lo, send_hi, recv_lo, recv_hi):
        """send_lo (this rank's lowest owned plane) goes to the lower neighbour's recv_hi, send_hi to the upper
        neighbour's recv_lo."""
        import torch.distributed as dist
        if lo == rank and hi == rank:  # one rank with a periodic z axis: its planes wrap onto itself
            recv_lo.copy_(send_hi)
            recv_hi.copy_(send_lo)
            return
        # Sends in the order (lower, upper), receives in the order (upper, lower): when two ranks are each other's
        # lower and upper neighbour (two ranks, periodic z), the k-th message from one meets the k-th receive of
        # the other, which is the matching pair.
        ops = []
        if lo is not None:
            ops.append(dist.P2POp(dist.isend, send_lo, lo, group=self.group))
        if hi is not None:
            ops.append(dist.P2POp(dist.isend, send_hi, hi, group=self.group))
        if hi is not None:
            ops.append(dist.P2POp(dist.irecv, recv_hi, hi, group=self.group))
        if lo is not None:
            ops.append(dist.P2POp(dist.irecv, recv_lo, lo, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()

    def allreduce(self, sums):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():  # one process without a group: its sums are the total
            dist.all_reduce(sums, group=self.group)


class ZSlab:
    """This process's part of a lattice split along z: planes z0 .. z0 + nz_own - 1 of nz_global, on the current
    CUDA device. geometry "bulk" or "slab" (the slab's z axis is free); periodic_xy for x and y; periodic_z for the
    global z axis (bulk only). exchange: a TorchExchange, or None when a LocalGroup drives the slab.

    stream: the torch.cuda.Stream the engine sweeps on and the exchange and all-reduce are enqueued on (one
    stream orders them without host waits). The default stream cannot serve (its handle, 0, means "the engine's
    own stream" at the C ABI), so by default the slab makes a stream of its own; slabs of one LocalGroup must
    share one."""

    def __init__(self, model, nx, ny, nz_global, rank, world, exchange=None, geometry="bulk", periodic_xy=(1, 1),
                 periodic_z=True, T=1.0, seed=1, ang_var=0.5, elecE=1.0, schedule_plan=None, stream=None):
        if geometry == "slab":
            periodic_z = False
        self.nx, self.ny, self.nz_global = nx, ny, nz_global
        self.rank, self.world, self.ex = rank, world, exchange
        self.z0, self.nz_own = partition(nz_global, world)[rank]
        self.lo, self.hi = neighbours(rank, world, periodic_z)
        self.periodic_z = periodic_z
        rep = Replica(nx, ny, self.nz_own + 2, geometry, (periodic_xy[0], periodic_xy[1], 0), T=T, elecE=elecE,
                      ang_var=ang_var, seed=seed)
        self.eng = Engine(model, [rep])
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.stream = stream if stream is not None else torch.cuda.Stream(self.device)
        if self.stream.cuda_stream == 0:
            raise ValueError("the default stream cannot carry a z-slab (handle 0 is the engine's own stream)")
        self.eng.set_stream(self.stream.cuda_stream)
        n = self.eng.zslab_init(nz_global, self.z0, periodic_z)
        if schedule_plan is not None:
            self.eng.set_plan(*schedule_plan)
        with torch.cuda.stream(self.stream):
            self.bufs = torch.zeros(4, n, dtype=torch.float32, device=self.device)  # send lo, hi; receive lo, hi
            self.sums = torch.zeros(N_SUMS, dtype=torch.float64, device=self.device)
        self.stream.synchronize()
        self._halos_current = False

    # ---- state ---------------------------------------------------------------------------------------------
    def local_planes(self, ni_global):
        """The local lattice (halo, owned planes, halo) cut from a whole lattice in the reference layout; a halo
        beyond a free boundary (never read) gets the adjacent owned plane."""
        g = np.asarray(ni_global, dtype=np.float32).reshape(self.nz_global, self.ny * self.nx * 3)
        idx = []
        for z in range(self.z0 - 1, self.z0 + self.nz_own + 1):
            if 0 <= z < self.nz_global:
                idx.append(z)
            elif self.periodic_z:
                idx.append(z % self.nz_global)
            else:
                idx.append(min(max(z, 0), self.nz_global - 1))
        return g[idx].reshape(-1)

    def upload_global(self, ni_global):
        self.eng.upload(0, self.local_planes(ni_global))
        self._halos_current = False

    def download_owned(self):
        """This rank's owned planes in the reference layout (nx ny nz_own x 3 floats)."""
        loc = self.eng.download(0).reshape(self.nz_own + 2, -1)
        return loc[1:-1].reshape(-1)

    def series(self):
        return self.eng.series(0)

    def set_temperature(self, T):
        self.eng.set_temperature(T)

    def set_sweep_counter(self, s):
        self.eng.set_sweep_counter(s)

    # ---- the steps of a sweep --------------------------------------------------------------------------------
    def pack(self):
        self.eng.zslab_pack(self.bufs[0].data_ptr() if self.lo is not None else 0,
                            self.bufs[1].data_ptr() if self.hi is not None else 0)

    def unpack(self):
        self.eng.zslab_unpack(self.bufs[2].data_ptr() if self.lo is not None else 0,
                              self.bufs[3].data_ptr() if self.hi is not None else 0)

    def colour_pass(self, colour, measure):
        self.eng.zslab_pass(colour, measure)
        self.pack()

    def local_sums(self, measure):
        self.eng.zslab_sums(measure, self.sums.data_ptr())

    def finalize(self, measure):
        self.eng.zslab_finalize(self.sums.data_ptr(), measure)

    def _exchange(self):
        self.ex.exchange(self.rank, self.lo, self.hi, self.bufs[0], self.bufs[1], self.bufs[2], self.bufs[3])
        self.unpack()

    def sweeps(self, n, measure=False):
        """n sweeps of the whole lattice (every rank calls this with the same n and measure)."""
        if self.ex is None:
            raise RuntimeError("this slab is driven by a LocalGroup")
        with torch.cuda.stream(self.stream):
            if not self._halos_current:
                self.pack()
                self._exchange()
                self._halos_current = True
            for _ in range(n):
                for colour in (0, 1):
                    self.colour_pass(colour, measure)
                    self._exchange()
                self.local_sums(measure)
                self.ex.allreduce(self.sums)
                self.finalize(measure)


class LocalGroup:
    """The ranks of a decomposition as slabs of one process on one device: the same steps as ZSlab.sweeps, with
    device copies between the slabs' buffers as the exchange and their sum as the all-reduce."""

    def __init__(self, slabs):
        self.slabs = sorted(slabs, key=lambda s: s.rank)
        self.stream = self.slabs[0].stream
        if any(s.stream is not self.stream for s in self.slabs):
            raise ValueError("the slabs of a LocalGroup must share one stream")
        self._halos_current = False

    def _exchange(self):
        for s in self.slabs:
            if s.lo is not None:
                s.bufs[2].copy_(self.slabs[s.lo].bufs[1])
            if s.hi is not None:
                s.bufs[3].copy_(self.slabs[s.hi].bufs[0])
        for s in self.slabs:
            s.unpack()

    def sweeps(self, n, measure=False):
        with torch.cuda.stream(self.stream):
            self._sweeps(n, measure)

    def _sweeps(self, n, measure):
        if not self._halos_current:
            for s in self.slabs:
                s.pack()
            self._exchange()
            self._halos_current = True
        for _ in range(n):
            for colour in (0, 1):
                for s in self.slabs:
                    s.colour_pass(colour, measure)
                self._exchange()
            for s in self.slabs:
                s.local_sums(measure)
            total = torch.stack([s.sums for s in self.slabs]).sum(0)
            for s in self.slabs:
                s.sums.copy_(total)
                s.finalize(measure)
