"""Serving loop: a stream of FMM requests on one GPU with continuous batching.

A request is one point set, one kernel and a list of densities.  This is the
reference's planned use (class_fmm.py:166-399): one FMM object, then
``build_expansions(tau)`` + ``evaluate_to_points(x, y, True)`` per density.
The server:

* admits waiting requests in arrival order whenever a slot is free and the
  estimated device memory of the admitted plans stays within ``hbm_budget``
  bytes (a request larger than the whole budget runs alone);
* runs each admitted request from its own worker thread on its own CUDA stream.
  The library releases the GIL in every call, so the tree builds, operator
  builds and applies of several requests overlap on the device, and a request
  that arrives while others run starts as soon as a slot and memory free up;
* keeps the request's tree, plan and translation operators on the device
  across its densities.  The first density runs the apply and captures it as a
  CUDA graph (``FMM.capture_apply``); each further density is one graph
  launch and one device-to-host copy of the potentials, after the density is
  in place on the device (a host-to-device copy of a given density, or a fresh
  N(0,1) draw made on the device, as the iterates of an iterative solve on the
  GPU would be);
* records arrival, admission and completion times.  Latency is completion
  minus arrival.

With ``packed=True`` the densities of all admitted requests advance in
lockstep instead: worker threads build each request's tree and operators and
apply its first density, then the request joins a ``PackedBatch``
(``kifmm_batch_capture``), one CUDA graph per set of requests in which the
M2L of every request is one tensor-core launch and the near field + L2P one
launch per kernel kind, the per-request passes running as parallel branches;
the batch draws every request's next density itself and sums its potentials
on the device.  Each step is one graph launch plus the device-to-host copies.

Results do not depend on what else runs: every request has its own plan and
buffers, the packed kernels run the same per-tile and per-leaf code as a
request's own launches, and the kernels are deterministic.
``tests/test_serving.py`` checks that a request gives the same potentials
alone and in the mix, packed or not.
"""
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field

import ctypes

import numpy as np

from . import _lib as B
from . import class_fmm as C


# admission budget of the serving stream: 80 GB of device memory for plans
DEFAULT_HBM_BUDGET = 80_000_000_000


@dataclass
class Request:
    """One FMM job: points (x, y), kernel ('laplace' or 'k0' with wavenumber
    k), Nequiv, Ncutoff and the densities to apply: either ``taus`` (float64
    host arrays of len(x), copied to the device per density) or ``napply``
    fresh N(0,1) densities drawn on the device, density i from the seed
    (tau_seed, i) (``device_density``), so that a long stream holds no
    densities in host memory.  ``arrival`` is in seconds from the start of the
    run."""
    x: np.ndarray
    y: np.ndarray
    taus: list = None
    kernel: str = "laplace"
    k: float = 0.0
    nequiv: int = 32
    ncutoff: int = 64
    arrival: float = 0.0
    rid: int = 0
    napply: int = 0
    tau_seed: int = 0

    def count(self):
        return len(self.taus) if self.taus is not None else self.napply

    def density(self, i):
        """Host copy of density i (for checks; the server draws it on the device)."""
        if self.taus is not None:
            return self.taus[i]
        import torch
        out = torch.empty(len(self.x), dtype=torch.float64, device="cuda")
        device_density(torch, self.tau_seed, i, out)
        return out.cpu().numpy()


DRAW_SKIP = (1 << 64) - 1  # lane seed of a packed batch whose density the caller writes


def device_density(torch, seed, i, out):
    """Fresh N(0,1) density i of a request, drawn into the contiguous float64
    CUDA tensor ``out`` on torch's current stream by the library's
    counter-based generator (``kifmm_fill_normal``, seed ``seed``, density
    number ``i``): the same numbers alone, in any mix and in a packed batch."""
    if not (out.is_cuda and out.dtype == torch.float64 and out.is_contiguous()):
        raise ValueError("device_density needs a contiguous float64 CUDA tensor")
    st = torch.cuda.current_stream(out.device).cuda_stream
    B.check(B.load().kifmm_fill_normal(out.data_ptr(), out.numel(), int(seed), int(i),
                                       ctypes.c_void_p(st if st else 1)))


class PackedBatch:
    """Packed applies of several FMM objects (``kifmm_batch_capture``): one
    CUDA graph whose M2L of all plans is one tensor-core launch and whose near
    field + L2P is one launch per kernel kind, with the per-plan passes as
    parallel branches.  ``fmms`` are mixed-precision FMM objects after
    precompute; ``taus`` / ``pots`` their float64 CUDA tensors (the graph keeps
    their addresses); ``stream`` a torch.cuda.Stream that orders the capture
    and every ``launch``.  Each result equals the plan's own apply."""

    def __init__(self, fmms, taus, pots, stream, check_self=True):
        import torch
        n = len(fmms)
        if not (n == len(taus) == len(pots)) or n == 0:
            raise ValueError("PackedBatch needs one tau and one pot tensor per FMM")
        for f, t, q in zip(fmms, taus, pots):
            for v in (t, q):
                if not (v.is_cuda and v.dtype == torch.float64 and v.is_contiguous() and v.numel() == f.N):
                    raise ValueError("PackedBatch needs contiguous float64 CUDA tensors of one value per point")
        self._lib = B.load()
        vp = ctypes.c_void_p * n
        plans = vp(*[f._plan.value for f in fmms])
        tp = vp(*[t.data_ptr() for t in taus])
        pp = vp(*[q.data_ptr() for q in pots])
        h = ctypes.c_void_p()
        B.check(self._lib.kifmm_batch_capture(plans, n, tp, pp, int(bool(check_self)),
                                              ctypes.c_void_p(stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        self._keep = (list(fmms), list(taus), list(pots), stream)  # the graph uses their memory

    def set_draws(self, seeds, index):
        """Lane r draws N(0,1) density index[r] of seed seeds[r] into its tau
        at the start of each later launch (``DRAW_SKIP``: the caller writes it)."""
        n = len(self._keep[0])
        sv = (ctypes.c_uint64 * n)(*[int(v) for v in seeds])
        iv = (ctypes.c_uint64 * n)(*[int(v) for v in index])
        B.check(self._lib.kifmm_batch_set_draws(self._h, sv, iv))

    def launch(self):
        B.check(self._lib.kifmm_batch_launch(self._h))

    def synchronize(self):
        B.check(self._lib.kifmm_batch_synchronize(self._h))

    def sums(self):
        """Per-lane sums of the potentials of the last launch (after synchronize)."""
        out = np.empty(len(self._keep[0]))
        B.check(self._lib.kifmm_batch_sums(self._h, out.ctypes.data))
        return out

    def info(self):
        """(tiles of the packed M2L launch, leaves of the packed leaf launches)"""
        t, l = ctypes.c_int64(), ctypes.c_int64()
        B.check(self._lib.kifmm_batch_info(self._h, ctypes.byref(t), ctypes.byref(l)))
        return t.value, l.value

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.kifmm_batch_destroy(h)
        self._h = None
        self._keep = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: torch may be gone already
            pass


@dataclass
class Result:
    rid: int
    pots: list = field(default_factory=list)   # potentials per density (keep_pots)
    sums: list = field(default_factory=list)   # sum of the potentials per density
    arrival: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    n: int = 0
    napply: int = 0
    error: str = ""

    @property
    def latency(self):
        return self.done - self.arrival


def estimate_plan_bytes(n, nequiv=32, ncutoff=64, levels=20):
    """Upper estimate of the device memory one plan holds: per point the
    coordinate, charge and potential arrays, sort keys and indices (about
    110 B); per node (about 10 n / ncutoff nodes) the check potentials and node
    tables; per level the FP64 operators with their FP32 copies, the tensor-core
    slices and the build temporaries."""
    q = int(nequiv)
    nodes = 10.0 * n / max(int(ncutoff), 1) + 64
    per_node = 2 * q * 8 + 120 + 0.25 * 5 * 4 * q
    stride = 153 * q * q + 4 * q
    per_level = stride * 8 * 1.5 + 102 * q * q * 8 + 9 * 16 * q * q * 5 + 97 * q * 8
    return int(160 * n + nodes * per_node + levels * per_level + (1 << 20))


class Scheduler:
    """Admission in arrival order under a slot count and a memory budget (no
    GPU here; the server drives it).  ``admit(now)`` returns the requests that
    may start at time ``now``; ``release(req)`` returns a finished request's
    slot and memory."""

    def __init__(self, requests, slots, budget, estimate=None):
        self.waiting = sorted(requests, key=lambda r: (r.arrival, r.rid))
        self.slots = int(slots)
        self.budget = int(budget)
        self.estimate = estimate or (lambda r: estimate_plan_bytes(len(r.x), r.nequiv, r.ncutoff))
        self.active = {}
        self.used = 0

    def admit(self, now):
        out = []
        while self.waiting and self.waiting[0].arrival <= now and len(self.active) < self.slots:
            r = self.waiting[0]
            need = self.estimate(r)
            if self.active and self.used + need > self.budget:
                break  # head of line waits for memory; later arrivals do not overtake it
            self.waiting.pop(0)
            self.active[r.rid] = need
            self.used += need
            out.append(r)
        return out

    def release(self, req):
        self.used -= self.active.pop(req.rid)

    def next_arrival(self):
        return self.waiting[0].arrival if self.waiting else None

    def idle(self):
        return not self.waiting and not self.active


class Server:
    """Continuous-batching FMM server on one GPU (see the module docstring)."""

    def __init__(self, device=0, slots=8, hbm_budget=None, precision="mixed", check_self=True, keep_pots=True,
                 graphs=True, packed=False):
        import torch
        self.keep_pots = bool(keep_pots)
        self.packed = bool(packed)
        if self.packed and precision != "mixed":
            raise ValueError("packed serving runs the mixed-precision form")
        self.torch = torch
        self.device = int(device)
        self.slots = int(slots)
        self.precision = precision
        self.check_self = bool(check_self)
        self.graphs = bool(graphs)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = min(DEFAULT_HBM_BUDGET, int(0.9 * free))
        self.hbm_budget = int(hbm_budget)
        # streams made by the library, one per slot (+ the batch stream): torch's
        # own stream pool hands the same 32 streams out again, and two slots, or
        # a slot and a capturing batch, must never share one
        self._raw_streams = []
        self._streams = [self._new_stream() for _ in range(self.slots)]
        self._free_streams = list(range(self.slots))
        self._lock = threading.Lock()
        self._dev_lock = threading.Lock()  # allocations vs graph captures (see _buffers)
        self._batch_stream = self._new_stream() if self.packed else None

    def _new_stream(self):
        h = ctypes.c_void_p()
        B.check(B.load().kifmm_stream_create(self.device, ctypes.byref(h)))
        self._raw_streams.append(h.value)
        return self.torch.cuda.ExternalStream(h.value, device=self.torch.device("cuda", self.device))

    def close(self):
        """Wait for the server's streams and release them."""
        raw, self._raw_streams = getattr(self, "_raw_streams", []), []
        if raw:
            self.torch.cuda.synchronize(self.device)
        for h in raw:
            B.load().kifmm_stream_destroy(ctypes.c_void_p(h))

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: torch may be gone already
            pass

    def _kernel(self, req):
        if req.kernel == "laplace":
            return C.LaplaceKernel()
        if req.kernel == "k0":
            return C.ModifiedHelmholtzKernel(req.k)
        raise ValueError(f"unknown kernel {req.kernel!r}")

    def _buffers(self, req, s, precision):
        """A request's device points, plan, density / potential / sum buffers
        and pinned host potentials.  Made under the server's device lock: an
        allocation can synchronise with every stream, which must not happen
        while another thread captures a CUDA graph."""
        torch = self.torch
        dev = torch.device("cuda", self.device)
        n = len(req.x)
        kern = self._kernel(req)
        with self._dev_lock:
            xd = torch.as_tensor(np.ascontiguousarray(req.x, dtype=np.float64), device=dev)
            yd = torch.as_tensor(np.ascontiguousarray(req.y, dtype=np.float64), device=dev)
            f = C.FMM(xd, yd, C.Get_Kernel_Functions(kern), C.prepare_numba_functions_on_the_fly(kern),
                      req.nequiv, req.ncutoff, precision=precision, device=self.device, stream=s.cuda_stream)
            tau = torch.empty(n, dtype=torch.float64, device=dev)
            pot = torch.empty(n, dtype=torch.float64, device=dev)
            tot = torch.empty((), dtype=torch.float64, device=dev)
            host = torch.empty(n, dtype=torch.float64, pin_memory=True)
        return xd, yd, f, tau, pot, tot, host

    def _run_one(self, req, res, t0):
        torch = self.torch
        with self._lock:
            si = self._free_streams.pop()
        s = self._streams[si]
        try:
            dev = torch.device("cuda", self.device)
            with torch.cuda.device(dev), torch.cuda.stream(s):
                xd, yd, f, tau_d, pot_d, tot, host = self._buffers(req, s, self.precision)
                f.build_tree()
                f.precompute()
                n = len(req.x)
                for i in range(req.count()):
                    if req.taus is not None:
                        tau_d.copy_(torch.as_tensor(np.ascontiguousarray(req.taus[i], dtype=np.float64)))
                    else:
                        device_density(torch, req.tau_seed, i, tau_d)
                    if not self.graphs:
                        f.build_expansions(tau_d)
                        f.evaluate_to_points(xd, yd, self.check_self, out=pot_d)
                    elif i == 0:
                        with self._dev_lock:
                            f.capture_apply(tau_d, pot_d, self.check_self)
                    else:
                        f.replay()
                    torch.sum(pot_d, dim=0, out=tot)
                    host.copy_(pot_d, non_blocking=True)
                    s.synchronize()
                    res.sums.append(float(tot))
                    if self.keep_pots:
                        res.pots.append(host.numpy().copy())
                f.synchronize()
                del f
            res.n, res.napply = n, req.count()
        except Exception as e:  # reported per request; the stream goes on
            res.error = f"{type(e).__name__}: {e}"
        finally:
            res.done = time.perf_counter() - t0
            with self._lock:
                self._free_streams.append(si)
        return req, res

    def _setup_packed(self, req, res, t0):
        """Packed mode, worker thread: plan, tree, operators and the first
        density of one request on its slot's stream; the request then joins
        the packed batch for its remaining densities."""
        torch = self.torch
        with self._lock:
            si = self._free_streams.pop()
        s = self._streams[si]
        live = _Live(req=req, res=res, si=si)
        try:
            dev = torch.device("cuda", self.device)
            with torch.cuda.device(dev), torch.cuda.stream(s):
                live.x, live.y, f, live.tau, live.pot, tot, live.host = self._buffers(req, s, "mixed")
                f.build_tree()
                f.precompute()
                n = len(req.x)
                if req.taus is not None:
                    live.tau.copy_(torch.as_tensor(np.ascontiguousarray(req.taus[0], dtype=np.float64)))
                else:
                    device_density(torch, req.tau_seed, 0, live.tau)
                f.build_expansions(live.tau)
                f.evaluate_to_points(live.x, live.y, self.check_self, out=live.pot)
                torch.sum(live.pot, dim=0, out=tot)
                live.host.copy_(live.pot, non_blocking=True)
                f.synchronize()
                s.synchronize()
                live.record(self.keep_pots, float(tot))
                live.f = f
            res.n, res.napply = n, req.count()
        except Exception as e:
            res.error = f"{type(e).__name__}: {e}"
        return live

    def _run_packed(self, requests, realtime):
        """The step loop of packed serving.  Every step applies one density of
        each request in the captured batch (one graph launch), then copies the
        potentials to pinned host memory.  A request that has had all its
        densities is done at once (slot and memory released); its lane stays
        in the graph, computing on its last density, until the next capture.
        The batch is captured again when the requests that wait to join plus
        these finished lanes reach half the batch (or nothing live is left),
        so that captures stay rare against steps."""
        torch = self.torch
        sched = Scheduler(requests, self.slots, self.hbm_budget)
        results = {}
        t0 = time.perf_counter()
        setups = {}
        ready, lanes = [], []
        batch = None
        bs = self._batch_stream
        stats = {"steps": 0, "captures": 0, "member_steps": 0, "idle_lane_steps": 0}

        def complete(live):
            live.done = True
            live.res.done = time.perf_counter() - t0
            with self._lock:
                self._free_streams.append(live.si)
            sched.release(live.req)

        with cf.ThreadPoolExecutor(max_workers=self.slots) as pool:
            while not sched.idle() or ready:
                now = time.perf_counter() - t0
                for r in sched.admit(now):
                    res = Result(rid=r.rid, arrival=r.arrival, admitted=now)
                    results[r.rid] = res
                    setups[pool.submit(self._setup_packed, r, res, t0)] = r
                live = [m for m in lanes if not m.done]
                if not live and not ready:
                    # nothing on the GPU from this thread: wait for a setup or an arrival
                    nxt = sched.next_arrival()
                    wait = max(nxt - now, 0.0) if nxt is not None else None
                    if setups:
                        cf.wait(list(setups), timeout=wait, return_when=cf.FIRST_COMPLETED)
                    elif wait is not None:
                        time.sleep(min(wait, 0.05))
                for fut in [f for f in setups if f.done()]:
                    lv = fut.result()
                    del setups[fut]
                    if lv.res.error or lv.i >= lv.req.count():
                        complete(lv)
                    else:
                        ready.append(lv)
                idle = len(lanes) - len(live)
                if ready and (batch is None or not live or len(ready) + idle >= max(1, len(lanes) // 2)):
                    if batch is not None:
                        batch.close()
                        batch = None
                    for m in lanes:
                        if m.done:
                            m.f = None  # the plan goes once no graph uses it
                    lanes = live + ready
                    live = list(lanes)
                    ready = []
                if not live:
                    continue
                with torch.cuda.stream(bs):
                    if batch is None:
                        with self._dev_lock:
                            batch = PackedBatch([m.f for m in lanes], [m.tau for m in lanes],
                                                [m.pot for m in lanes], bs, self.check_self)
                        stats["captures"] += 1
                    seeds, index = [], []
                    for m in lanes:  # given densities are copied here; fresh ones are drawn by the batch
                        draw = not m.done and m.req.taus is None
                        if not m.done and not draw:
                            m.next_density(torch, bs)
                        seeds.append(m.req.tau_seed if draw else DRAW_SKIP)
                        index.append(m.i if draw else 0)
                    batch.set_draws(seeds, index)
                    batch.launch()
                    for m in live:
                        m.host.copy_(m.pot, non_blocking=True)
                batch.synchronize()
                sums = batch.sums()
                stats["steps"] += 1
                stats["member_steps"] += len(live)
                stats["idle_lane_steps"] += len(lanes) - len(live)
                for r, m in enumerate(lanes):
                    if m.done:
                        continue
                    m.record(self.keep_pots, float(sums[r]))
                    if m.i >= m.req.count():
                        complete(m)
                if all(m.done for m in lanes):
                    batch.close()
                    batch = None
                    for m in lanes:
                        m.f = None
                    lanes = []
            if batch is not None:
                batch.close()
        wall = time.perf_counter() - t0
        out = summarize(results, wall, self.slots, self.hbm_budget)
        out.update(stats)
        out["mean_batch"] = stats["member_steps"] / stats["steps"] if stats["steps"] else 0.0
        return results, out

    def run(self, requests, realtime=True):
        """Serve ``requests``; with realtime=True a request is not admitted
        before its arrival time (seconds from the start), otherwise all are
        present at the start.  Returns {rid: Result} and a stats dict."""
        if not realtime:
            for r in requests:
                r.arrival = 0.0
        if self.packed:
            return self._run_packed(requests, realtime)
        sched = Scheduler(requests, self.slots, self.hbm_budget)
        results = {}
        t0 = time.perf_counter()
        running = {}
        with cf.ThreadPoolExecutor(max_workers=self.slots) as pool:
            while not sched.idle():
                now = time.perf_counter() - t0
                for r in sched.admit(now):
                    res = Result(rid=r.rid, arrival=r.arrival, admitted=now)
                    results[r.rid] = res
                    running[pool.submit(self._run_one, r, res, t0)] = r
                nxt = sched.next_arrival()
                now = time.perf_counter() - t0
                # sleep until the next arrival, or (head already here but no slot
                # or memory) until a request finishes; never spin
                wait = nxt - now if nxt is not None and nxt > now else None
                if not running:
                    time.sleep(min(wait if wait is not None else 0.001, 0.05))
                    continue
                done, _ = cf.wait(list(running), timeout=wait, return_when=cf.FIRST_COMPLETED)
                for fut in done:
                    req, _ = fut.result()
                    sched.release(req)
                    del running[fut]
        wall = time.perf_counter() - t0
        return results, summarize(results, wall, self.slots, self.hbm_budget)


@dataclass
class _Live:
    """A request of the packed server between its setup and its last density."""
    req: Request
    res: Result
    si: int
    f: object = None
    x: object = None
    y: object = None
    tau: object = None
    pot: object = None
    host: object = None
    i: int = 0  # next density index
    done: bool = False

    def next_density(self, torch, stream):
        if self.req.taus is not None:
            self.tau.copy_(torch.as_tensor(np.ascontiguousarray(self.req.taus[self.i], dtype=np.float64)))
        else:
            device_density(torch, self.req.tau_seed, self.i, self.tau)

    def record(self, keep, total):
        self.res.sums.append(total)
        if keep:
            self.res.pots.append(self.host.numpy().copy())
        self.i += 1


def summarize(results, wall, slots, budget):
    lat = np.array([r.latency for r in results.values()]) * 1e3
    pts = sum(r.n * r.napply for r in results.values())
    return {
        "requests": len(results),
        "failed": sum(1 for r in results.values() if r.error),
        "wall_s": wall,
        "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
        "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
        "mean_ms": float(lat.mean()) if len(lat) else None,
        "requests_per_s": len(results) / wall if wall > 0 else None,
        "point_applies_per_s": pts / wall if wall > 0 else None,
        "slots": slots,
        "hbm_budget_bytes": budget,
    }


def make_stream(nreq, rate_per_s, seed=0, nmin=1_000, nmax=300_000, k0_frac=0.3, applies=(8, 32)):
    """Synthetic request stream: Poisson arrivals at ``rate_per_s`` (0: all at
    once); N log-uniform in [nmin, nmax]; request i seeded with 1000 + i; 70%
    Laplace, 30% K0 with k in {1, 10, 50}; 8-32 densities per request (made on
    demand, see Request); points are the 16-Gaussian mixture plus 20% unit
    circle of the 1M workload."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, nreq) if rate_per_s > 0 else np.zeros(nreq)
    arrivals = np.cumsum(gaps) - gaps[0]
    reqs = []
    for i in range(nreq):
        r = np.random.default_rng(1000 + i)
        n = int(round(10 ** r.uniform(np.log10(nmin), np.log10(nmax))))
        x, y = _mixture_points(r, n)
        k0 = r.uniform() < k0_frac
        k = float(r.choice([1.0, 10.0, 50.0])) if k0 else 0.0
        na = int(r.integers(applies[0], applies[1] + 1))
        reqs.append(Request(x=x, y=y, kernel="k0" if k0 else "laplace", k=k, nequiv=32, ncutoff=64,
                            arrival=float(arrivals[i]), rid=i, napply=na, tau_seed=1000 + i))
    return reqs


def _mixture_points(rng, n):
    nc = int(0.2 * n)
    ng = n - nc
    th = rng.uniform(0, 2 * np.pi, nc)
    cx = rng.uniform(-1, 1, 16)
    cy = rng.uniform(-1, 1, 16)
    sig = 10 ** rng.uniform(-3, -1, 16)
    lab = rng.integers(0, 16, ng)
    x = np.concatenate([cx[lab] + sig[lab] * rng.standard_normal(ng), np.cos(th)])
    y = np.concatenate([cy[lab] + sig[lab] * rng.standard_normal(ng), np.sin(th)])
    return x, y
