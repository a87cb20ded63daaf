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

Results do not depend on what else runs: every request has its own plan and
buffers, and the kernels are deterministic.  ``tests/test_serving.py`` checks
that a request gives the same potentials alone and in the mix.
"""
import concurrent.futures as cf
import threading
import time
from dataclasses import dataclass, field

import numpy as np

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


def device_density(torch, seed, i, out):
    """Fresh N(0,1) density i of a request, drawn into the CUDA tensor ``out``
    by a generator seeded with (seed, i): the same numbers alone and in any mix."""
    g = torch.Generator(device=out.device)
    g.manual_seed(int(seed) * 4096 + int(i))
    out.normal_(0.0, 1.0, generator=g)


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
                 graphs=True):
        import torch
        self.keep_pots = bool(keep_pots)
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
        dev = torch.device("cuda", self.device)
        self._streams = [torch.cuda.Stream(dev) for _ in range(self.slots)]
        self._free_streams = list(range(self.slots))
        self._lock = threading.Lock()

    def _kernel(self, req):
        if req.kernel == "laplace":
            return C.LaplaceKernel()
        if req.kernel == "k0":
            return C.ModifiedHelmholtzKernel(req.k)
        raise ValueError(f"unknown kernel {req.kernel!r}")

    def _run_one(self, req, res, t0):
        torch = self.torch
        with self._lock:
            si = self._free_streams.pop()
        s = self._streams[si]
        try:
            dev = torch.device("cuda", self.device)
            with torch.cuda.device(dev), torch.cuda.stream(s):
                kern = self._kernel(req)
                xd = torch.as_tensor(np.ascontiguousarray(req.x, dtype=np.float64), device=dev)
                yd = torch.as_tensor(np.ascontiguousarray(req.y, dtype=np.float64), device=dev)
                f = C.FMM(xd, yd, C.Get_Kernel_Functions(kern), C.prepare_numba_functions_on_the_fly(kern),
                          req.nequiv, req.ncutoff, precision=self.precision, device=self.device,
                          stream=s.cuda_stream)
                f.build_tree()
                f.precompute()
                n = len(req.x)
                tau_d = torch.empty(n, dtype=torch.float64, device=dev)
                pot_d = torch.empty(n, dtype=torch.float64, device=dev)
                for i in range(req.count()):
                    if req.taus is not None:
                        tau_d.copy_(torch.as_tensor(np.ascontiguousarray(req.taus[i], dtype=np.float64)))
                    else:
                        device_density(torch, req.tau_seed, i, tau_d)
                    if not self.graphs:
                        f.build_expansions(tau_d)
                        f.evaluate_to_points(xd, yd, self.check_self, out=pot_d)
                    elif i == 0:
                        f.capture_apply(tau_d, pot_d, self.check_self)
                    else:
                        f.replay()
                    pot = pot_d.cpu().numpy()
                    res.sums.append(float(pot.sum()))
                    if self.keep_pots:
                        res.pots.append(pot)
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

    def run(self, requests, realtime=True):
        """Serve ``requests``; with realtime=True a request is not admitted
        before its arrival time (seconds from the start), otherwise all are
        present at the start.  Returns {rid: Result} and a stats dict."""
        if not realtime:
            for r in requests:
                r.arrival = 0.0
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
