"""Serving loop: admission on CPU; on the GPU, graph replay against the plain
apply and each request's result alone against the same request in a mix.

Tolerance: the kernels are deterministic and every request has its own plan
and buffers, so alone/in-mix and replay/plain potentials are compared at 1e-12
relative to the largest potential (they are expected to be identical)."""
import numpy as np
import pytest

from conftest import has_gpu
from pykifmm2d_b200 import serving as S

TOL = 1e-12


def _req(rid, n, arrival=0.0):
    return S.Request(x=np.zeros(n), y=np.zeros(n), taus=[np.zeros(n)], arrival=arrival, rid=rid)


def test_scheduler_respects_slots_and_arrival_order():
    reqs = [_req(i, 1000, arrival=0.1 * i) for i in range(6)]
    sch = S.Scheduler(reqs, slots=2, budget=1 << 40)
    assert [r.rid for r in sch.admit(0.0)] == [0]
    assert [r.rid for r in sch.admit(0.25)] == [1]          # slot limit: 2 active
    assert sch.admit(0.25) == []
    sch.release(reqs[0])
    assert [r.rid for r in sch.admit(0.25)] == [2]
    assert sch.admit(0.25) == []                            # rid 3 has not arrived yet


def test_scheduler_memory_budget_head_of_line():
    est = {0: 60, 1: 50, 2: 10}
    reqs = [_req(i, 10) for i in range(3)]
    sch = S.Scheduler(reqs, slots=8, budget=100, estimate=lambda r: est[r.rid])
    assert [r.rid for r in sch.admit(0.0)] == [0]           # 60 + 50 > 100: rid 1 waits, rid 2 may not overtake
    sch.release(reqs[0])
    assert [r.rid for r in sch.admit(0.0)] == [1, 2]
    big = [S.Request(x=np.zeros(5), y=np.zeros(5), taus=[], rid=9)]
    sch2 = S.Scheduler(big, slots=2, budget=1, estimate=lambda r: 1000)
    assert [r.rid for r in sch2.admit(0.0)] == [9]          # larger than the budget: runs alone


def test_estimate_grows_with_n_and_nequiv():
    assert S.estimate_plan_bytes(10_000) < S.estimate_plan_bytes(100_000)
    assert S.estimate_plan_bytes(10_000, nequiv=24) < S.estimate_plan_bytes(10_000, nequiv=40)


def test_make_stream_shapes():
    reqs = S.make_stream(5, rate_per_s=100.0, seed=3, nmin=1000, nmax=5000, applies=(2, 3))
    assert len(reqs) == 5 and reqs[0].arrival == 0.0
    assert all(np.all(np.diff([r.arrival for r in reqs]) >= 0) for _ in [0])
    for r in reqs:
        assert 1000 <= len(r.x) <= 5000 and 2 <= r.count() <= 3
        assert r.kernel in ("laplace", "k0")
        assert r.taus is None and r.tau_seed == 1000 + r.rid


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_device_densities_are_fresh_normals():
    """Each density of a request is its own N(0,1) draw on the device, the same
    on every call (seeded by request and density index)."""
    r = S.make_stream(1, rate_per_s=0.0, seed=3, nmin=20000, nmax=20000, applies=(3, 3))[0]
    d = [r.density(i) for i in range(3)]
    assert np.array_equal(d[1], r.density(1))
    for i in range(3):
        assert abs(d[i].mean()) < 0.05 and abs(d[i].std() - 1.0) < 0.05
    assert abs(np.corrcoef(d[0], d[1])[0, 1]) < 0.05 and abs(np.corrcoef(d[1], d[2])[0, 1]) < 0.05


gpu = [pytest.mark.gpu, pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_graph_replay_matches_plain_apply():
    import torch

    import pykifmm2d_b200 as P
    rng = np.random.default_rng(5)
    n = 30_000
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    taus = [rng.standard_normal(n) for _ in range(3)]
    kern = P.LaplaceKernel()
    xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        f = P.FMM(xd, yd, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), 32, 64,
                  precision="mixed", stream=s.cuda_stream)
        f.build_tree()
        f.precompute()
        tau_d = torch.empty(n, dtype=torch.float64, device="cuda")
        pot_d = torch.empty_like(tau_d)
        got = []
        for i, t in enumerate(taus):
            tau_d.copy_(torch.from_numpy(t))
            if i == 0:
                f.capture_apply(tau_d, pot_d, True)
            else:
                f.replay()
            got.append(pot_d.cpu().numpy())
        f.synchronize()
    g = P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), 32, 64,
              precision="mixed")
    for t, p in zip(taus, got):
        g.build_expansions(t)
        ref = g.evaluate_to_points(x, y, True)
        assert _rel(p, ref) <= TOL


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_each_result_same_alone_and_in_the_mix():
    reqs = S.make_stream(8, rate_per_s=0.0, seed=11, nmin=2_000, nmax=40_000, k0_frac=0.4, applies=(2, 4))
    mix, st_mix = S.Server(slots=4).run(reqs, realtime=False)
    assert st_mix["failed"] == 0, [r.error for r in mix.values() if r.error]
    alone, st_alone = S.Server(slots=1).run(reqs, realtime=False)
    assert st_alone["failed"] == 0
    kinds = set()
    for rid, r in mix.items():
        a = alone[rid]
        assert len(r.pots) == len(a.pots) == reqs[rid].count()
        for p, q in zip(r.pots, a.pots):
            assert _rel(p, q) <= TOL
        kinds.add(reqs[rid].kernel)
    assert kinds == {"laplace", "k0"}
    assert st_mix["p99_ms"] >= st_mix["p50_ms"] > 0


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_packed_batch_matches_each_plans_own_apply():
    """kifmm_batch_capture / kifmm_batch_launch: Laplace and K0 plans of
    different sizes (one small enough to be a single leaf) in one packed graph,
    three densities; each plan's potentials against its own unpacked apply."""
    import torch

    import pykifmm2d_b200 as P
    rng = np.random.default_rng(21)
    specs = [(25_000, P.LaplaceKernel()), (7_000, P.ModifiedHelmholtzKernel(10.0)), (50, P.LaplaceKernel()),
             (60_000, P.ModifiedHelmholtzKernel(1.0)), (12_000, P.LaplaceKernel())]
    bs = torch.cuda.Stream()
    fmms, xs, taus, pots, hosts = [], [], [], [], []
    for n, kern in specs:
        x, y = S._mixture_points(rng, n)
        xs.append((x, y, kern))
        s = torch.cuda.Stream()
        xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
        f = P.FMM(xd, yd, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), 32, 64,
                  precision="mixed", stream=s.cuda_stream)
        f.build_tree()
        f.precompute()
        fmms.append(f)
        taus.append(torch.empty(n, dtype=torch.float64, device="cuda"))
        pots.append(torch.empty(n, dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    dens = [[rng.standard_normal(n) for n, _ in specs] for _ in range(3)]
    with torch.cuda.stream(bs):
        for t, d in zip(taus, dens[0]):
            t.copy_(torch.from_numpy(d))
        b = S.PackedBatch(fmms, taus, pots, bs)
        tiles, leaves = b.info()
        assert tiles > 0 and leaves > 0
        got = []
        for k in range(3):
            for t, d in zip(taus, dens[k]):
                t.copy_(torch.from_numpy(d))
            b.launch()
            got.append([p.cpu().numpy() for p in pots])
        b.synchronize()
        b.close()
    for r, (x, y, kern) in enumerate(xs):
        g = P.FMM(x, y, P.Get_Kernel_Functions(kern), P.prepare_numba_functions_on_the_fly(kern), 32, 64,
                  precision="mixed")
        for k in range(3):
            g.build_expansions(dens[k][r])
            ref = g.evaluate_to_points(x, y, True)
            assert _rel(got[k][r], ref) <= TOL, (r, k)


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA GPU")
def test_packed_server_same_alone_and_in_the_mix():
    """Packed serving: each request's potentials in the packed mix against the
    same request served alone (one at a time, unpacked)."""
    reqs = S.make_stream(10, rate_per_s=0.0, seed=12, nmin=500, nmax=40_000, k0_frac=0.4, applies=(2, 5))
    mix, st = S.Server(slots=6, packed=True).run(reqs, realtime=False)
    assert st["failed"] == 0, [r.error for r in mix.values() if r.error]
    assert st["captures"] >= 1 and st["mean_batch"] > 1
    alone, st_alone = S.Server(slots=1).run(reqs, realtime=False)
    assert st_alone["failed"] == 0
    for rid, r in mix.items():
        a = alone[rid]
        assert len(r.pots) == len(a.pots) == reqs[rid].count()
        for p, q in zip(r.pots, a.pots):
            assert _rel(p, q) <= TOL
