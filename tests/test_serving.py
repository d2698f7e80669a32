"""The serving loop (qhk_server_*): its admission policy on the CPU, and on the device that every
request's volume is the same alone and in a mixed stream (bitwise: each request runs in its own
workspace with deterministic kernels), equal to the Pipeline and within 1e-4 of the oracle, under a
budget tight enough to force evictions, with CUDA-graph replays, from several threads."""

from __future__ import annotations

import random
import threading

import numpy as np
import pytest

from conftest import contrast_err

GiB = 1 << 30


# ---- admission policy (host only) -----------------------------------------------------------


def test_admission_reuses_idle_then_allocates_within_budget():
    from qoraholo_b200 import capi

    # registration holds 1+3 (geometry 0) + 1+2 (geometry 1) = 7 GiB; at most two requests run
    got = capi.admission_simulate(10 * GiB, 2, 2, [GiB, GiB], [3 * GiB, 2 * GiB], [0, 0, 1, -1, 0, -1, -1])
    assert got == [(0, 0, 7 * GiB), (1, 1, 10 * GiB), (2, 0, 10 * GiB), (3, 0, 10 * GiB)]


def test_admission_evicts_least_recently_used_idle_workspace():
    from qoraholo_b200 import capi

    # 9 GiB after registration; a second workspace of geometry 1 needs 3 GiB: the idle workspace of
    # geometry 0 (4 GiB) is released first
    got = capi.admission_simulate(10 * GiB, 4, 2, [GiB, GiB], [4 * GiB, 3 * GiB], [0, -1, 1, 1])
    assert got == [(0, 0, 9 * GiB), (1, 0, 9 * GiB), (2, 2, 8 * GiB)]


def test_admission_passes_over_the_head_a_bounded_number_of_times():
    from qoraholo_b200 import capi

    # a large request (geometry 0, 6 GiB workspaces) cannot start while another one runs; small
    # requests behind it are admitted past it at most max_pass = 2 times, then it gets the next
    # free workspace
    got = capi.admission_simulate(10 * GiB, 8, 2, [0, 0], [6 * GiB, GiB], [0, 0, 1, 1, 1, -1])
    assert [a for a, _, _ in got] == [0, 2, 3, 1, 4]
    assert [b for _, b, _ in got] == [0, 0, 1, 0, 1]


def test_admission_never_exceeds_budget_or_slots_and_admits_everything():
    from qoraholo_b200 import capi

    rng = random.Random(7)
    resident = [GiB // 2, GiB // 4, GiB]
    workspace = [3 * GiB, GiB, 5 * GiB]
    budget = 12 * GiB
    ops = []
    for _ in range(300):
        ops.append(rng.randrange(3) if rng.random() < 0.6 else -1)
    ops += [-1] * 400
    got = capi.admission_simulate(budget, 3, 4, resident, workspace, ops)
    submitted = sum(1 for o in ops if o >= 0)
    assert sorted(a for a, _, _ in got) == list(range(submitted))
    assert all(u <= budget for _, _, u in got)


def test_admission_rejects_a_geometry_that_cannot_fit():
    from qoraholo_b200 import capi

    with pytest.raises(ValueError):
        capi.admission_simulate(4 * GiB, 2, 2, [GiB], [4 * GiB], [0])


# ---- the server on the device -----------------------------------------------------------------

G = np.array([0.532, 1.337, 1.2, 0.2], np.float32)


def _geometry_cases():
    """Three geometries of different sizes and solvers: (name, options, hologram pixel)."""
    return [
        ("gp64", dict(count=9, hologram_size=64, center=(18, 18), radius=14.0, output_size=32, iterations=4,
                      solver="gp")),
        ("tv128", dict(count=9, hologram_size=128, center=(36, 36), radius=30.0, output_size=64, iterations=3,
                       solver="tv", tv_weight=1e-2, tv_inner=4)),
        ("c2c96", dict(count=6, hologram_size=96, center=(27, 27), radius=20.0, output_size=48, iterations=3,
                       solver="gp", gp_transform="c2c", nz=32)),
    ]


def _stack(O, opts, sample, seed):
    """Holograms and backgrounds of one geometry: spheres `sample` seen under a circular scan."""
    n, m, count = opts["hologram_size"], opts["output_size"], opts["count"]
    hg = G.copy()
    hg[3] = G[3] * m / n  # hologram pixel = field pixel * m / N
    il = O.circular_scan(count, 0.9, G)
    ratio = O.forward_fields(sample, il, hg, n)
    c = opts["center"][0] / (n * hg[3])
    holo = O.synthesize_holograms(ratio, il, hg, carrier=(c, c), noise=0.02, seed=seed)
    bg = O.synthesize_holograms(np.ones_like(ratio), il, hg, carrier=(c, c), noise=0.02, seed=1000 + seed)
    return il, holo.astype(np.float32), bg.astype(np.float32)


@pytest.fixture(scope="module")
def workload(cuda):
    """Per geometry: illuminations, background, and three distinct request stacks, plus the
    volume each request gives through the Pipeline alone."""
    import qoraholo_b200 as qh
    from oracle import qh_oracle as O

    samples = [
        np.array([[0.0, 0.0, 0.0, 2.0, 1.36]], np.float32),
        np.array([[0.0, 0.5, -0.4, 1.5, 1.37]], np.float32),
        np.array([[0.0, -0.6, 0.3, 2.2, 1.35], [0.0, -0.6, 0.3, 0.8, 1.38]], np.float32),
    ]
    out = {}
    for name, opts in _geometry_cases():
        stacks = []
        il = bg = None
        for k, s in enumerate(samples):
            il, holo, bg_k = _stack(O, opts, s, seed=k + 1)
            bg = bg_k if bg is None else bg
            stacks.append(holo)
        o = dict(opts)
        p = qh.Pipeline(o.pop("count"), o.pop("hologram_size"), o.pop("center"), il,
                        qh.Geometry(wavelength=float(G[0]), n_medium=float(G[1]), na=float(G[2]), pixel=float(G[3])),
                        **o)
        p.set_background(bg)
        alone = [p.run(h).copy() for h in stacks]
        out[name] = dict(opts=opts, il=il, bg=bg, stacks=stacks, alone=alone, filled=p.filled)
    return out


def _register(server, workload):
    ids = {}
    for name, w in workload.items():
        o = dict(w["opts"])
        ids[name] = server.add_geometry(o.pop("count"), o.pop("hologram_size"), o.pop("center"), w["il"], G, w["bg"],
                                        **o)
    return ids


def _mixed_stream(workload, repeats=3, seed=3):
    reqs = [(name, k) for name in workload for k in range(len(workload[name]["stacks"]))] * repeats
    random.Random(seed).shuffle(reqs)
    return reqs


@pytest.mark.gpu
def test_server_results_equal_alone_and_in_a_mix(workload):
    from qoraholo_b200 import capi

    with capi.Server(hbm_budget=8 * GiB, max_inflight=4) as sv:
        ids = _register(sv, workload)
        reqs = _mixed_stream(workload)
        tickets = [(sv.submit(ids[name], workload[name]["stacks"][k]), name, k) for name, k in reqs]
        for t, name, k in tickets:
            ri, filled, times = sv.wait(t)
            assert np.array_equal(ri, workload[name]["alone"][k]), (name, k)
            assert filled == workload[name]["filled"]
            assert times["total"] >= times["service"] >= 0 and times["gpu"] > 0
        st = sv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["graph_launches"] > 0 and st["peak_inflight"] > 1
        assert st["peak_used"] <= 8 * GiB


@pytest.mark.gpu
def test_server_matches_the_oracle(workload):
    """One request per geometry against the oracle's CPU restatement (1e-4, the reference's
    CPU/CUDA bar)."""
    from oracle import qh_oracle as O
    from qoraholo_b200 import capi

    with capi.Server(hbm_budget=8 * GiB, max_inflight=3) as sv:
        ids = _register(sv, workload)
        for name, w in workload.items():
            o = dict(w["opts"])
            count, n, center = o.pop("count"), o.pop("hologram_size"), o.pop("center")
            radius, out = o.pop("radius"), o.pop("output_size")
            ri = sv.wait(sv.submit(ids[name], w["stacks"][0]))[0]
            crop = dict(center=center, radius=radius, output_size=out)
            fields = O.field_ratio(O.extract_fields(w["stacks"][0], **crop), O.extract_fields(w["bg"], **crop))
            ref = O.reconstruct(O.rytov(fields), w["il"], G, **o)[0]
            assert contrast_err(ri, ref, float(G[1])) < 1e-4, name


@pytest.mark.gpu
def test_server_evicts_under_a_tight_budget_and_stays_exact(workload):
    from qoraholo_b200 import capi

    # room for the resident state and about one workspace of each geometry at a time
    probe = capi.Server(hbm_budget=64 * GiB, max_inflight=1)
    ids = _register(probe, workload)
    need = probe.stats()["used"]
    probe.close()
    with capi.Server(hbm_budget=need + need // 3, max_inflight=3) as sv:
        ids = _register(sv, workload)
        reqs = _mixed_stream(workload, repeats=2, seed=11)
        tickets = [(sv.submit(ids[name], workload[name]["stacks"][k]), name, k) for name, k in reqs]
        for t, name, k in tickets:
            assert np.array_equal(sv.wait(t)[0], workload[name]["alone"][k]), (name, k)
        st = sv.stats()
        assert st["peak_used"] <= need + need // 3
        assert st["failed"] == 0


@pytest.mark.gpu
def test_server_graph_replays_are_bitwise_equal(workload):
    from qoraholo_b200 import capi

    w = workload["tv128"]
    with capi.Server(hbm_budget=8 * GiB, max_inflight=1) as sv:
        gid = _register(sv, {"tv128": w})["tv128"]
        outs = [sv.wait(sv.submit(gid, w["stacks"][1]))[0] for _ in range(3)]
        assert sv.stats()["graph_launches"] == 2
    for o in outs:
        assert np.array_equal(o, w["alone"][1])
    with capi.Server(hbm_budget=8 * GiB, max_inflight=1, use_graphs=False) as sv:
        gid = _register(sv, {"tv128": w})["tv128"]
        assert np.array_equal(sv.wait(sv.submit(gid, w["stacks"][1]))[0], w["alone"][1])
        assert sv.stats()["graph_launches"] == 0


@pytest.mark.gpu
def test_server_accepts_submissions_from_several_threads(workload):
    from qoraholo_b200 import capi

    reqs = _mixed_stream(workload, repeats=2, seed=5)
    results = {}
    with capi.Server(hbm_budget=8 * GiB, max_inflight=4) as sv:
        ids = _register(sv, workload)

        def client(part):
            for i, (name, k) in part:
                results[i] = (name, k, sv.wait(sv.submit(ids[name], workload[name]["stacks"][k]))[0])

        items = list(enumerate(reqs))
        threads = [threading.Thread(target=client, args=(items[j::3],)) for j in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert len(results) == len(reqs)
    for name, k, ri in results.values():
        assert np.array_equal(ri, workload[name]["alone"][k])


@pytest.mark.gpu
def test_server_errors(workload):
    from qoraholo_b200 import capi

    w = workload["gp64"]
    with capi.Server(hbm_budget=8 * GiB, max_inflight=2) as sv:
        gid = _register(sv, {"gp64": w})["gp64"]
        with pytest.raises(ValueError):
            sv.submit(gid, np.zeros((3, 64, 64), np.float32))
        with pytest.raises(KeyError):
            sv.submit(gid + 7, w["stacks"][0])
        with pytest.raises(ValueError):
            sv.wait(12345)
        t = sv.submit(gid, w["stacks"][0])
        with pytest.raises(capi.QhkError) as e:
            sv.remove_geometry(gid)  # a request of it has not been waited for
        assert e.value.code == capi.LOGIC_ERROR
        sv.wait(t)
        sv.remove_geometry(gid)
        assert sv.stats()["geometries"] == 0
    with capi.Server(hbm_budget=1 << 20, max_inflight=2) as sv:
        with pytest.raises(ValueError):
            _register(sv, {"gp64": w})


@pytest.mark.gpu
def test_server_cancels_queued_requests(workload):
    """A request not admitted yet can be withdrawn: it fails with QHK_LOGIC_ERROR, takes no device
    time, and the requests around it complete unchanged."""
    from qoraholo_b200 import capi

    w = workload["tv128"]
    with capi.Server(hbm_budget=8 * GiB, max_inflight=1) as sv:
        gid = _register(sv, {"tv128": w})["tv128"]
        tickets = [sv.submit(gid, w["stacks"][k % 3]) for k in range(8)]
        withdrawn = [t for t in tickets[4:] if sv.cancel(t)]
        assert withdrawn  # one slot: the tail of the queue has not started yet
        for k, t in enumerate(tickets):
            if t in withdrawn:
                with pytest.raises(capi.QhkError) as e:
                    sv.wait(t)
                assert e.value.code == capi.LOGIC_ERROR
            else:
                assert np.array_equal(sv.wait(t)[0], w["alone"][k % 3])
        st = sv.stats()
        assert st["cancelled"] == len(withdrawn) and st["completed"] == len(tickets) - len(withdrawn)
