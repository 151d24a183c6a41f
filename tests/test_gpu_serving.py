"""Pools and the serving loop on the GPU: a pool runs the same kernels as
gemsgpu_md_steps, and a served job's result does not depend on the jobs it
shares the device with."""
import numpy as np
import pytest

gems = pytest.importorskip("gems_b200")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = gems.Context()
    yield c
    c.close()


def au():
    from gems_b200 import workloads as W
    return W.SMATB["Au"], W.MASS["Au"]


def test_pool_equals_md_steps(ctx):
    from gems_b200 import workloads as W
    sm, m = au()
    cl = [W.cluster(n, np.random.default_rng(n)) for n in (40, 200, 90)]

    def mk(p, seed):
        g = gems.System(p, m, ctx=ctx)
        g.set_smatb(*sm)
        g.set_precision(gems.PREC_MIXED)
        g.set_lanes(4, 1)
        g.set_ermak(0.002, 1.0, 500.0, seed=seed)
        return g

    a = [mk(p, 10 + k) for k, p in enumerate(cl)]
    b = [mk(p, 10 + k) for k, p in enumerate(cl)]
    for g in a + b:
        g.interact()
    ctx.batch_md_steps(a, 100)
    pool = gems.Pool(ctx, 8, 2000, ff=gems.FF_SMATB, prec=gems.PREC_MIXED, lanes=4, variant=1, chunk=50)
    pool.set(b)
    pool.run(2)
    for ga, gb in zip(a, b):
        np.testing.assert_array_equal(ga.pos, gb.pos)
        np.testing.assert_array_equal(ga.vel, gb.vel)
    pool.close()


def test_server_result_alone_equals_mixed(ctx):
    from gems_b200 import workloads as W
    sm, m = au()
    target_fire = W.cluster(147, np.random.default_rng(5), jitter=0.1)
    target_md = W.cluster(60, np.random.default_rng(6))
    srv = gems.Server(ctx, max_jobs=16, max_atoms=6000, lanes=4, variant=1, chunk=50)
    a1 = srv.submit(target_fire, m, sm, gems.JOB_FIRE, 3000, dt=0.002, fmax=1e-3)
    a2 = srv.submit(target_md, m, sm, gems.JOB_MD, 500, temp=600.0, seed=9)
    while srv.step()[0] or any(srv.poll(j)["state"] != gems.JOB_DONE for j in (a1, a2)):
        pass
    alone = [srv.poll(a1, True), srv.poll(a2, True)]
    # the same two jobs, arriving while six others run and others queue
    rng = np.random.default_rng(1)
    others = []
    for k in range(4):
        others.append(srv.submit(W.cluster(int(rng.integers(13, 400)), rng), m, sm,
                                 gems.JOB_FIRE if k % 2 else gems.JOB_MD, 300, temp=400.0, seed=100 + k))
    srv.step()
    srv.step()
    b1 = srv.submit(target_fire, m, sm, gems.JOB_FIRE, 3000, dt=0.002, fmax=1e-3)
    for k in range(4):
        others.append(srv.submit(W.cluster(int(rng.integers(13, 400)), rng), m, sm,
                                 gems.JOB_MD, 800, temp=700.0, seed=200 + k))
    srv.step()
    b2 = srv.submit(target_md, m, sm, gems.JOB_MD, 500, temp=600.0, seed=9)
    for _ in range(2000):
        srv.step()
        if all(srv.poll(j)["state"] == gems.JOB_DONE for j in [b1, b2] + others):
            break
    mixed = [srv.poll(b1, True), srv.poll(b2, True)]
    for x, y in zip(alone, mixed):
        assert x["iters"] == y["iters"]
        assert x["epot_ev"] == y["epot_ev"]
        np.testing.assert_array_equal(x["pos"], y["pos"])
    assert alone[0]["fmax_ev"] < 1e-3
    srv.close()


def test_server_admission_by_footprint(ctx):
    from gems_b200 import workloads as W
    sm, m = au()
    srv = gems.Server(ctx, max_jobs=8, max_atoms=1000, lanes=4, chunk=50)
    big = srv.submit(W.cluster(900, np.random.default_rng(1)), m, sm, gems.JOB_MD, 100, seed=1)
    small = srv.submit(W.cluster(80, np.random.default_rng(2)), m, sm, gems.JOB_MD, 100, seed=2)
    blocked = srv.submit(W.cluster(500, np.random.default_rng(3)), m, sm, gems.JOB_MD, 100, seed=3)
    tiny = srv.submit(W.cluster(13, np.random.default_rng(4)), m, sm, gems.JOB_MD, 100, seed=4)
    running, queued, _ = srv.step()
    # 900 + 80 fit; 500 does not (1480 > 1000) and waits; 13 fits behind it
    assert srv.poll(big)["state"] in (gems.JOB_RUNNING, gems.JOB_DONE)
    assert srv.poll(blocked)["state"] == gems.JOB_QUEUED
    assert srv.poll(tiny)["state"] in (gems.JOB_RUNNING, gems.JOB_DONE)
    for _ in range(50):
        srv.step()
    assert all(srv.poll(j)["state"] == gems.JOB_DONE for j in (big, small, blocked, tiny))
    with pytest.raises(gems.GemsGpuError):
        srv.submit(np.zeros((1001, 3)), m, sm, gems.JOB_MD, 100)
    srv.close()


def test_pool_refuses_what_its_step_does_not_run(ctx):
    """A pool's captured step runs velocity Verlet, Ermak and FIRE and no
    thermostat: a predictor-corrector, Brownian or thermostatted system, or
    one of another force field or precision, is refused by pool_set rather
    than advanced wrongly."""
    from gems_b200 import workloads as W
    sm, m = au()
    pool = gems.Pool(ctx, 4, 2000, ff=gems.FF_SMATB, prec=gems.PREC_MIXED, lanes=4, variant=1, chunk=50)

    def mk(setup, prec=gems.PREC_MIXED):
        g = gems.System(W.cluster(40, np.random.default_rng(3)), m, ctx=ctx)
        g.set_smatb(*sm)
        g.set_precision(prec)
        setup(g)
        return g
    ok = mk(lambda g: g.set_ermak(0.002, 1.0, 300.0))
    pool.set([ok])
    bad = [mk(lambda g: g.set_pred_corr(0.002)),
           mk(lambda g: g.set_brownian(0.002, 300.0, 1.0)),
           mk(lambda g: (g.set_vv(0.002), g.set_scalvel(300.0, 10))),
           mk(lambda g: (g.set_vv(0.002), g.set_andersen(300.0))),
           mk(lambda g: g.set_vv(0.002), prec=gems.PREC_FP64)]
    for g in bad:
        with pytest.raises(gems.GemsGpuError):
            pool.set([ok, g])
    pool.set([ok])
    pool.run(1)
    pool.close()
    for g in bad + [ok]:
        g.destroy()
