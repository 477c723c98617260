"""The continuous-batching serving loop (lt_server_*).

Requests of mixed kinds and sizes are submitted while others are on the GPU; each
result must equal, bit for bit, the same request evaluated alone through the server, and
the single-grid calls of the same precision (conftest.plane_close: the Hessian maps bit
for bit); admission must respect the server's HBM arena."""
import time

import numpy as np
import pytest

import lenstool_hpc_b200 as lt
from lenstool_hpc_b200 import catalog

from conftest import plane_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from lenstool_hpc_b200 import build
    build.build()
    c = lt.Context(0)
    yield c
    c.close()


def _alone(ctx, cat, g, kinds, precision, D, scale):
    import torch
    res = {}
    hk = [k for k in kinds if k not in ("potential", "deflection_x", "deflection_y")]
    dev = lambda: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")  # noqa: E731
    if hk:
        outs = [dev() for _ in hk]
        ctx.hessian_maps(cat, g, hk, precision=precision, dlsds=D, out=outs)
        res.update(zip(hk, outs))
    if "potential" in kinds:
        res["potential"] = ctx.potential_grid(cat, g, precision=precision, scale=scale, out=dev())
    if "deflection_x" in kinds:
        ax, ay = ctx.gradient_grid(cat, g, precision=precision, scale=scale, out=(dev(), dev()))
        res["deflection_x"], res["deflection_y"] = ax, ay
    ctx.synchronize()
    return {k: v.cpu().numpy() for k, v in res.items()}


KINDS = (["kappa", "gamma1", "gamma2", "mu"], ["deflection_x", "deflection_y"], ["ampli1", "potential"])


def _mixed(ctx, n, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    cats = []
    for i, nh in enumerate((50, 200, 700)):
        cats.append(ctx.upload(catalog.cluster_galaxy_catalog(max(1, nh // 100), nh - max(1, nh // 100), 40 + i)))
    out = []
    for i in range(n):
        c = cats[int(rng.integers(len(cats)))]
        size = int(rng.choice([64, 128, 256, 301]))
        g = catalog.Grid.square(100., size)
        out.append((c, g, KINDS[i % len(KINDS)]))
    return cats, out


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_server_mixed_equals_alone(ctx, precision):
    import torch
    cats, work = _mixed(ctx, 18, 1)
    D, scale = 0.55, 1.7
    expect = [_alone(ctx, c, g, kinds, precision, D, scale) for c, g, kinds in work]
    with ctx.server(precision=precision, slots=8, window=4) as srv:
        outs = []
        for i, (c, g, kinds) in enumerate(work):
            if i % 2:  # host outputs (staged in the arena), pinned
                o = {k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64).pin_memory() for k in kinds}
            else:  # device outputs
                o = {k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda") for k in kinds}
            outs.append(o)
        # the server writes device outputs from its own stream: their fills must be done
        torch.cuda.synchronize()
        tickets = [srv.submit(lt.Request(c, g, o, dlsds=D, scale=scale)) for (c, g, kinds), o in zip(work, outs)]
        for t in tickets:
            srv.wait(t, 300.)
        st = srv.stats()
        assert st["completed"] == len(work) and st["failed"] == 0
        assert st["max_inflight"] > 1  # requests overlapped on the GPU
        torch.cuda.synchronize()
        for i, (o, exp) in enumerate(zip(outs, expect)):
            for k, v in o.items():
                assert plane_close(v.cpu().numpy(), exp[k], k, precision), (precision, i, k)
        # one request alone through the server gives the same planes as in the mix, bit for bit
        mixed = {k: v.cpu().numpy() for k, v in outs[3].items()}
        c, g, kinds = work[3]
        o = {k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda") for k in kinds}
        torch.cuda.synchronize()
        t = srv.submit(lt.Request(c, g, o, dlsds=D, scale=scale))
        srv.wait(t, 300.)
        q, gpu, total = srv.times(t)
        assert 0. <= q <= total and 0. <= gpu <= total
        torch.cuda.synchronize()
        for k, v in o.items():
            assert np.array_equal(v.cpu().numpy(), mixed[k])


def test_server_admission_by_arena(ctx):
    """A small arena admits two 256^2 x 4-plane requests at a time; the rest wait and
    complete as results free the arena; a request larger than the arena is refused."""
    cats, _ = _mixed(ctx, 1, 2)
    g = catalog.Grid.square(100., 256)
    plane = 256 * 256 * 8
    arena = 2 * 4 * plane
    with ctx.server(precision="fp32c", output_bytes=arena) as srv:
        outs, tickets = [], []
        for i in range(6):
            o = {k: np.full((256, 256), np.nan) for k in ("kappa", "gamma1", "gamma2", "mu")}
            outs.append(o)
            tickets.append(srv.submit(lt.Request(cats[1], g, o, dlsds=0.6)))
        for t in tickets:
            srv.wait(t, 300.)
        st = srv.stats()
        assert st["completed"] == 6
        assert st["arena_peak"] <= st["arena_bytes"] == arena
        for o in outs[1:]:
            for k in o:
                assert np.array_equal(o[k], outs[0][k])
        big = catalog.Grid.square(100., 512)
        with pytest.raises(lt.LensError) as e:
            srv.submit(lt.Request(cats[0], big, {"kappa": np.empty((512, 512)), "mu": np.empty((512, 512)),
                                                 "gamma1": np.empty((512, 512))}))
        assert e.value.status == 6  # LT_ERR_BUDGET


def test_server_idle_exit_and_relaunch(ctx):
    """The persistent kernel leaves after idle_us without work and is relaunched by the
    next submission; catalogues released while the server runs stay valid until it ends."""
    import torch
    cat = ctx.upload(catalog.cluster_galaxy_catalog(1, 80, 9))
    g = catalog.Grid.square(50., 96)
    exp = _alone(ctx, cat, g, ["kappa"], "fp32c", 0.6, 1.0)["kappa"]
    with ctx.server(precision="fp32c", idle_us=2000) as srv:
        o1 = {"kappa": torch.empty((96, 96), dtype=torch.float64, device="cuda")}
        srv.wait(srv.submit(lt.Request(cat, g, o1, dlsds=0.6)), 120.)
        time.sleep(0.2)  # the loop kernel leaves after ~2 ms idle
        o2 = {"kappa": torch.empty((96, 96), dtype=torch.float64, device="cuda")}
        t2 = srv.submit(lt.Request(cat, g, o2, dlsds=0.6))
        srv.wait(t2, 120.)
        assert srv.stats()["loop_launches"] >= 2
        cat.release()  # deferred: the server still runs
        torch.cuda.synchronize()
        assert np.array_equal(o1["kappa"].cpu().numpy(), exp)
        assert np.array_equal(o2["kappa"].cpu().numpy(), exp)


@pytest.mark.parametrize("precision", ["fp32c", "fp64"])
def test_server_chi2_requests_in_a_mix(ctx, precision):
    """chi2 requests interleaved with map requests: each chi2 and predicted-image count
    equals lt_chi2_batch_precision's in the same precision (the grid is served by the loop
    with the same per-pixel arithmetic; the delensing and chi2 are the same kernels), and
    the map results are unchanged by the loop's yields for the delensing."""
    import torch
    from lenstool_hpc_b200.images import generate_systems
    frame = (-100., 100., -100., 100.)
    base = catalog.cluster_galaxy_catalog(2, 198, 20261203)
    dbase = ctx.upload(base)
    ic = int(np.argmax(base.b0))
    systems = generate_systems(lambda bx, by, dr: ctx.delense(dbase, frame, 1024, bx, by, dr), 12, 31, dr=0.6,
                               centre=(base.position_x[ic], base.position_y[ic]), source_radius=8.)
    rng = np.random.Generator(np.random.PCG64(17))
    models = [dbase] + [ctx.upload(catalog.perturb_catalog(base, rng)) for _ in range(3)]
    sizes = [512, 1024, 256, 768]
    expect = [ctx.chi2(m, frame, n, systems, precision=precision) for m, n in zip(models, sizes)]
    cats, work = _mixed(ctx, 8, 5)
    D, scale = 0.55, 1.7
    exp_maps = [_alone(ctx, c, g, kinds, precision, D, scale) for c, g, kinds in work]
    with ctx.server(precision=precision, slots=8, window=4) as srv:
        outs = [{k: torch.full((g.ny, g.nx), np.nan, dtype=torch.float64, device="cuda") for k in kinds}
                for c, g, kinds in work]
        torch.cuda.synchronize()
        map_t, chi_t = [], []
        for i, ((c, g, kinds), o) in enumerate(zip(work, outs)):
            map_t.append(srv.submit(lt.Request(c, g, o, dlsds=D, scale=scale)))
            if i % 2 == 0:
                k = i // 2
                chi_t.append(srv.submit_chi2(models[k], frame, sizes[k], systems))
        for t in map_t + chi_t:
            srv.wait(t, 300.)
        st = srv.stats()
        assert st["completed"] == len(map_t) + len(chi_t) and st["failed"] == 0
        for t, (chi, found) in zip(chi_t, expect):
            got, gfound = srv.chi2_result(t)
            assert gfound == found and got == chi, (precision, got, chi, gfound, found)
        torch.cuda.synchronize()
        for i, (o, exp) in enumerate(zip(outs, exp_maps)):
            for k, v in o.items():
                assert plane_close(v.cpu().numpy(), exp[k], k, precision), (precision, i, k)
        with pytest.raises(lt.LensError):
            srv.chi2_result(map_t[0])  # not a chi2 ticket


def test_lost_descriptor_times_out_and_the_loop_serves_on(ctx):
    """Failure injection on the host: the next admitted request is published without its
    descriptor (a lost message).  The loop's bounded wait for it runs out on the device
    (a 50 ms limit here), the request fails with LT_ERR_TIMEOUT through the C ABI, and the
    requests submitted before and after it complete with the results of the single-grid
    calls.  No trap, no unbounded wait: the kernel reports and leaves, the host relaunches."""
    import torch
    cat = ctx.upload(catalog.cluster_galaxy_catalog(1, 60, 17))
    g = catalog.Grid.square(60., 256)
    D = 0.6
    want = _alone(ctx, cat, g, ["kappa", "mu"], "fp32c", D, 1.0)
    dev = lambda: torch.empty((g.ny, g.nx), dtype=torch.float64, device="cuda")  # noqa: E731
    with ctx.server(precision="fp32c", slots=8, window=4, descriptor_wait_us=50000) as srv:
        before = {"kappa": dev(), "mu": dev()}
        tb = srv.submit(lt.Request(cat, g, before, dlsds=D))
        srv.wait(tb, 60.)
        srv.inject_fault(1)
        lost = srv.submit(lt.Request(cat, g, {"kappa": dev(), "mu": dev()}, dlsds=D))
        with pytest.raises(lt.LensError) as e:
            srv.wait(lost, 60.)
        assert e.value.status == 8  # LT_ERR_TIMEOUT
        after = [{"kappa": dev(), "mu": dev()} for _ in range(3)]
        tickets = [srv.submit(lt.Request(cat, g, o, dlsds=D)) for o in after]
        for t in tickets:
            srv.wait(t, 60.)
        st = srv.stats()
        assert st["timed_out"] == 1 and st["failed"] == 1 and st["completed"] == 4
    for o in [before] + after:
        for k in ("kappa", "mu"):
            assert plane_close(o[k].cpu().numpy(), want[k], k, "fp32c"), k
    # the context is usable afterwards
    m = ctx.hessian_maps(cat, g, ["kappa", "mu"], precision="fp32c", dlsds=D)
    assert np.array_equal(m["kappa"], want["kappa"]) and np.array_equal(m["mu"], want["mu"])
