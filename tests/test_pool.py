"""Element pools (include/dgmx_pool.h): many independent LSRK14 solves stepped
together by one persistent stage launch per (physics, order) arena.

Bars: each pooled FP64 solve equals the same solve run alone through
dgmx_advance (the last step shortened to land on its end time) and agrees
with the FP64 oracle to 1e-12; a solve's result is bit-for-bit the same
alone and in a mix that changes while it runs; the mixed form stays within
1e-6 of the FP64 oracle; the memory budget refuses admission and frees on
removal; a non-physical state names its solve.
"""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


IV = lambda x, y, z: ics.isentropic_vortex(x, y, beta=5.0, period=(10.0, 10.0))
IV2 = lambda x, y, z: ics.isentropic_vortex(x, y, beta=3.0, x0=1.0, y0=-0.5, period=(10.0, 10.0))
TG = lambda x, y, z: ics.taylor_green(x, y, z, Ma=0.1)
GB = lambda x, y, z: ics.gaussian_bump(x, y, a=0.3, w=0.5)

# name, physics, dim, n, lo, hi, p, ic, dt, t_end
SOLVES = [
    ("vortex-p3", 1, 2, (6, 5), -5, 5, 3, IV, 0.01, 0.047),
    ("vortex-p5", 1, 2, (4, 4), -5, 5, 5, IV2, 0.005, 0.0312),
    ("bump-p2", 30, 2, (5, 4), -2, 2, 2, GB, 0.001, 0.0057),
    ("tgv-p3", 8, 3, (2, 3, 2), 0, 2 * np.pi, 3, TG, 0.002, 0.0075),
]


def steps_of(dt, t_end):
    """The steps the pool takes: dt until the last one, shortened to land on t_end."""
    t, hs = 0.0, []
    while True:
        h = min(dt, t_end - t)
        hs.append(h)
        t = t_end if h < dt else t + h
        if t_end - t <= 1e-12 * max(abs(t_end), dt):
            return hs


def mesh_ic(case):
    import dgm_b200
    _, phys, dim, n, lo, hi, p, ic, dt, t_end = case
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux="laxfriedrichs")
    if phys == oracle.SHALLOW:
        P.set_sw_balance(False)
    x, y, z = P.coords()
    return m, P, ic(x, y, z)


def run_pool(pool, cases):
    ids = {}
    for c in cases:
        m, _, f = mesh_ic(c)
        ids[c[0]] = pool.add(m, c[1], f, c[8], c[9])
    for _ in range(100):
        pool.step(10)
        if pool.stats()[2] == 0:
            break
    return ids


def test_pool_matches_lone_domains_and_oracle():
    import dgm_b200
    pool = dgm_b200.Pool(dgm_b200.FP64)
    ids = run_pool(pool, SOLVES)
    done = set(pool.finished())
    assert done == set(ids.values())
    for c in SOLVES:
        name, phys, dt, t_end = c[0], c[1], c[8], c[9]
        sid = ids[name]
        t, nst, fin = pool.info(sid)
        hs = steps_of(dt, t_end)
        assert fin and t == t_end and nst == len(hs), (name, t, nst, len(hs))
        m, P, f = mesh_ic(c)
        D = dgm_b200.Domain(m, phys, inttype=dgm_b200.LSRK14, sw_balance=False)
        D.set_state(f)
        P.set_state(P.project(f))
        for h in hs:
            D.advance(h, 1)
            P.advance(14, h, 1)
        got = pool.state(sid)
        assert rel(got, D.state()) <= 1e-14, name
        assert rel(got, P.state()) <= 1e-12, name
    assert pool.launch_count() > 0


def test_same_result_alone_and_in_a_changing_mix():
    import dgm_b200
    target = SOLVES[0]
    alone = dgm_b200.Pool(dgm_b200.FP64)
    a_ids = run_pool(alone, [target])
    ref = alone.state(a_ids[target[0]])

    mix = dgm_b200.Pool(dgm_b200.FP64)
    # a solve of the same (physics, order) ahead of the target in its arena
    ma, _, fa = mesh_ic(("ahead", 1, 2, (3, 5), -5, 5, 3, IV2, 0.01, 1.0))
    first = mix.add(ma, 1, fa, 0.01, 1.0)
    m1, _, f1 = mesh_ic(SOLVES[1])
    mix.add(m1, SOLVES[1][1], f1, SOLVES[1][8], 1.0)              # runs throughout
    mix.step(3)
    m0, _, f0 = mesh_ic(target)
    sid = mix.add(m0, target[1], f0, target[8], target[9])        # joins mid-run
    m2, _, f2 = mesh_ic(SOLVES[2])
    mix.add(m2, SOLVES[2][1], f2, SOLVES[2][8], SOLVES[2][9])     # other physics
    mix.step(2)
    mix.remove(first)                                             # leaves mid-run
    m3, _, f3 = mesh_ic(SOLVES[3])
    mix.add(m3, SOLVES[3][1], f3, SOLVES[3][8], 0.02)
    for _ in range(20):
        mix.step(1)
        if mix.info(sid)[2]:
            break
    assert mix.info(sid)[2]
    assert np.array_equal(mix.state(sid), ref)


@pytest.mark.parametrize("case", [SOLVES[0], SOLVES[2], SOLVES[3]], ids=lambda c: c[0])
def test_mixed_pool_within_1e6_of_fp64_oracle(case):
    import dgm_b200
    pool = dgm_b200.Pool(dgm_b200.MIXED)
    ids = run_pool(pool, [case])
    m, P, f = mesh_ic(case)
    P.set_state(P.project(f))
    for h in steps_of(case[8], case[9]):
        P.advance(14, h, 1)
    err = rel(pool.state(ids[case[0]]), P.state())
    assert err <= 1e-6, err


def test_budget_refuses_and_frees():
    import dgm_b200
    pool = dgm_b200.Pool(dgm_b200.FP64, budget_bytes=12 << 20, autotune=False)
    m, _, f = mesh_ic(("v", 1, 2, (16, 16), -5, 5, 3, IV, 0.01, 0.05))
    admitted = []
    with pytest.raises(dgm_b200.PoolFull):
        for _ in range(64):
            admitted.append(pool.add(m, 1, f, 0.01, 0.05))
    assert len(admitted) >= 1
    assert pool.stats()[0] <= 12 << 20
    pool.remove(admitted[0])
    again = pool.add(m, 1, f, 0.01, 0.05)
    pool.step(10)
    assert pool.info(again)[2]


def test_nonphysical_state_names_its_solve():
    import dgm_b200
    pool = dgm_b200.Pool(dgm_b200.FP64, autotune=False)
    m, _, f = mesh_ic(SOLVES[0])
    good = pool.add(m, 1, f, 0.01, 0.05)
    bad_f = f.copy()
    bad_f[0, : bad_f.shape[1] // 3] = -1.0       # negative density
    bad = pool.add(m, 1, bad_f, 0.01, 0.05)
    with pytest.raises(dgm_b200.NonPhysicalState, match=f"solve {bad}"):
        pool.step(1)
    assert pool.info(good)[1] == 1


def _order_mix():
    """Euler 2-D vortices at p = 2..7 and shallow-water bumps at p = 2, 3
    (q = p + 2), one solve each, of uneven sizes."""
    cases = []
    for k, p in enumerate(range(2, 8)):
        n = (3 + k % 3, 4 + k % 2)
        cases.append((f"vortex-p{p}", 1, 2, n, -5, 5, p, IV if k % 2 else IV2, 0.004, 0.02))
    cases.append(("bump-p2", 30, 2, (5, 4), -2, 2, 2, GB, 0.001, 0.004))
    cases.append(("bump-p3", 30, 2, (3, 6), -2, 2, 3, GB, 0.001, 0.004))
    return cases


def test_fused_multi_order_launch_is_one_per_stage():
    """The 2-D arenas of every order step together: 14 launches per step
    (one per LSRK stage) whatever the mix of orders and physics; the same
    pool stepped per arena issues 14 per arena."""
    import dgm_b200
    cases = _order_mix()
    counts = {}
    for fused in (True, False):
        pool = dgm_b200.Pool(dgm_b200.FP64, fused=fused)
        for c in cases:
            m, _, f = mesh_ic(c)
            pool.add(m, c[1], f, c[8], c[9])
        pool.step(1)
        l0 = pool.launch_count()
        pool.step(2)
        counts[fused] = (pool.launch_count() - l0) // 2
        pool.close()
    arenas = len({(c[1], c[6]) for c in cases})
    assert counts[True] == 14, counts
    assert counts[False] == 14 * arenas, counts


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_fused_and_per_arena_paths_agree(precision):
    """One fused launch per stage across orders gives each solve the result
    of its own arena's launches (the same stage body per element)."""
    import dgm_b200
    cases = _order_mix()
    states = {}
    for fused in (True, False):
        pool = dgm_b200.Pool(precision, fused=fused)
        ids = run_pool(pool, cases)
        states[fused] = {name: pool.state(sid) for name, sid in ids.items()}
        pool.close()
    for name in states[True]:
        assert rel(states[True][name], states[False][name]) <= (1e-14 if precision == 0 else 1e-6), name


def test_async_steps_overlap_admission_with_the_same_results():
    """Steps enqueued without a wait (dgmx_pool_step_async) while new solves
    are admitted give each solve the result of the synchronous sequence;
    finished() asks for the sync first."""
    import dgm_b200
    first, second = SOLVES[0], SOLVES[2]
    res = {}
    for mode in ("sync", "async"):
        pool = dgm_b200.Pool(dgm_b200.FP64)
        m0, _, f0 = mesh_ic(first)
        a = pool.add(m0, first[1], f0, first[8], first[9])
        m1, _, f1 = mesh_ic(second)
        if mode == "sync":
            pool.step(1)
            b = pool.add(m1, second[1], f1, second[8], second[9])
        else:
            pool.step_async(1)
            b = pool.add(m1, second[1], f1, second[8], second[9])   # while the step runs
            with pytest.raises(dgm_b200.DgmxError):
                pool.finished()
            pool.sync()
        for _ in range(20):
            pool.step(1)
            if pool.stats()[2] == 0:
                break
        res[mode] = (pool.state(a), pool.state(b))
        pool.close()
    assert np.array_equal(res["sync"][0], res["async"][0])
    assert np.array_equal(res["sync"][1], res["async"][1])
