"""J-only and K-only screens (the reference's CVHFnrs8_vj_prescreen and
CVHFnrs8_vk_prescreen, pyscf/lib/vhf/optimizer.c:119-167), which SCF.get_jk
switches to when only one of J, K is built (pyscf/scf/hf.py:2069-2077).

The workload is a chain of waters in 6-31G built from the H2O/6-31G fixture
(segmented basis: a segment quartet is a shell quartet, so the engine's count
is the reference's count) with a block-diagonal density (one random block per
water): quartets between two waters then pass the J terms of the screen but
not the K terms, so the three screens keep different quartet sets.  The
engine's quartet count must equal the oracle's count of the same screen
(oracle/count.py restates optimizer.c:90-167 over CVHFdot_nrs8's quartet
set), and J/K must match the unscreened oracle J/K within the screen's
tolerance.
"""
import numpy
import pytest

from conftest import load_fixture

pytestmark = pytest.mark.gpu


def water_chain(f, n, spacing=3.0 / 0.52917721092):
    """(H2O)n along x from one water's atm/bas/env (coordinates in Bohr)."""
    atm0, bas0, env0 = f['atm'], f['bas'], f['env']
    env = list(env0)
    atm, bas = [], []
    for w in range(n):
        for a in atm0:
            row = a.copy()
            p = int(a[1])
            row[1] = len(env)
            env.extend([env0[p] + w * spacing, env0[p + 1], env0[p + 2]])
            atm.append(row)
        for b in bas0:
            row = b.copy()
            row[0] += w * atm0.shape[0]
            bas.append(row)
    return numpy.array(atm, numpy.int32), numpy.array(bas, numpy.int32), numpy.array(env)


def block_density(bas, n_water, seed=7):
    l = bas[:, 1]
    ao_loc = numpy.concatenate([[0], numpy.cumsum(2 * l + 1)])
    nao = ao_loc[-1]
    per = nao // n_water
    rng = numpy.random.default_rng(seed)
    dm = numpy.zeros((nao, nao))
    for w in range(n_water):
        a = rng.uniform(-1, 1, (per, per))
        dm[w * per:(w + 1) * per, w * per:(w + 1) * per] = a + a.T
    return dm


@pytest.fixture(scope='module')
def chain():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    f = load_fixture('h2o_631g')
    atm, bas, env = water_chain(f, 6)
    dm = block_density(bas, 6)
    return atm, bas, env, dm


@pytest.mark.parametrize('screen, with_j, with_k', [(0, 1, 1), (1, 1, 0), (2, 0, 1)])
def test_screen_counts_and_values(chain, screen, with_j, with_k):
    import oracle
    from oracle.count import count_quartets
    from pyscf_b200 import lib
    atm, bas, env, dm = chain
    tol = 1e-13
    plan = lib.Plan(atm, bas, env, direct_scf_tol=tol)
    plan.set_prescreen(screen)
    vj, vk = plan.get_jk(dm, hermi=1, with_j=bool(with_j), with_k=bool(with_k))
    n_engine = plan.stats()['quartets']
    n_ref = count_quartets(plan.q_cond, oracle.dm_cond(dm, bas), tol, screen=screen)
    assert n_engine == n_ref
    rj, rk, _ = oracle.get_jk(dm, atm, bas, env, hermi=1, screen=False)
    if with_j:
        assert abs(vj - rj).max() < 1e-10
    if with_k:
        assert abs(vk - rk).max() < 1e-10


def test_screens_differ_on_this_workload(chain):
    """The block-diagonal density makes the three screens keep different
    quartet sets (otherwise the count test above would prove nothing)."""
    import oracle
    from oracle.count import count_quartets
    from pyscf_b200 import lib
    atm, bas, env, dm = chain
    plan = lib.Plan(atm, bas, env, direct_scf_tol=1e-13)
    dmc = oracle.dm_cond(dm, bas)
    n = [count_quartets(plan.q_cond, dmc, 1e-13, screen=s) for s in (0, 1, 2)]
    assert n[1] < n[0] and n[2] < n[0] and n[1] != n[2]


def test_vhfopt_prescreen_follows_temporary_env(chain):
    """SCF.get_jk sets vhfopt.prescreen with lib.temporary_env around a J-only
    build; the drop-in VHFOpt passes the current screen to each build."""
    from pyscf_b200 import _vhf

    class Mol:
        pass
    atm, bas, env, dm = chain
    mol = Mol()
    mol._atm, mol._bas, mol._env, mol.cart = atm, bas, env, False
    opt = _vhf.VHFOpt(mol, direct_scf_tol=1e-13)
    _vhf.direct(dm, atm, bas, env, opt, hermi=1, with_k=False)
    n_s8 = opt.plan.stats()['quartets']
    saved = opt.prescreen
    opt.prescreen = 'CVHFnrs8_vj_prescreen'
    try:
        _vhf.direct(dm, atm, bas, env, opt, hermi=1, with_k=False)
        n_vj = opt.plan.stats()['quartets']
    finally:
        opt.prescreen = saved
    _vhf.direct(dm, atm, bas, env, opt, hermi=1, with_k=False)
    assert opt.plan.stats()['quartets'] == n_s8
    assert n_vj < n_s8
