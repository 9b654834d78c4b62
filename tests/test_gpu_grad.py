"""Parity of the CUDA nuclear-gradient J/K build with the reference.

Expected values come from the reference (tests/golden/grad_*.npz, written by
make_grad_golden.py with PySCF's own grad.rhf.get_jk, grad.RHF and SCF
energies at displaced geometries), and from the reference's published
gradient fingerprint.  The GPU path is called through the C ABI.

Tolerances: vj/vk of grad.rhf.get_jk to 1e-10 (the J/K parity bar); the
derivative Schwarz bound to 1e-10 relative; RHF gradients to 1e-7 Eh/Bohr of
grad.RHF; against central finite differences of the reference energy
(h = 1e-4 Bohr, SCF converged to 1e-12) to 5e-6 Eh/Bohr, the precision of the
reference's own finite-difference check (pyscf/grad/test/test_rhf.py:153,
5 places): screened incremental direct-SCF energies at displaced geometries
carry ~1e-10 Eh of noise, which the 2h = 2e-4 Bohr division amplifies.
"""
import numpy
import pytest

from conftest import lib_fp

pytestmark = pytest.mark.gpu

TOL_JK = 1e-10
TOL_DE = 1e-7


def _grad_fixture(name):
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, 'golden', 'grad_%s.npz' % name)
    if not os.path.exists(path):
        pytest.skip('fixture grad_%s missing (run tests/golden/make_grad_golden.py)' % name)
    return dict(numpy.load(path))


@pytest.fixture(scope='module')
def b2():
    from pyscf_b200 import lib
    if lib.device_count() == 0:
        pytest.fail('no CUDA device visible to libb200jk')
    return lib


def _plan(b2, f):
    return b2.Plan(f['atm'], f['bas'], f['env'], cart=bool(f['cart']), direct_scf_tol=1e-13)


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz'])
def test_grad_q_cond(b2, name):
    f = _grad_fixture(name)
    q = _plan(b2, f).grad_q_cond
    ref = f['gq_cond']
    assert abs(q - ref).max() <= 1e-10 * max(1.0, abs(ref).max())


@pytest.mark.parametrize('name,dm_key,ref_key', [('h2o_631g', 'dm0', ''), ('h2o_631g', 'dm_ns', '_ns'),
                                                 ('h2o2_vtz', 'dm0', '')])
def test_grad_jk(b2, name, dm_key, ref_key):
    f = _grad_fixture(name)
    p = _plan(b2, f)
    vj, vk = p.grad_jk(f[dm_key])
    assert vj.shape == (3, int(f['nao']), int(f['nao']))
    assert abs(vj - f['gvj' + ref_key]).max() < TOL_JK
    assert abs(vk - f['gvk' + ref_key]).max() < TOL_JK
    assert p.grad_stats()['quartets'] > 0


def test_grad_jk_stack_and_unscreened(b2):
    """A stack of densities matches one-by-one builds; tol <= 0 (no screen)
    changes the result only below the screen's threshold."""
    f = _grad_fixture('h2o_631g')
    p = _plan(b2, f)
    dms = numpy.stack([f['dm0'], f['dm_ns']])
    vj, vk = p.grad_jk(dms)
    assert vj.shape == (2, 3) + f['dm0'].shape
    assert abs(vj[1] - f['gvj_ns']).max() < TOL_JK
    assert abs(vk[0] - f['gvk']).max() < TOL_JK
    vj0, vk0 = p.grad_jk(f['dm0'], direct_scf_tol=0.0)
    assert abs(vj0 - f['gvj']).max() < 1e-9
    assert abs(vk0 - f['gvk']).max() < 1e-9


def test_grad_device_pointers(b2):
    import torch
    f = _grad_fixture('h2o2_vtz')
    p = _plan(b2, f)
    vj, vk = p.grad_jk_device(torch.tensor(f['dm0'], device='cuda:0'))
    torch.cuda.synchronize()
    assert abs(vj.cpu().numpy() - f['gvj']).max() < TOL_JK
    assert abs(vk.cpu().numpy() - f['gvk']).max() < TOL_JK


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o16_vdz'])
def test_rhf_gradient(b2, name):
    """One-electron part from the reference fixture + two-electron part from
    the GPU = grad.RHF(mf).kernel(); and = finite differences of the
    reference energy."""
    from pyscf_b200 import grad
    f = _grad_fixture(name)
    p = _plan(b2, f)
    vj, vk = p.grad_jk(f['dm0'])
    de2 = grad.grad_2e(vj, vk, f['dm0'], f['aoslice'])
    assert abs(de2 - f['de_2e']).max() < TOL_DE
    de = f['de'] - f['de_2e'] + de2
    assert abs(de - f['de']).max() < TOL_DE
    h = float(f['fd_h'])
    fd = (f['fd_energies'][:, 0] - f['fd_energies'][:, 1]) / (2 * h)
    an = de.ravel()[f['fd_coords']]
    assert abs(an - fd).max() < 5e-6
    if name == 'h2o_631g':
        # pyscf/grad/test/test_rhf.py:148-153 (conv_tol 1e-14, 6 places)
        assert abs(lib_fp(de) - 0.0055115512502467556) < 5e-7


def test_autograd_two_electron_energy(b2):
    """dE2/dR from the ip1 backward kernel equals central differences of the
    GPU's own E2(R) at fixed AO density; dE2/dD = J - K/2."""
    import torch
    from pyscf_b200 import grad
    f = _grad_fixture('h2o_631g')
    coords = torch.tensor(f['coords'], dtype=torch.float64, requires_grad=True)
    dm = torch.tensor(f['dm0'], device='cuda:0', requires_grad=True)
    e2 = grad.two_electron_energy(coords, dm, f['atm'], f['bas'], f['env'])
    e2.backward()
    g = coords.grad.numpy()
    assert abs(g - f['de_2e']).max() < TOL_DE
    h = 1e-4
    c0 = f['coords']
    for t in (2, 4, 8):
        cp, cm = c0.copy(), c0.copy()
        cp[t // 3, t % 3] += h
        cm[t // 3, t % 3] -= h
        ep = grad.two_electron_energy(torch.tensor(cp), dm.detach(), f['atm'], f['bas'], f['env']).item()
        em = grad.two_electron_energy(torch.tensor(cm), dm.detach(), f['atm'], f['bas'], f['env']).item()
        assert abs((ep - em) / (2 * h) - g[t // 3, t % 3]) < 1e-7
    p = _plan(b2, f)
    vj, vk = p.get_jk(f['dm0'], hermi=1)
    assert abs(dm.grad.cpu().numpy() - (vj - 0.5 * vk)).max() < 1e-10


def test_sharded_gradient(b2):
    f = _grad_fixture('h2o2_vtz')
    vj = vk = 0
    for r in range(3):
        p = _plan(b2, f)
        p.set_shard(r, 3)
        j, k = p.grad_jk(f['dm0'])
        vj, vk = vj + j, vk + k
    assert abs(vj - f['gvj']).max() < TOL_JK
    assert abs(vk - f['gvk']).max() < TOL_JK


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz', 'h2o16_vdz'])
def test_grad_contract_fused(b2, name):
    """b200jk_grad_contract: the two-electron RHF gradient contracted inside
    the derivative kernels equals the reference's de_2e (grad_elec's
    get_veff term, pyscf/grad/rhf.py:62-68) and the host contraction of the
    engine's own vj/vk, without forming them."""
    from pyscf_b200 import grad
    f = _grad_fixture(name)
    if 'de_2e' not in f:
        pytest.skip('fixture without de_2e')
    p = _plan(b2, f)
    de = grad.grad_2e_fused(p, f['dm0'])
    assert de.shape == (int(f['atm'].shape[0]), 3)
    assert abs(de - f['de_2e']).max() < TOL_DE
    vj, vk = p.grad_jk(f['dm0'])
    host = grad.grad_2e(vj, vk, f['dm0'], f['aoslice'])
    assert abs(de - host).max() < 1e-10
    # the same from a device density, into a device array
    import torch
    ded = p.grad_contract(torch.tensor(f['dm0'], device='cuda:0'))
    assert abs(ded.cpu().numpy() - de).max() < 1e-12


def test_plan_update_coords_matches_new_plan(b2):
    """A plan moved to another geometry builds the same J/K and gradient as a
    plan created there."""
    from pyscf_b200 import grad
    f = _grad_fixture('h2o_631g')
    p = _plan(b2, f)
    p.get_jk(f['dm0'], hermi=1)
    p.int1e()
    coords = f['coords'].copy()
    coords[1, 2] += 0.05
    env2 = grad._env_with_coords(f['atm'], f['env'], coords)
    p.update_coords(env2)
    q = b2.Plan(f['atm'], f['bas'], env2, direct_scf_tol=1e-13)
    vj1, vk1 = p.get_jk(f['dm0'], hermi=1)
    vj2, vk2 = q.get_jk(f['dm0'], hermi=1)
    assert abs(vj1 - vj2).max() < 1e-12 and abs(vk1 - vk2).max() < 1e-12
    assert abs(p.grad_contract(f['dm0']) - q.grad_contract(f['dm0'])).max() < 1e-12
    assert abs(p.q_cond - q.q_cond).max() == 0.0
    # one-electron integrals follow the move too
    S1, H1 = p.int1e()
    S2, H2 = q.int1e()
    assert abs(S1 - S2).max() == 0.0 and abs(H1 - H2).max() == 0.0


def _e_nuc(atm, coords):
    z = numpy.asarray(atm)[:, 0].astype(float)
    e = 0.0
    for a in range(len(z)):
        for b in range(a):
            e += z[a] * z[b] / numpy.linalg.norm(coords[a] - coords[b])
    return e


def test_rhf_gradient_finite_differences_h2o16(b2):
    """(H2O)16/cc-pVDZ (the gradient bench workload): the analytic gradient
    (reference one-electron part + GPU two-electron part, fused) against
    central differences (h = 1e-4 Bohr) of RHF energies computed entirely on
    the GPU -- one-electron integrals, unscreened J/K, SCF to 1e-12 -- at
    the 12 seeded coordinates, to 1e-7 Eh/Bohr."""
    from pyscf_b200 import grad, rhf
    f = _grad_fixture('h2o16_vdz')
    p0 = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    de = f['de'] - f['de_2e'] + grad.grad_2e_fused(p0, f['dm0'])
    h = 1e-4
    plan = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=0.0)
    nelec = int(f['nelec'])

    def energy(coords):
        plan.update_coords(grad._env_with_coords(f['atm'], f['env'], coords))
        S, H = plan.int1e()
        conv, e, *_ = rhf.kernel(H, S, nelec, _e_nuc(f['atm'], coords), lambda d: plan.get_jk(d, hermi=1),
                                 conv_tol=1e-12, dm0=f['dm0'])
        assert conv
        return e
    c0 = f['coords']
    for t in f['fd_coords']:
        cp, cm = c0.copy(), c0.copy()
        cp[t // 3, t % 3] += h
        cm[t // 3, t % 3] -= h
        fd = (energy(cp) - energy(cm)) / (2 * h)
        assert abs(fd - de.ravel()[t]) < 1e-7, (t, fd, de.ravel()[t])


def test_autograd_two_electron_energy_h2o16(b2):
    """The autograd Function on the (H2O)16 workload: dE2/dR through the
    fused backward equals the reference's de_2e, and central differences of
    its own forward (plan moved between geometries) to 1e-7."""
    import torch
    from pyscf_b200 import grad
    f = _grad_fixture('h2o16_vdz')
    coords = torch.tensor(f['coords'], dtype=torch.float64, requires_grad=True)
    dm = torch.tensor(f['dm0'], device='cuda:0')
    e2 = grad.two_electron_energy(coords, dm, f['atm'], f['bas'], f['env'])
    e2.backward()
    g = coords.grad.numpy()
    assert abs(g - f['de_2e']).max() < TOL_DE
    h = 1e-4
    c0 = f['coords']
    for t in (5, 70, 131):
        cp, cm = c0.copy(), c0.copy()
        cp[t // 3, t % 3] += h
        cm[t // 3, t % 3] -= h
        ep = grad.two_electron_energy(torch.tensor(cp), dm, f['atm'], f['bas'], f['env']).item()
        em = grad.two_electron_energy(torch.tensor(cm), dm, f['atm'], f['bas'], f['env']).item()
        assert abs((ep - em) / (2 * h) - g[t // 3, t % 3]) < 1e-7


def _grad1e_fixture(name):
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    path = os.path.join(here, 'golden', 'grad1e_%s.npz' % name)
    if not os.path.exists(path):
        pytest.skip('fixture grad1e_%s missing (run tests/golden/make_grad1e_golden.py)' % name)
    return dict(numpy.load(path))


def _grad_nuc(atm, coords):
    """grad_nuc (pyscf/grad/rhf.py:86-107)."""
    z = atm[:, 0].astype(float)
    dr = coords[:, None, :] - coords[None]
    d = numpy.linalg.norm(dr, axis=2)
    numpy.fill_diagonal(d, numpy.inf)
    return -numpy.einsum('i,j,ijx,ij->ix', z, z, dr, 1.0 / d ** 3)


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz', 'h2o16_vdz'])
def test_grad_int1e(b2, name):
    """b200jk_grad_int1e: the hcore and overlap lines of grad_elec
    (pyscf/grad/rhf.py:57-66, hcore_generator :121-143, get_ovlp :145-146)
    against the reference's for the same dm0 and energy-weighted density, to
    1e-9 Eh/Bohr."""
    f, g1 = _grad_fixture(name), _grad1e_fixture(name)
    p = _plan(b2, f)
    de1 = p.grad_int1e(f['dm0'], g1['dme0'])
    assert abs(de1 - g1['de_1e']).max() < 1e-9, abs(de1 - g1['de_1e']).max()
    assert abs(_grad_nuc(f['atm'], f['coords']) - g1['de_nuc']).max() < 1e-12


@pytest.mark.parametrize('name', ['h2o_631g', 'h2o2_vtz', 'h2o16_vdz'])
def test_rhf_gradient_all_on_gpu(b2, name):
    """The whole RHF gradient from the GPU: one-electron part
    (b200jk_grad_int1e, W = 1/2 D F D with F from the GPU's one-electron
    integrals and J/K), two-electron part (b200jk_grad_contract) and nuclear
    repulsion, against grad.RHF, to 1e-7 Eh/Bohr."""
    from pyscf_b200 import grad
    f = _grad_fixture(name)
    p = _plan(b2, f)
    D = f['dm0']
    S, H = p.int1e()
    vj, vk = p.get_jk(D, hermi=1)
    W = 0.5 * D @ (H + vj - 0.5 * vk) @ D
    de = p.grad_int1e(D, W) + grad.grad_2e_fused(p, D) + _grad_nuc(f['atm'], f['coords'])
    assert abs(de - f['de']).max() < TOL_DE, abs(de - f['de']).max()


def test_autograd_rhf_energy(b2):
    """grad.rhf_energy: the RHF energy as a torch scalar whose backward is the
    whole SCF gradient on the GPU (one-electron, two-electron and nuclear
    parts).  At the converged density of H2O/6-31G its value is the
    reference RHF energy (1e-9 Eh) and its gradient grad.RHF (1e-7); against
    central differences (h = 1e-4 Bohr) of RHF energies converged on the GPU
    to 1e-12 at the fixture's 9 coordinates, 1e-7."""
    import torch
    from pyscf_b200 import grad, rhf
    f = _grad_fixture('h2o_631g')
    p = _plan(b2, f)
    D = f['dm0']
    S, H = p.int1e()
    vj, vk = p.get_jk(D, hermi=1)
    W = 0.5 * D @ (H + vj - 0.5 * vk) @ D
    coords = torch.tensor(f['coords'], requires_grad=True)
    e = grad.rhf_energy(coords, torch.tensor(D), torch.tensor(W), f['atm'], f['bas'], f['env'])
    e.backward()
    assert abs(e.item() - float(f['e_rhf'])) < 1e-9
    de = coords.grad.numpy()
    assert abs(de - f['de']).max() < TOL_DE, abs(de - f['de']).max()
    plan = b2.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=0.0)
    nelec = int(f['nelec'])

    def energy(c):
        plan.update_coords(grad._env_with_coords(f['atm'], f['env'], c))
        S, H = plan.int1e()
        conv, e, *_ = rhf.kernel(H, S, nelec, _e_nuc(f['atm'], c), lambda d: plan.get_jk(d, hermi=1),
                                 conv_tol=1e-12, dm0=D)
        assert conv
        return e
    h = 1e-4
    c0 = f['coords']
    for t in f['fd_coords']:
        cp, cm = c0.copy(), c0.copy()
        cp[t // 3, t % 3] += h
        cm[t // 3, t % 3] -= h
        fd = (energy(cp) - energy(cm)) / (2 * h)
        assert abs(fd - de.ravel()[t]) < 1e-7, (t, fd, de.ravel()[t])
