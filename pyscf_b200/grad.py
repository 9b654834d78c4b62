"""Nuclear gradients of the two-electron energy on the GPU.

``get_jk(mol, dm)`` is the drop-in for ``pyscf.grad.rhf.get_jk``
(pyscf/grad/rhf.py:149-178): J/K with the first bra function differentiated
(libcint's int2e_ip1), screened as CVHFgrad_jk_prescreen does with the
reference's threshold 1e-14, returned negated, shape (3, nao, nao) per
density.  ``patch_pyscf_grad()`` rebinds it in an unmodified PySCF, where
``GradientsBase.get_jk`` looks it up through the module (pyscf/grad/rhf.py:321).

``grad_2e(vj, vk, dm, aoslice)`` contracts that result into the two-electron
part of the RHF gradient, the term grad_elec adds (pyscf/grad/rhf.py:62-68):
    de[A] = 2 sum_x sum_{i in A} sum_j (vj - vk/2)[x, i, j] D[i, j];
``grad_2e_fused(plan, dm)`` gets the same (natm, 3) array from the GPU without
forming vj/vk (b200jk_grad_contract: the quartets are contracted with
D (x) D inside the derivative kernels).

``TwoElectronEnergy`` is a torch.autograd.Function of the nuclear coordinates
(and the density): forward builds J/K on the GPU for the geometry and returns
E2 = 1/2 tr(D J) - 1/4 tr(D K); backward runs the fused int2e_ip1 kernels and
returns dE2/dR (at fixed AO density) and dE2/dD = J - K/2.  One plan per
molecule is kept and moved to each new geometry (b200jk_plan_update_coords).
"""
import numpy

from . import lib

GRAD_SCREEN_TOL = 1e-14     # _VHFOpt's default threshold in grad.rhf.get_jk
PTR_COORD = 1


def aoslice_by_atom(atm, bas, cart=False):
    """(natm, 2) AO ranges of every atom (shells of an atom are contiguous in _bas)."""
    bas = numpy.asarray(bas)
    l = bas[:, 1]
    nf = ((l + 1) * (l + 2) // 2 if cart else 2 * l + 1) * bas[:, 3]
    ao_loc = numpy.concatenate([[0], numpy.cumsum(nf)])
    natm = len(atm)
    out = numpy.zeros((natm, 2), dtype=numpy.int64)
    for a in range(natm):
        idx = numpy.where(bas[:, 0] == a)[0]
        if len(idx):
            out[a] = ao_loc[idx[0]], ao_loc[idx[-1] + 1]
        else:
            out[a] = ao_loc[-1], ao_loc[-1]
    return out


_plans = {}


def _plan_for(mol):
    key = (id(mol), mol._env.tobytes(), mol._bas.tobytes(), mol._atm.tobytes(), bool(mol.cart))
    p = _plans.get(key)
    if p is None:
        _plans.clear()
        p = lib.Plan(mol._atm, mol._bas, mol._env, cart=bool(mol.cart), direct_scf_tol=1e-13)
        _plans[key] = p
    return p


def get_jk(mol, dm):
    """pyscf.grad.rhf.get_jk(mol, dm) on the GPU: (vj, vk), each (3, nao, nao)
    for one density or (n_dm, 3, nao, nao) for a stack."""
    dm = numpy.asarray(dm, dtype=numpy.double)
    return _plan_for(mol).grad_jk(dm, direct_scf_tol=GRAD_SCREEN_TOL)


def grad_2e(vj, vk, dm, aoslice):
    """Two-electron part of the RHF nuclear gradient from grad_jk's output."""
    vhf = vj - 0.5 * vk
    return numpy.array([2.0 * numpy.einsum('xij,ij->x', vhf[:, p0:p1], dm[p0:p1]) for p0, p1 in aoslice])


def grad_2e_fused(plan, dm, direct_scf_tol=GRAD_SCREEN_TOL):
    """The same (natm, 3) two-electron gradient of a symmetric density, with
    the contraction fused into the derivative kernels (no vj/vk formed)."""
    return plan.grad_contract(dm, direct_scf_tol=direct_scf_tol)


# one plan per molecule for TwoElectronEnergy, moved between geometries
_ad_plans = {}


def _ad_plan(atm, bas, env, cart, device):
    key = (numpy.asarray(atm).tobytes(), numpy.asarray(bas).tobytes(), bool(cart), int(device))
    p = _ad_plans.get(key)
    if p is None:
        if len(_ad_plans) >= 4:
            _ad_plans.pop(next(iter(_ad_plans))).close()
        p = lib.Plan(atm, bas, env, cart=bool(cart), direct_scf_tol=1e-13, device=device)
        _ad_plans[key] = p
    elif not numpy.array_equal(p.env, env):
        p.update_coords(env)
    return p


_saved = {}


def patch_pyscf_grad():
    """Route pyscf.grad.rhf.get_jk (RHF/RKS nuclear gradients) through the GPU."""
    import pyscf.grad.rhf as ref
    if _saved:
        return
    _saved['get_jk'] = ref.get_jk
    ref.get_jk = get_jk


def unpatch_pyscf_grad():
    import pyscf.grad.rhf as ref
    if not _saved:
        return
    ref.get_jk = _saved.pop('get_jk')


def _env_with_coords(atm, env, coords):
    env = numpy.array(env, dtype=numpy.double, copy=True)
    for a, row in enumerate(numpy.asarray(atm)):
        p = int(row[PTR_COORD])
        env[p:p + 3] = coords[a]
    return env


def _torch_function():
    import torch

    class TwoElectronEnergy(torch.autograd.Function):
        """E2(R, D) = 1/2 tr(D J[D]) - 1/4 tr(D K[D]) for a symmetric AO density
        D at nuclear coordinates R (Bohr, (natm, 3)); J/K and the ip1 backward
        run on the GPU.  Usage:
            E2 = TwoElectronEnergy.apply(coords, dm, atm, bas, env, cart)
        """

        @staticmethod
        def forward(ctx, coords, dm, atm, bas, env, cart=False):
            c = coords.detach().cpu().numpy().astype(numpy.double)
            env2 = _env_with_coords(atm, env, c)
            plan = _ad_plan(atm, bas, env2, cart, dm.device.index if dm.is_cuda else 0)
            d = dm.detach()
            if d.is_cuda:
                vj, vk = plan.get_jk_device(d.contiguous(), hermi=1)
            else:
                vj, vk = plan.get_jk(d.numpy(), hermi=1)
                vj, vk = torch.from_numpy(vj), torch.from_numpy(vk)
            veff = vj - 0.5 * vk
            e2 = 0.5 * torch.sum(d * veff)
            ctx.plan = plan
            ctx.env = env2
            ctx.save_for_backward(d, veff)
            return e2.to(coords.dtype).to(coords.device)

        @staticmethod
        def backward(ctx, grad_out):
            d, veff = ctx.saved_tensors
            g_coords = g_dm = None
            if ctx.needs_input_grad[0]:
                # the shared plan may have moved to another geometry since
                # this forward pass (another forward ran in between)
                if not numpy.array_equal(ctx.plan.env, ctx.env):
                    ctx.plan.update_coords(ctx.env)
                if d.is_cuda:
                    g = grad_2e_fused(ctx.plan, d.contiguous())
                else:
                    g = torch.from_numpy(grad_2e_fused(ctx.plan, d.numpy()))
                g_coords = (grad_out.to(g.device) * g).to(grad_out.device)
            if ctx.needs_input_grad[1]:
                g_dm = grad_out.to(veff.device) * veff
            return g_coords, g_dm, None, None, None, None

    class RHFEnergy(torch.autograd.Function):
        """E(R) = tr(D h(R)) + 1/2 tr(D J[D]) - 1/4 tr(D K[D]) + E_nuc(R) for a
        symmetric AO density D at nuclear coordinates R (Bohr, (natm, 3)),
        with the gradient of the SCF energy: the backward pass is the
        derivative of the Lagrangian E - tr(W (S(R) - S)) at fixed D and the
        energy-weighted density W, i.e. grad_elec + grad_nuc
        (pyscf/grad/rhf.py:33-76, 86-107) when D and W are the converged ones
        (W = 2 C_occ e_occ C_occ^T, or 1/2 D F D).  Everything runs on the GPU:
        int1e and J/K forward, b200jk_grad_int1e + b200jk_grad_contract
        backward.  Usage:
            E = RHFEnergy.apply(coords, dm, dme, atm, bas, env, cart)
        """

        @staticmethod
        def forward(ctx, coords, dm, dme, atm, bas, env, cart=False):
            c = coords.detach().cpu().numpy().astype(numpy.double)
            env2 = _env_with_coords(atm, env, c)
            plan = _ad_plan(atm, bas, env2, cart, dm.device.index if dm.is_cuda else 0)
            d = dm.detach().cpu().numpy()
            S, H = plan.int1e()
            vj, vk = plan.get_jk(d, hermi=1)
            e = float(numpy.sum(d * H) + 0.5 * numpy.sum(d * (vj - 0.5 * vk)) + _e_nuc(atm, c))
            ctx.plan = plan
            ctx.env = env2
            ctx.coords = c
            ctx.atm = atm
            ctx.d = d
            ctx.w = dme.detach().cpu().numpy()
            return torch.tensor(e, dtype=coords.dtype, device=coords.device)

        @staticmethod
        def backward(ctx, grad_out):
            g_coords = None
            if ctx.needs_input_grad[0]:
                if not numpy.array_equal(ctx.plan.env, ctx.env):
                    ctx.plan.update_coords(ctx.env)
                g = (ctx.plan.grad_int1e(ctx.d, ctx.w) + grad_2e_fused(ctx.plan, ctx.d) +
                     _grad_nuc(ctx.atm, ctx.coords))
                g_coords = grad_out * torch.from_numpy(g).to(grad_out.device, grad_out.dtype)
            return g_coords, None, None, None, None, None, None

    return TwoElectronEnergy, RHFEnergy


def _e_nuc(atm, coords):
    z = numpy.asarray(atm)[:, 0].astype(float)
    e = 0.0
    for a in range(len(z)):
        for b in range(a):
            e += z[a] * z[b] / numpy.linalg.norm(coords[a] - coords[b])
    return e


def _grad_nuc(atm, coords):
    """grad_nuc (pyscf/grad/rhf.py:86-107) for point charges."""
    z = numpy.asarray(atm)[:, 0].astype(float)
    dr = coords[:, None, :] - coords[None]
    r = numpy.linalg.norm(dr, axis=2)
    numpy.fill_diagonal(r, numpy.inf)
    return -numpy.einsum('i,j,ijx,ij->ix', z, z, dr, 1.0 / r ** 3)


_fn = None


def two_electron_energy(coords, dm, atm, bas, env, cart=False):
    """E2(coords, dm) as a differentiable torch scalar (see TwoElectronEnergy)."""
    global _fn
    if _fn is None:
        _fn = _torch_function()
    return _fn[0].apply(coords, dm, atm, bas, env, cart)


def rhf_energy(coords, dm, dme, atm, bas, env, cart=False):
    """The RHF energy at coords for the density dm as a differentiable torch
    scalar whose gradient is the SCF energy gradient (see RHFEnergy)."""
    global _fn
    if _fn is None:
        _fn = _torch_function()
    return _fn[1].apply(coords, dm, dme, atm, bas, env, cart)
