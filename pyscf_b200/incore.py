"""The in-core J/K path: a stored two-electron integral tensor on the GPU.

Drop-ins for the reference's
  * ``_vhf.incore(eri, dms, hermi=0, with_j=True, with_k=True)``
    (pyscf/scf/_vhf.py:318-401): ``eri`` the s8-packed vector or the s4
    (nao_pair, nao_pair) matrix, as a host array (copied to the GPU on every
    call) or as a CUDA tensor; J = einsum('ijkl,ji->kl'), K =
    einsum('ijkl,jk->il'), then hermi_triu as the reference;
  * ``mol.intor('int2e', aosym='s8')`` (GTO2e_cart_or_sph,
    pyscf/lib/vhf/fill_nr_s8.c:110-138): ``int2e_s8(mol)`` fills the tensor on
    the GPU (a CUDA tensor, or a host array with device=False);
  * the in-core branch of ``RHF.get_jk`` (pyscf/scf/hf.py:2400-2414) under
    ``pyscf_b200.scf.patch_pyscf(incore=True)``: the tensor is filled once on
    the GPU and kept there (``mf._eri`` stays None), and every build is
    contracted from it (``rhf_get_jk`` below).
Errors follow the reference: a tensor whose size fits neither symmetry
raises RuntimeError ('Array shape not consistent').
"""
import ctypes

import numpy

from . import lib, _vhf


def _is_cuda(a):
    try:
        import torch
    except ImportError:
        return False
    return isinstance(a, torch.Tensor) and a.is_cuda


def int2e_s8(mol, device=True):
    """s8 ERI tensor of ``mol`` (PySCF Mole or an object with _atm, _bas,
    _env, cart), env[PTR_RANGE_OMEGA] selecting the operator as in the
    reference."""
    plan = _vhf.make_plan(mol._atm, mol._bas, mol._env, getattr(mol, 'cart', False), 0.0)
    return plan.int2e_s8(device=device)


def incore(eri, dms, hermi=0, with_j=True, with_k=True):
    """J and K of one or several densities from a stored tensor
    (pyscf/scf/_vhf.py:318-401).  Host arrays in, host arrays out; a CUDA
    tensor ``eri`` keeps the work on its GPU (``dms`` may then be a host
    array or a CUDA tensor; the outputs follow ``dms``)."""
    if not with_j and not with_k:
        return None, None
    l = lib.load()
    if _is_cuda(eri):
        import torch
        dev = eri.device
        if eri.dtype != torch.float64:
            raise RuntimeError('eri must be float64')
        dms_cuda = _is_cuda(dms)
        d = dms.to(device=dev, dtype=torch.float64) if dms_cuda else \
            torch.as_tensor(numpy.asarray(dms, dtype=numpy.double), device=dev)
        shape = tuple(d.shape)
        nao = shape[-1]
        d = d.reshape(-1, nao, nao).contiguous()
        e = eri.contiguous().reshape(-1)
        vj = torch.empty_like(d) if with_j else None
        vk = torch.empty_like(d) if with_k else None
        stream = torch.cuda.current_stream(dev).cuda_stream
        lib.check(l.b200jk_incore_jk(ctypes.c_void_p(e.data_ptr()), e.numel(), nao, ctypes.c_void_p(d.data_ptr()),
                                     d.shape[0], int(hermi), int(bool(with_j)), int(bool(with_k)),
                                     ctypes.c_void_p(vj.data_ptr()) if with_j else None,
                                     ctypes.c_void_p(vk.data_ptr()) if with_k else None, 1, dev.index or 0,
                                     ctypes.c_void_p(stream)))
        if with_j:
            vj = vj.reshape(shape)
        if with_k:
            vk = vk.reshape(shape)
        if not dms_cuda:
            vj = vj.cpu().numpy() if with_j else None
            vk = vk.cpu().numpy() if with_k else None
        return vj, vk
    eri = numpy.asarray(eri)
    if eri.dtype != numpy.double:
        raise RuntimeError('eri must be float64')
    eri = numpy.ascontiguousarray(eri)
    dms = numpy.asarray(dms, order='C', dtype=numpy.double)
    shape = dms.shape
    nao = shape[-1]
    dms = dms.reshape(-1, nao, nao)
    vj = numpy.empty_like(dms) if with_j else None
    vk = numpy.empty_like(dms) if with_k else None
    lib.check(l.b200jk_incore_jk(lib._ptr(eri), eri.size, nao, lib._ptr(dms), dms.shape[0], int(hermi),
                                 int(bool(with_j)), int(bool(with_k)), lib._ptr(vj) if with_j else None,
                                 lib._ptr(vk) if with_k else None, 0, 0, None))
    return (vj.reshape(shape) if with_j else None), (vk.reshape(shape) if with_k else None)


# GPU memory the stored tensor of the in-core SCF path may take
INCORE_FRACTION = 0.4


def incore_fits(nao, device=0):
    """Whether the s8 tensor of nao functions fits the in-core budget of the
    GPU (a fraction of its memory) and the contraction's shared memory."""
    import torch
    npair = nao * (nao + 1) // 2
    need = 8 * npair * (npair + 1) // 2
    total = torch.cuda.get_device_properties(device).total_memory
    return nao <= 880 and need <= INCORE_FRACTION * total


def _mol_key(mol):
    return (numpy.asarray(mol._atm).tobytes(), numpy.asarray(mol._bas).tobytes(), numpy.asarray(mol._env).tobytes(),
            bool(getattr(mol, 'cart', False)))


def device_eri(mf, mol):
    """The GPU tensor of ``mol`` kept on the SCF object (filled on first use
    and again when the molecule changes)."""
    key = _mol_key(mol)
    held = getattr(mf, '_b200_eri', None)
    if held is None or held[0] != key:
        mf._b200_eri = None
        mf._b200_eri = (key, int2e_s8(mol, device=True))
    return mf._b200_eri[1]


def rhf_get_jk(mf, mol=None, dm=None, hermi=1, with_j=True, with_k=True, omega=None):
    """RHF.get_jk (pyscf/scf/hf.py:2400-2414) with the in-core branch on the
    GPU: when the reference would go in core (no omega; a stored mf._eri,
    mol.incore_anyway, or a tensor that fits) the build contracts the GPU
    tensor (a host mf._eri set by the caller is contracted as it is);
    otherwise the direct build."""
    if mol is None:
        mol = mf.mol
    if dm is None:
        dm = mf.make_rdm1()
    from pyscf.scf import hf as ref_hf
    if not omega and mf._eri is not None:
        return incore(mf._eri, dm, hermi, with_j, with_k)
    if not omega and (getattr(mol, 'incore_anyway', False) or incore_fits(mol.nao_nr())):
        return incore(device_eri(mf, mol), dm, hermi, with_j, with_k)
    return ref_hf.SCF.get_jk(mf, mol, dm, hermi, with_j, with_k, omega)
