"""PySCF-facing J/K API and the plug-in switch.

``get_jk(mol, dm, hermi, vhfopt, with_j, with_k, omega)`` mirrors
pyscf.scf.hf.get_jk (pyscf/scf/hf.py:948-1022), including the split of a
complex density into real and imaginary parts and the range-separated
operators of omega > 0 (erf) and omega < 0 (erfc).

``patch_pyscf()`` makes an unmodified ``scf.RHF(mol).run()`` use the GPU
engine for every J/K build:
  * ``pyscf.scf._vhf.direct`` is rebound (hf.get_jk looks it up at call time,
    pyscf/scf/hf.py:1007);
  * ``SCF.init_direct_scf`` returns a pyscf_b200 VHFOpt, so the Schwarz
    conditioner is computed on the GPU too (pyscf/scf/hf.py:2045-2054);
  * ``SCF._is_mem_enough`` returns False so RHF.get_jk takes the direct branch
    instead of building the in-core ERI tensor (pyscf/scf/hf.py:2400-2414,
    2150-2152), as ``mf.max_memory = 0`` does in the reference tests.
``patch_pyscf(incore=True)`` instead keeps the reference's in-core choice
for small molecules and runs it on the GPU: ``RHF.get_jk`` fills the s8
tensor once on the GPU and contracts every build from it, and
``pyscf.scf._vhf.incore`` is rebound (dot_eri_dm looks it up at call time,
pyscf/scf/hf.py:887-935), see pyscf_b200/incore.py.
``unpatch_pyscf()`` restores the originals.
"""
import numpy

from . import _vhf

_saved = {}


def get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True, omega=None):
    dm = numpy.asarray(dm, order='C')
    dm_shape = dm.shape
    dm_dtype = dm.dtype
    nao = dm_shape[-1]
    if dm_dtype == numpy.complex128:
        dm = numpy.vstack((dm.real, dm.imag)).reshape(-1, nao, nao)
        hermi = 0
    env = mol._env
    if omega:
        # mol.with_range_coulomb(omega) (pyscf/scf/hf.py:1006): the operator is
        # selected by env[PTR_RANGE_OMEGA]
        env = _vhf._with_omega(env, omega)
    vj, vk = _vhf.direct(dm, mol._atm, mol._bas, env, vhfopt, hermi, mol.cart, with_j, with_k)
    if dm_dtype == numpy.complex128:
        if with_j:
            vj = vj.reshape((2,) + dm_shape)
            vj = vj[0] + vj[1] * 1j
        if with_k:
            vk = vk.reshape((2,) + dm_shape)
            vk = vk[0] + vk[1] * 1j
    else:
        if with_j:
            vj = vj.reshape(dm_shape)
        if with_k:
            vk = vk.reshape(dm_shape)
    return vj, vk


def _init_direct_scf(self, mol=None):
    if mol is None:
        mol = self.mol
    return _vhf.VHFOpt(mol, 'int2e', 'CVHFnrs8_prescreen', 'CVHFnr_int2e_q_cond',
                       'CVHFnr_dm_cond', self.direct_scf_tol)


def _no_incore(self):
    return False


def patch_pyscf(incore=False):
    """Route PySCF's J/K through the GPU engine (idempotent): direct builds
    always; with incore=True the in-core branch of RHF.get_jk on the GPU."""
    import pyscf.scf._vhf as ref_vhf
    import pyscf.scf.hf as ref_hf
    if _saved:
        return
    _saved['direct'] = ref_vhf.direct
    _saved['init_direct_scf'] = ref_hf.SCF.init_direct_scf
    _saved['_is_mem_enough'] = ref_hf.SCF._is_mem_enough
    ref_vhf.direct = _vhf.direct
    ref_hf.SCF.init_direct_scf = _init_direct_scf
    ref_hf.SCF._is_mem_enough = _no_incore
    if incore:
        from . import incore as gpu_incore
        _saved['incore'] = ref_vhf.incore
        _saved['rhf_get_jk'] = ref_hf.RHF.get_jk
        ref_vhf.incore = gpu_incore.incore
        ref_hf.RHF.get_jk = gpu_incore.rhf_get_jk


def unpatch_pyscf():
    import pyscf.scf._vhf as ref_vhf
    import pyscf.scf.hf as ref_hf
    if not _saved:
        return
    ref_vhf.direct = _saved.pop('direct')
    ref_hf.SCF.init_direct_scf = _saved.pop('init_direct_scf')
    ref_hf.SCF._is_mem_enough = _saved.pop('_is_mem_enough')
    if 'incore' in _saved:
        ref_vhf.incore = _saved.pop('incore')
        ref_hf.RHF.get_jk = _saved.pop('rhf_get_jk')
