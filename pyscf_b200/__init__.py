"""pyscf_b200 — a B200-native direct-SCF Coulomb/exchange (J/K) engine.

A drop-in for PySCF's direct J/K path: ``pyscf_b200._vhf.direct`` has the
signature of ``pyscf.scf._vhf.direct`` and ``pyscf_b200.scf.get_jk`` that of
``pyscf.scf.hf.get_jk``; ``pyscf_b200.patch_pyscf()`` routes an unmodified
``scf.RHF(mol).run()`` through the GPU.  The arithmetic runs in hand-written
sm_100a CUDA kernels behind a C ABI (include/b200jk.h, libb200jk.so).
"""
from . import lib
from . import _vhf
from .scf import get_jk, patch_pyscf, unpatch_pyscf
from ._vhf import direct, VHFOpt

__all__ = ['lib', 'direct', 'VHFOpt', 'get_jk', 'patch_pyscf', 'unpatch_pyscf']
