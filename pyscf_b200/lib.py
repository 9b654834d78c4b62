"""ctypes binding of libb200jk.so (C ABI declared in include/b200jk.h).

The library is built in-tree by ``pyscf_b200.build``.  Loading fails loudly:
there is no CPU fallback for the J/K engine.
"""
import ctypes
import os
import threading

import numpy

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libb200jk.so')

B200JK_OK = 0
B200JK_EINVAL = 1
B200JK_EUNSUPPORTED = 2
B200JK_ECUDA = 3
B200JK_ENOMEM = 4
PREC_FP64 = 0
PREC_MIXED = 1
SCREEN_NRS8 = 0
SCREEN_VJ = 1
SCREEN_VK = 2

# every entry point of include/b200jk.h
EXPORTS = (
    'b200jk_version', 'b200jk_last_error', 'b200jk_device_count', 'b200jk_plan_create',
    'b200jk_plan_destroy', 'b200jk_plan_dims', 'b200jk_get_q_cond', 'b200jk_get_jk',
    'b200jk_stats', 'b200jk_hostcheck_cart_quartet', 'b200jk_class_stats', 'b200jk_set_profiling',
    'b200jk_measure_fp64_peak', 'b200jk_get_jk_noalloc', 'b200jk_set_mixed_threshold',
    'b200jk_hostcheck_cart_quartet_fp32', 'b200jk_grad_jk', 'b200jk_grad_stats', 'b200jk_get_grad_q_cond',
    'b200jk_set_shard', 'b200jk_grad_class_stats', 'b200jk_autotune', 'b200jk_get_tuning', 'b200jk_set_tuning', 'b200jk_set_tile', 'b200jk_batch_get_jk_async', 'b200jk_batch_create', 'b200jk_batch_destroy', 'b200jk_batch_get_jk', 'b200jk_batch_stats', 'b200jk_debug_fail_alloc', 'b200jk_set_prescreen', 'b200jk_grad_contract', 'b200jk_plan_update_coords', 'b200jk_set_class_thresholds', 'b200jk_get_class_thresholds', 'b200jk_autotune_mixed', 'b200jk_int1e',
    'b200jk_int2e_s8', 'b200jk_incore_jk', 'b200jk_grad_int1e',
)


class B200JKError(RuntimeError):
    def __init__(self, code, msg):
        RuntimeError.__init__(self, 'b200jk error %d: %s' % (code, msg))
        self.code = code


class Stats(ctypes.Structure):
    _fields_ = [('quartets', ctypes.c_int64), ('prim_quartets', ctypes.c_int64),
                ('shell_pairs', ctypes.c_int64), ('prim_pairs', ctypes.c_int64),
                ('flops', ctypes.c_double), ('last_build_ms', ctypes.c_double),
                ('nao', ctypes.c_int32), ('nao_cart', ctypes.c_int32),
                ('nbas', ctypes.c_int32), ('nseg', ctypes.c_int32),
                ('kernel_launches', ctypes.c_int64), ('fp32_quartets', ctypes.c_int64),
                ('fp32_prim_quartets', ctypes.c_int64)]


class ClassStat(ctypes.Structure):
    _fields_ = [('la', ctypes.c_int32), ('lb', ctypes.c_int32), ('lc', ctypes.c_int32), ('ld', ctypes.c_int32),
                ('quartets', ctypes.c_int64), ('prim_quartets', ctypes.c_int64), ('ms', ctypes.c_double),
                ('family', ctypes.c_int32), ('pad', ctypes.c_int32), ('fp32_quartets', ctypes.c_int64)]


_lib = None
_lock = threading.Lock()


def load(path=LIB_PATH):
    """Load (once) and return the library handle with typed entry points."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise B200JKError(5, 'libb200jk.so is not built (run python -m pyscf_b200.build): %s' % path)
        lib = ctypes.CDLL(path)
        vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib.b200jk_version.restype = ip
        lib.b200jk_last_error.restype = ctypes.c_char_p
        lib.b200jk_device_count.argtypes = [ctypes.POINTER(ip)]
        lib.b200jk_plan_create.argtypes = [vp, ip, vp, ip, vp, ip, ip, dp, ip, ctypes.POINTER(vp)]
        lib.b200jk_plan_destroy.argtypes = [vp]
        lib.b200jk_plan_dims.argtypes = [vp, ctypes.POINTER(ip), ctypes.POINTER(ip)]
        lib.b200jk_get_q_cond.argtypes = [vp, vp]
        lib.b200jk_get_jk.argtypes = [vp, vp, ip, ip, ip, ip, vp, vp, ip, ip, vp]
        lib.b200jk_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        lib.b200jk_hostcheck_cart_quartet.argtypes = [vp, ip, vp, ip, vp, vp, vp]
        lib.b200jk_hostcheck_cart_quartet_fp32.argtypes = [vp, ip, vp, ip, vp, vp, vp]
        lib.b200jk_class_stats.argtypes = [vp, ctypes.POINTER(ClassStat), ip, ctypes.POINTER(ip)]
        lib.b200jk_set_profiling.argtypes = [vp, ip]
        lib.b200jk_measure_fp64_peak.argtypes = [ip, ctypes.POINTER(dp)]
        lib.b200jk_get_jk_noalloc.argtypes = [vp, vp, ip, ip, ip, ip, vp, vp, vp]
        lib.b200jk_set_mixed_threshold.argtypes = [vp, dp]
        lib.b200jk_set_prescreen.argtypes = [vp, ip]
        lib.b200jk_grad_contract.argtypes = [vp, vp, vp, ip, dp, vp]
        lib.b200jk_plan_update_coords.argtypes = [vp, vp, ip]
        lib.b200jk_int1e.argtypes = [vp, vp, vp, ip, vp]
        lib.b200jk_int2e_s8.argtypes = [vp, vp, ctypes.c_longlong, ip, vp]
        lib.b200jk_grad_int1e.argtypes = [vp, vp, vp, vp, ip, vp]
        lib.b200jk_incore_jk.argtypes = [vp, ctypes.c_longlong, ip, vp, ip, ip, ip, ip, vp, vp, ip, ip, vp]
        lib.b200jk_set_class_thresholds.argtypes = [vp, vp, ip]
        lib.b200jk_get_class_thresholds.argtypes = [vp, vp, ip, ctypes.POINTER(ip)]
        lib.b200jk_autotune_mixed.argtypes = [vp, vp, ip, dp, vp, vp]
        lib.b200jk_debug_fail_alloc.argtypes = [ip]
        lib.b200jk_grad_jk.argtypes = [vp, vp, ip, ip, ip, vp, vp, ip, dp, vp]
        lib.b200jk_grad_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                          ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_int64)]
        lib.b200jk_get_grad_q_cond.argtypes = [vp, vp]
        lib.b200jk_set_shard.argtypes = [vp, ip, ip]
        lib.b200jk_grad_class_stats.argtypes = [vp, ctypes.POINTER(ClassStat), ip, ctypes.POINTER(ip)]
        lib.b200jk_autotune.argtypes = [vp, vp, ip, vp]
        lib.b200jk_get_tuning.argtypes = [vp, ip, ctypes.POINTER(ip), ip, ctypes.POINTER(ip)]
        lib.b200jk_set_tuning.argtypes = [vp, ip, ctypes.POINTER(ip), ip]
        lib.b200jk_set_tile.argtypes = [vp, ip]
        lib.b200jk_batch_create.argtypes = [vp, ip, ctypes.POINTER(vp)]
        lib.b200jk_batch_destroy.argtypes = [vp]
        lib.b200jk_batch_get_jk.argtypes = [vp, vp, ip, ip, ip, vp, vp, ip, vp]
        lib.b200jk_batch_get_jk_async.argtypes = [vp, vp, ip, ip, ip, vp, vp, ip, vp]
        lib.b200jk_batch_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                           ctypes.POINTER(dp), ctypes.POINTER(ctypes.c_int64)]
        _lib = lib
        return lib


def check(code):
    if code != B200JK_OK:
        msg = load().b200jk_last_error()
        raise B200JKError(code, msg.decode() if msg else '')


def device_count():
    n = ctypes.c_int(0)
    check(load().b200jk_device_count(ctypes.byref(n)))
    return n.value


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Plan:
    """One molecule/basis on one GPU: shell pairs, primitive pairs and q_cond.

    Mirrors what PySCF keeps in a _VHFOpt (pyscf/scf/_vhf.py:151-264)."""

    def __init__(self, atm, bas, env, cart=False, direct_scf_tol=1e-13, device=0):
        lib = load()
        self.atm = numpy.asarray(atm, dtype=numpy.int32, order='C')
        self.bas = numpy.asarray(bas, dtype=numpy.int32, order='C')
        self.env = numpy.asarray(env, dtype=numpy.double, order='C')
        self.cart = bool(cart)
        self.direct_scf_tol = float(direct_scf_tol)
        self.device = int(device)
        h = ctypes.c_void_p()
        check(lib.b200jk_plan_create(_ptr(self.atm), self.atm.shape[0], _ptr(self.bas), self.bas.shape[0],
                                     _ptr(self.env), self.env.size, int(self.cart), self.direct_scf_tol,
                                     self.device, ctypes.byref(h)))
        self._h = h
        nao, nbas = ctypes.c_int(), ctypes.c_int()
        check(lib.b200jk_plan_dims(h, ctypes.byref(nao), ctypes.byref(nbas)))
        self.nao, self.nbas = nao.value, nbas.value

    def update_coords(self, env):
        """Re-plan for a new geometry (env with new coordinates, same atoms
        and basis), keeping workspaces and tuning."""
        env = numpy.array(env, dtype=numpy.double, order='C', copy=True)
        if env.shape != self.env.shape:
            raise ValueError('env of a different molecule')
        check(load().b200jk_plan_update_coords(self._h, _ptr(env), env.size))
        self.env = env

    def close(self):
        if getattr(self, '_h', None):
            load().b200jk_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def q_cond(self):
        q = numpy.empty((self.nbas, self.nbas))
        check(load().b200jk_get_q_cond(self._h, _ptr(q)))
        return q

    def stats(self):
        s = Stats()
        check(load().b200jk_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def class_stats(self):
        n = ctypes.c_int(0)
        buf = (ClassStat * 64)()
        check(load().b200jk_class_stats(self._h, buf, 64, ctypes.byref(n)))
        return [{k: getattr(buf[i], k) for k, _ in ClassStat._fields_} for i in range(n.value)]

    def set_profiling(self, on=True):
        check(load().b200jk_set_profiling(self._h, int(bool(on))))

    def autotune(self, dm):
        """Pick the faster launch variant per quartet class on FP64 builds of
        `dm` (host array or CUDA tensor), then for the float32 pass on mixed
        builds; returns the FP64 variants."""
        try:
            import torch
            is_dev = isinstance(dm, torch.Tensor) and dm.is_cuda
        except ImportError:
            is_dev = False
        if is_dev:
            d = dm.contiguous()
            stream = torch.cuda.current_stream(d.device).cuda_stream
            check(load().b200jk_autotune(self._h, ctypes.c_void_p(d.data_ptr()), 1, ctypes.c_void_p(stream)))
        else:
            d = numpy.ascontiguousarray(dm, dtype=numpy.double)
            check(load().b200jk_autotune(self._h, _ptr(d), 0, None))
        return self.tuning()

    def set_prescreen(self, screen=SCREEN_NRS8):
        """Density part of the quartet screen of later builds: SCREEN_NRS8
        (CVHFnrs8_prescreen), SCREEN_VJ (CVHFnrs8_vj_prescreen) or SCREEN_VK
        (CVHFnrs8_vk_prescreen)."""
        check(load().b200jk_set_prescreen(self._h, int(screen)))

    def set_tile(self, tile_b):
        """Bra pairs per tile of the ket-chunk-major order (0: bra-major)."""
        check(load().b200jk_set_tile(self._h, int(tile_b)))

    def tuning(self, precision=PREC_FP64):
        """Variant per quartet class for float64 quartets, or with
        PREC_MIXED for the float32 pass of mixed builds."""
        n = ctypes.c_int(0)
        buf = (ctypes.c_int * 64)()
        check(load().b200jk_get_tuning(self._h, int(precision), buf, 64, ctypes.byref(n)))
        return list(buf[:n.value])

    def set_tuning(self, variants, precision=PREC_FP64):
        v = (ctypes.c_int * len(variants))(*[int(x) for x in variants])
        check(load().b200jk_set_tuning(self._h, int(precision), v, len(variants)))

    def set_shard(self, index, count):
        """Evaluate only bra pairs ij = index (mod count): partial J/K for one of count GPUs."""
        check(load().b200jk_set_shard(self._h, int(index), int(count)))

    def int1e(self, device=False):
        """(S, hcore): overlap and kinetic + nuclear-attraction matrices of the
        basis (host arrays, or CUDA tensors with device=True)."""
        if device:
            import torch
            dev = torch.device('cuda', self.device)
            S = torch.empty((self.nao, self.nao), dtype=torch.float64, device=dev)
            H = torch.empty_like(S)
            stream = torch.cuda.current_stream(dev).cuda_stream
            check(load().b200jk_int1e(self._h, ctypes.c_void_p(S.data_ptr()), ctypes.c_void_p(H.data_ptr()), 1,
                                      ctypes.c_void_p(stream)))
            return S, H
        S = numpy.empty((self.nao, self.nao))
        H = numpy.empty((self.nao, self.nao))
        check(load().b200jk_int1e(self._h, _ptr(S), _ptr(H), 0, None))
        return S, H

    def grad_int1e(self, dm, dme):
        """One-electron part of the RHF nuclear gradient (natm, 3): the hcore
        and overlap lines of grad_elec for the density dm and the
        energy-weighted density dme (host arrays)."""
        dm = numpy.ascontiguousarray(dm, dtype=numpy.double)
        dme = numpy.ascontiguousarray(dme, dtype=numpy.double)
        if dm.shape != (self.nao, self.nao) or dme.shape != (self.nao, self.nao):
            raise RuntimeError('dm and dme must be (nao, nao) = (%d, %d)' % (self.nao, self.nao))
        de = numpy.empty((self.atm.shape[0], 3))
        check(load().b200jk_grad_int1e(self._h, _ptr(dm), _ptr(dme), _ptr(de), 0, None))
        return de

    def int2e_s8(self, device=True):
        """The s8-packed ERI tensor of the basis (mol.intor('int2e',
        aosym='s8')): a CUDA tensor of nao_pair (nao_pair + 1) / 2 doubles,
        or a host array with device=False."""
        npair = self.nao * (self.nao + 1) // 2
        n = npair * (npair + 1) // 2
        if device:
            import torch
            dev = torch.device('cuda', self.device)
            eri = torch.empty(n, dtype=torch.float64, device=dev)
            stream = torch.cuda.current_stream(dev).cuda_stream
            check(load().b200jk_int2e_s8(self._h, ctypes.c_void_p(eri.data_ptr()), n, 1, ctypes.c_void_p(stream)))
            return eri
        eri = numpy.empty(n)
        check(load().b200jk_int2e_s8(self._h, _ptr(eri), n, 0, None))
        return eri

    def class_thresholds(self):
        """The float32 threshold of every quartet class (55) in mixed builds."""
        out = numpy.zeros(64)
        n = ctypes.c_int(0)
        check(load().b200jk_get_class_thresholds(self._h, _ptr(out), 64, ctypes.byref(n)))
        return out[:n.value].copy()

    def set_class_thresholds(self, tau=None):
        """Per-class float32 thresholds (55 values), or None for the single one."""
        if tau is None:
            check(load().b200jk_set_class_thresholds(self._h, None, 0))
            return
        t = numpy.ascontiguousarray(tau, dtype=numpy.double)
        check(load().b200jk_set_class_thresholds(self._h, _ptr(t), t.size))

    def autotune_mixed(self, dm, budget=1e-7):
        """Pick per-class float32 thresholds for dm within an E2 error budget
        (Eh); returns {'tau', 'dE2', 'max_dJ', 'max_dK'} of the accepted build."""
        res = numpy.zeros(4)
        try:
            import torch
            is_dev = isinstance(dm, torch.Tensor) and dm.is_cuda
        except ImportError:
            is_dev = False
        if is_dev:
            d = dm.contiguous()
            stream = torch.cuda.current_stream(d.device).cuda_stream
            check(load().b200jk_autotune_mixed(self._h, ctypes.c_void_p(d.data_ptr()), 1, float(budget), _ptr(res),
                                               ctypes.c_void_p(stream)))
        else:
            d = numpy.ascontiguousarray(dm, dtype=numpy.double)
            check(load().b200jk_autotune_mixed(self._h, _ptr(d), 0, float(budget), _ptr(res), None))
        return {'tau': res[0], 'dE2': res[1], 'max_dJ': res[2], 'max_dK': res[3]}

    def set_mixed_threshold(self, tau):
        """tau of precision=PREC_MIXED: quartets with q_ij q_kl max|D| < tau run in float32."""
        check(load().b200jk_set_mixed_threshold(self._h, float(tau)))

    def get_jk(self, dms, hermi=1, with_j=True, with_k=True, out_j=None, out_k=None,
               precision=PREC_FP64, stream=None):
        """J/K of host densities (n_dm, nao, nao) -> host arrays."""
        dms = numpy.asarray(dms, dtype=numpy.double, order='C')
        shape = dms.shape
        nao = shape[-1]
        if nao != self.nao or shape[-2] != nao:
            raise ValueError('density shape %s does not match nao=%d' % (shape, self.nao))
        dms = dms.reshape(-1, nao, nao)
        n_dm = dms.shape[0]
        vj = vk = None
        if with_j:
            vj = out_j if out_j is not None else numpy.empty((n_dm, nao, nao))
        if with_k:
            vk = out_k if out_k is not None else numpy.empty((n_dm, nao, nao))
        check(load().b200jk_get_jk(self._h, _ptr(dms), n_dm, int(hermi), int(bool(with_j)), int(bool(with_k)),
                                   _ptr(vj) if with_j else None, _ptr(vk) if with_k else None,
                                   0, int(precision), stream))
        if with_j:
            vj = vj.reshape(shape)
        if with_k:
            vk = vk.reshape(shape)
        return vj, vk

    def get_jk_device(self, dms, hermi=1, with_j=True, with_k=True, precision=PREC_FP64):
        """J/K of CUDA torch tensors on the plan's device -> CUDA tensors."""
        import torch
        if not (isinstance(dms, torch.Tensor) and dms.is_cuda and dms.dtype == torch.float64):
            raise TypeError('dms must be a float64 CUDA tensor')
        if dms.device.index != self.device:
            raise ValueError('dms is on cuda:%s, plan is on cuda:%d' % (dms.device.index, self.device))
        shape = dms.shape
        nao = shape[-1]
        d = dms.reshape(-1, nao, nao).contiguous()
        n_dm = d.shape[0]
        vj = torch.empty_like(d) if with_j else None
        vk = torch.empty_like(d) if with_k else None
        stream = torch.cuda.current_stream(d.device).cuda_stream
        check(load().b200jk_get_jk(self._h, ctypes.c_void_p(d.data_ptr()), n_dm, int(hermi),
                                   int(bool(with_j)), int(bool(with_k)),
                                   ctypes.c_void_p(vj.data_ptr()) if with_j else None,
                                   ctypes.c_void_p(vk.data_ptr()) if with_k else None,
                                   1, int(precision), ctypes.c_void_p(stream)))
        return (vj.reshape(shape) if with_j else None), (vk.reshape(shape) if with_k else None)

    def grad_jk(self, dms, with_j=True, with_k=True, direct_scf_tol=1e-14):
        """pyscf.grad.rhf.get_jk of host densities: (vj, vk) with shape
        (3, nao, nao) per density (leading n_dm axis kept if given)."""
        dms = numpy.asarray(dms, dtype=numpy.double, order='C')
        nao = dms.shape[-1]
        if nao != self.nao or dms.shape[-2] != nao:
            raise ValueError('density shape %s does not match nao=%d' % (dms.shape, self.nao))
        d = dms.reshape(-1, nao, nao)
        n_dm = d.shape[0]
        vj = numpy.empty((n_dm, 3, nao, nao)) if with_j else None
        vk = numpy.empty((n_dm, 3, nao, nao)) if with_k else None
        check(load().b200jk_grad_jk(self._h, _ptr(d), n_dm, int(bool(with_j)), int(bool(with_k)),
                                    _ptr(vj) if with_j else None, _ptr(vk) if with_k else None,
                                    0, float(direct_scf_tol), None))
        shape = dms.shape[:-2] + (3, nao, nao)
        return (vj.reshape(shape) if with_j else None), (vk.reshape(shape) if with_k else None)

    def grad_jk_device(self, dms, with_j=True, with_k=True, direct_scf_tol=1e-14):
        """grad_jk of a float64 CUDA tensor (..., nao, nao) -> CUDA tensors (..., 3, nao, nao)."""
        import torch
        if not (isinstance(dms, torch.Tensor) and dms.is_cuda and dms.dtype == torch.float64):
            raise TypeError('dms must be a float64 CUDA tensor')
        nao = dms.shape[-1]
        d = dms.reshape(-1, nao, nao).contiguous()
        n_dm = d.shape[0]
        vj = torch.empty((n_dm, 3, nao, nao), dtype=torch.float64, device=d.device) if with_j else None
        vk = torch.empty((n_dm, 3, nao, nao), dtype=torch.float64, device=d.device) if with_k else None
        stream = torch.cuda.current_stream(d.device).cuda_stream
        check(load().b200jk_grad_jk(self._h, ctypes.c_void_p(d.data_ptr()), n_dm, int(bool(with_j)),
                                    int(bool(with_k)), ctypes.c_void_p(vj.data_ptr()) if with_j else None,
                                    ctypes.c_void_p(vk.data_ptr()) if with_k else None, 1,
                                    float(direct_scf_tol), ctypes.c_void_p(stream)))
        shape = tuple(dms.shape[:-2]) + (3, nao, nao)
        return (vj.reshape(shape) if with_j else None), (vk.reshape(shape) if with_k else None)

    def grad_contract(self, dm, direct_scf_tol=1e-14):
        """Two-electron part of the RHF nuclear gradient, (natm, 3), for one
        symmetric density (host array or float64 CUDA tensor), contracted on
        the GPU without forming vj/vk (b200jk_grad_contract)."""
        natm = self.atm.shape[0]
        try:
            import torch
            is_dev = isinstance(dm, torch.Tensor) and dm.is_cuda
        except ImportError:
            is_dev = False
        if is_dev:
            d = dm.contiguous()
            if tuple(d.shape) != (self.nao, self.nao) or d.dtype != torch.float64:
                raise ValueError('dm must be a float64 (nao, nao) tensor')
            de = torch.empty((natm, 3), dtype=torch.float64, device=d.device)
            stream = torch.cuda.current_stream(d.device).cuda_stream
            check(load().b200jk_grad_contract(self._h, ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(de.data_ptr()),
                                              1, float(direct_scf_tol), ctypes.c_void_p(stream)))
            return de
        d = numpy.ascontiguousarray(dm, dtype=numpy.double)
        if d.shape != (self.nao, self.nao):
            raise ValueError('density shape %s does not match nao=%d' % (d.shape, self.nao))
        de = numpy.empty((natm, 3))
        check(load().b200jk_grad_contract(self._h, _ptr(d), _ptr(de), 0, float(direct_scf_tol), None))
        return de

    def grad_stats(self):
        q, pq, n = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        ms = ctypes.c_double(0)
        check(load().b200jk_grad_stats(self._h, ctypes.byref(q), ctypes.byref(pq), ctypes.byref(ms), ctypes.byref(n)))
        return {'quartets': q.value, 'prim_quartets': pq.value, 'last_build_ms': ms.value, 'kernel_launches': n.value}

    def grad_class_stats(self):
        n = ctypes.c_int(0)
        buf = (ClassStat * 100)()
        check(load().b200jk_grad_class_stats(self._h, buf, 100, ctypes.byref(n)))
        return [{k: getattr(buf[i], k) for k, _ in ClassStat._fields_} for i in range(n.value)]

    @property
    def grad_q_cond(self):
        """(2, nbas, nbas): derivative Schwarz bound and q_cond of the gradient screen."""
        nbas = self.nbas
        q = numpy.empty((2, nbas, nbas))
        check(load().b200jk_get_grad_q_cond(self._h, _ptr(q)))
        return q


class Batch:
    """J/K of many molecules (one Plan each, same GPU) in one launch per quartet class."""

    def __init__(self, plans):
        self.plans = list(plans)
        arr = (ctypes.c_void_p * len(self.plans))(*[p._h for p in self.plans])
        h = ctypes.c_void_p()
        check(load().b200jk_batch_create(arr, len(self.plans), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, '_h', None)
        if h and _lib is not None:
            _lib.b200jk_batch_destroy(h)
            self._h = None

    def get_jk_device(self, dms, hermi=1, with_j=True, with_k=True, precision=PREC_FP64):
        """dms: list of float64 CUDA tensors (nao_m, nao_m) -> lists vj, vk."""
        import torch
        if len(dms) != len(self.plans):
            raise ValueError('one density per molecule of the batch')
        ds = [d.contiguous() for d in dms]
        for d, p in zip(ds, self.plans):
            if not (d.is_cuda and d.dtype == torch.float64 and tuple(d.shape) == (p.nao, p.nao)):
                raise ValueError('density must be a float64 CUDA tensor (nao, nao) of its molecule')
        vj = [torch.empty_like(d) for d in ds] if with_j else None
        vk = [torch.empty_like(d) for d in ds] if with_k else None
        P = ctypes.c_void_p * len(ds)
        pd = P(*[d.data_ptr() for d in ds])
        pj = P(*[t.data_ptr() for t in vj]) if with_j else None
        pk = P(*[t.data_ptr() for t in vk]) if with_k else None
        stream = torch.cuda.current_stream(ds[0].device).cuda_stream
        check(load().b200jk_batch_get_jk(self._h, pd, int(hermi), int(bool(with_j)), int(bool(with_k)),
                                         pj, pk, int(precision), ctypes.c_void_p(stream)))
        return vj, vk

    def get_jk_device_async(self, dms, vj, vk, hermi=1, precision=PREC_FP64):
        """The launches of one batched build into the caller's tensors, on the
        current stream, with no allocation or synchronisation (capturable in a
        torch.cuda.CUDAGraph after one get_jk_device call)."""
        import torch
        P = ctypes.c_void_p * len(dms)
        pd = P(*[d.data_ptr() for d in dms])
        pj = P(*[t.data_ptr() for t in vj])
        pk = P(*[t.data_ptr() for t in vk])
        stream = torch.cuda.current_stream(dms[0].device).cuda_stream
        check(load().b200jk_batch_get_jk_async(self._h, pd, int(hermi), 1, 1, pj, pk, int(precision),
                                               ctypes.c_void_p(stream)))

    def stats(self):
        q, q32, n = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
        ms = ctypes.c_double(0)
        check(load().b200jk_batch_stats(self._h, ctypes.byref(q), ctypes.byref(q32), ctypes.byref(ms), ctypes.byref(n)))
        return {'quartets': q.value, 'fp32_quartets': q32.value, 'last_build_ms': ms.value, 'kernel_launches': n.value}


def measure_fp64_peak(device=0):
    """FP64 FMA throughput of the device in TFLOP/s (register-resident loop)."""
    t = ctypes.c_double(0)
    check(load().b200jk_measure_fp64_peak(int(device), ctypes.byref(t)))
    return t.value


def hostcheck_cart_quartet(atm, bas, env, shls, fp32=False):
    """Host replay of the kernels' integral arithmetic for one quartet of
    segmented shells; returns the Cartesian block [a][b][c][d].  fp32=True
    replays the float32 pass of mixed precision."""
    lib = load()
    atm = numpy.asarray(atm, dtype=numpy.int32, order='C')
    bas = numpy.asarray(bas, dtype=numpy.int32, order='C')
    env = numpy.asarray(env, dtype=numpy.double, order='C')
    shls = numpy.asarray(shls, dtype=numpy.int32)
    nc = [(int(bas[s, 1]) + 1) * (int(bas[s, 1]) + 2) // 2 for s in shls]
    out = numpy.zeros(nc)
    fn = lib.b200jk_hostcheck_cart_quartet_fp32 if fp32 else lib.b200jk_hostcheck_cart_quartet
    check(fn(_ptr(atm), atm.shape[0], _ptr(bas), bas.shape[0], _ptr(env), _ptr(shls), _ptr(out)))
    return out
