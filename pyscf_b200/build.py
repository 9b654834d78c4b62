"""Build the CUDA engine in-tree: pyscf_b200/libb200jk.so for sm_100a.

    python -m pyscf_b200.build          (or python pyscf_b200/build.py)

The library is a plain shared object with a C ABI (include/b200jk.h); the
Python package loads it with ctypes.  It is built next to the sources so it
travels with the repository snapshot.  The per-class kernels are split into
one translation unit per quartet class (jk_classes.cu compiled 55 times), the
gradient kernels and the s8 integral fill into one per bra class
(grad_classes.cu and fill_classes.cu, 10 times each), all compiled in
parallel.
"""
import os
import subprocess
import sys
import shutil
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
OBJ = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libb200jk.so')
HEADERS = ['rys_math.cuh', 'jk_kernels.cuh', 'jk_launch.h', 'rys_table.inc', 'rys_table_f.inc',
           'grad_kernels.cuh', 'grad_launch.h', 'int1e_kernels.cuh', 'fill_kernels.cuh', 'fill_launch.h',
           'incore_launch.h']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
PAIR_CLASSES = [(la, lb) for la in range(4) for lb in range(la + 1)]
QUARTET_CLASSES = [(la, lb, lc, ld) for x, (la, lb) in enumerate(PAIR_CLASSES)
                   for y, (lc, ld) in enumerate(PAIR_CLASSES) if y <= x]


def nvcc_path():
    for p in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if p and os.path.exists(p):
            return p
    raise RuntimeError('nvcc not found')


def _deps():
    files = [os.path.join(CSRC, f) for f in
             ['b200jk.cu', 'jk_classes.cu', 'jk_qcond.cu', 'grad_classes.cu', 'fill_classes.cu', 'incore.cu',
              'hostcheck.cpp'] + HEADERS]
    files.append(os.path.join(ROOT, 'include', 'b200jk.h'))
    files.append(os.path.abspath(__file__))
    return files


def up_to_date(target=LIB):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(f) <= t for f in _deps())


# headers each translation unit includes (directly or through another header)
_RYS = ['rys_math.cuh', 'rys_table.inc', 'rys_table_f.inc']
_JK = _RYS + ['jk_kernels.cuh', 'jk_launch.h']
_GRAD = _JK + ['grad_kernels.cuh', 'grad_launch.h']
_FILL = _JK + ['fill_kernels.cuh', 'fill_launch.h']
UNIT_DEPS = {
    'b200jk.cu': _GRAD + _FILL + ['int1e_kernels.cuh', 'incore_launch.h', '../../include/b200jk.h'],
    'jk_qcond.cu': _JK,
    'jk_classes.cu': _JK,
    'grad_classes.cu': _GRAD,
    'fill_classes.cu': _FILL,
    'incore.cu': ['incore_launch.h'],
    'hostcheck.cpp': _RYS + ['../../include/b200jk.h'],
}


def _stale(obj, src, flags_file):
    """Whether obj must be rebuilt: missing, older than its source or one of
    its headers, or built with other flags (the command line, recorded next
    to the object, stands for everything this script decides about it)."""
    if not os.path.exists(obj) or not os.path.exists(flags_file):
        return True
    t = os.path.getmtime(obj)
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in UNIT_DEPS[src]]
    return any(os.path.getmtime(d) > t for d in deps)


# blocks per SM the register-family kernels of a quartet class are compiled
# for (absent: 0, the compiler's own allocation): 4 caps a thread at 128
# registers, 3 at 168.  Each entry is the faster build of the class on the
# FP64 build of (H2O)64/cc-pVTZ (class CUDA events, builds compiled with 0,
# 3 and 4 for every class, launch variants 0 and 2 each, with the part
# counts below): a few spills buy 12 or 16 resident warps instead of 8.
# B2_THREAD_MINB=<n> (every class) or "la lb lc ld:n,..." in the environment
# overrides it.
THREAD_MINB = {
    (1, 0, 0, 0): 4, (1, 1, 0, 0): 4, (2, 0, 0, 0): 4, (2, 1, 0, 0): 4,
    (3, 0, 1, 0): 3, (2, 2, 0, 0): 3, (3, 1, 0, 0): 3,
}


# parts of the register family per quartet class where the build overrides
# the register budget's choice (thread_parts<> in jk_kernels.cuh; a part
# re-runs the primitive loop for its share of the bra components): fewer
# parts than the budget allows, measured faster on the FP64 build of
# (H2O)64/cc-pVTZ ((31|10) 397 -> 204 ms with 2 parts instead of 5, (21|10)
# 595 -> 466 ms with 1 instead of 2): re-running the roots and 2D integrals
# costs more than the spills of the larger blocks.
# B2_THREAD_PARTS="la lb lc ld:n,..." in the environment replaces it.
THREAD_PARTS = {
    (3, 1, 1, 0): 2, (3, 0, 1, 1): 2, (3, 0, 3, 0): 2, (3, 3, 0, 0): 2,
    (2, 1, 1, 0): 1, (2, 0, 1, 1): 1, (3, 0, 2, 0): 1, (3, 2, 0, 0): 1,
}


# blocks per SM of the shared-memory family's float64 kernels where the
# build overrides warp_min_blocks<> (jk_kernels.cuh: 4 where the groups'
# shared memory admits 4 blocks, else 0); B2_WARP_MINB="la lb lc ld:n,..."
# in the environment replaces it.  Empty: without the cap of 4 (128
# registers) the tuned half-width (21|20) and (22|10) kernels took 852 and
# 359 ms instead of 720 and 327 ms on the FP64 build of (H2O)64/cc-pVTZ.
WARP_MINB = {}


def _class_table(text):
    """'la lb lc ld:n,...' -> {(la, lb, lc, ld): n}"""
    table = {}
    for item in text.split(','):
        c, n = item.split(':')
        table[tuple(int(x) for x in c.split())] = int(n)
    return table


def _thread_parts(cls):
    env = os.environ.get('B2_THREAD_PARTS')
    table = _class_table(env) if env else THREAD_PARTS
    return table.get(cls)


def _warp_minb(cls):
    env = os.environ.get('B2_WARP_MINB')
    table = _class_table(env) if env else WARP_MINB
    return table.get(cls)


def _thread_minb(cls):
    env = os.environ.get('B2_THREAD_MINB')
    if env:
        # one value for every class, or a per-class table
        return _class_table(env).get(cls, 0) if ':' in env else int(env)
    return THREAD_MINB.get(cls, 0)


def _units():
    nvcc = nvcc_path()
    common = [nvcc, *ARCH, '-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC',
              '-I', os.path.join(ROOT, 'include'), '-I', CSRC, '-c']
    units = []
    units.append((common + [os.path.join(CSRC, 'b200jk.cu'), '-o', os.path.join(OBJ, 'b200jk.o')],
                  os.path.join(OBJ, 'b200jk.o')))
    units.append((common + [os.path.join(CSRC, 'jk_qcond.cu'), '-o', os.path.join(OBJ, 'jk_qcond.o')],
                  os.path.join(OBJ, 'jk_qcond.o')))
    for la, lb, lc, ld in QUARTET_CLASSES:
        tag = '%d%d%d%d' % (la, lb, lc, ld)
        o = os.path.join(OBJ, 'jk_%s.o' % tag)
        units.append((common + ['-DB2_BRA_LA=%d' % la, '-DB2_BRA_LB=%d' % lb, '-DB2_KET_LC=%d' % lc,
                                '-DB2_KET_LD=%d' % ld, '-DB2_FN_NAME=launch_jk_%s' % tag,
                                '-DB2_NP_NAME=launch_jk_%s_np' % tag,
                                '-DB2_THREAD_MINB=%d' % _thread_minb((la, lb, lc, ld))] +
                     (['-DB2_THREAD_PARTS=%d' % _thread_parts((la, lb, lc, ld))]
                      if _thread_parts((la, lb, lc, ld)) else []) +
                     (['-DB2_WARP_MINB=%d' % _warp_minb((la, lb, lc, ld))]
                      if _warp_minb((la, lb, lc, ld)) is not None else []) +
                     [os.path.join(CSRC, 'jk_classes.cu'), '-o', o], o))
    for la, lb in PAIR_CLASSES:
        o = os.path.join(OBJ, 'grad_%d%d.o' % (la, lb))
        units.append((common + ['-DB2_BRA_LA=%d' % la, '-DB2_BRA_LB=%d' % lb,
                                os.path.join(CSRC, 'grad_classes.cu'), '-o', o], o))
    for la, lb in PAIR_CLASSES:
        o = os.path.join(OBJ, 'fill_%d%d.o' % (la, lb))
        units.append((common + ['-DB2_BRA_LA=%d' % la, '-DB2_BRA_LB=%d' % lb,
                                os.path.join(CSRC, 'fill_classes.cu'), '-o', o], o))
    o = os.path.join(OBJ, 'incore.o')
    units.append((common + [os.path.join(CSRC, 'incore.cu'), '-o', o], o))
    o = os.path.join(OBJ, 'hostcheck.o')
    units.append((['g++', '-O2', '-std=c++17', '-fPIC', '-I', os.path.join(ROOT, 'include'), '-I', CSRC,
                   '-c', os.path.join(CSRC, 'hostcheck.cpp'), '-o', o], o))
    return units


def _source_of(cmd):
    for a in cmd:
        if a.startswith(CSRC + os.sep):
            return os.path.basename(a)
    raise ValueError(cmd)


def build(force=False, verbose=False, extra=(), jobs=None):
    # every unit is checked against its own sources (an object compiled while
    # its source was being edited is older than the edit even when the library
    # was linked after it); the library is relinked when an object changed
    os.makedirs(OBJ, exist_ok=True)
    units = _units()
    if extra:
        units = [(cmd[:-3] + list(extra) + cmd[-3:] if cmd[0] != 'g++' else cmd, o) for cmd, o in units]
    # rebuild only the units whose sources, headers or flags changed
    todo = []
    for cmd, o in units:
        flags_file = o + '.cmd'
        line = ' '.join(cmd)
        same_flags = os.path.exists(flags_file) and open(flags_file).read() == line
        if force or not same_flags or _stale(o, _source_of(cmd), flags_file):
            todo.append((cmd, o))

    def run(u):
        cmd, o = u
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            with open(o + '.cmd', 'w') as fh:
                fh.write(' '.join(cmd))
        return cmd, r

    with ThreadPoolExecutor(jobs or min(12, os.cpu_count() or 4)) as ex:
        results = list(ex.map(run, todo))
    msgs = []
    for cmd, r in results:
        if r.returncode != 0:
            raise RuntimeError('compile failed: %s\n%s%s' % (' '.join(cmd), r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            msgs.append(r.stdout + r.stderr)
    objs = [o for _, o in units]
    if not todo and os.path.exists(LIB) and all(os.path.getmtime(o) <= os.path.getmtime(LIB) for o in objs):
        return LIB
    link = [nvcc_path(), *ARCH, '--shared', '-Xcompiler', '-fPIC', '-o', LIB + '.tmp'] + objs
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n' + r.stdout + r.stderr)
    os.replace(LIB + '.tmp', LIB)
    if verbose:
        print('\n'.join(msgs))
    return LIB


if __name__ == '__main__':
    extra = []
    if '--ptxas-v' in sys.argv:
        extra += ['-Xptxas', '-v']
    build(force='--force' in sys.argv or bool(extra), verbose=True, extra=extra)
    print('built', LIB)
