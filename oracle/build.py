"""Build recipe for the CPU oracle.

ORACLE / TEST INFRASTRUCTURE: builds the checker, never the product.

Two outputs:

* ``oracle/liboracle.so`` — this project's CPU restatement of the direct-SCF
  J/K path: the libcint-ABI integral library (``cint/cint_shim.c``) and the
  restated driver (``jk_direct.c``).  No reference source goes into it.

* ``oracle/_ref/`` (only where the reference tree is readable) — PySCF's own
  C drivers compiled from their sources where they lie under the reference
  checkout, linked against the integral library above because upstream
  libcint v6.1.3 is an un-vendored dependency:

    - libnp_helper  pyscf/lib/np_helper/*.c
    - libcgto       pyscf/lib/gto/{fill_int2c,fill_nr_3c,fill_r_3c,fill_int2e,
                    fill_r_4c,ft_ao,ft_ao_deriv,ft_ao_ppnl,fill_grids_int2c,
                    grid_ao_drv,nr_ecp,nr_ecp_deriv}.c
    - libcvhf       pyscf/lib/vhf/*.c except nr_sr_vhf.c (needs libcint's
                    private cint_funcs.h)
    - libao2mo      pyscf/lib/ao2mo/*.c
    - libcint       cint_shim.c plus generated stubs for every libcint symbol
                    the objects above reference but the direct-SCF path never
                    calls (each stub aborts with a message if reached).

  The libraries land in ``oracle/_ref/pyext/pyscf/lib`` so that
  ``PYSCF_EXT_PATH=oracle/_ref/pyext`` lets an unmodified ``import pyscf``
  find them (pyscf/__init__.py:43-57 and pyscf/lib/misc.py:95-107).
  gto/deriv1.c, deriv2.c and autocode/auto_eval1.c are left out: they need
  libcint's spinor transforms, which are outside this path.
"""
import os
import subprocess
import sys
import glob

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_REF = os.path.join(HERE, '_ref')


def _recorded_root():
    """The checkout an earlier build_ref() compiled from (recorded in the
    git-ignored oracle/_ref), so later runs find it without the variable."""
    p = os.path.join(OUT_REF, 'reference_root')
    return open(p).read().strip() if os.path.exists(p) else ''


# the reference checkout: PYSCF_REFERENCE_ROOT, else the one the last
# build_ref() used; without either only the restatement (liboracle.so) builds
REF_ROOT = os.environ.get('PYSCF_REFERENCE_ROOT') or _recorded_root()
REF_LIB = os.path.join(REF_ROOT, 'pyscf', 'lib')
OUT_LIBDIR = os.path.join(OUT_REF, 'pyext', 'pyscf', 'lib')
CFLAGS = ['-O2', '-fPIC', '-fopenmp', '-std=gnu99', '-w']


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('command failed: %s\n%s\n%s' % (' '.join(cmd), r.stdout, r.stderr))
    return r.stdout


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources)


def find_blas():
    """A BLAS exporting the plain Fortran symbol dgemm_ (the reference calls
    dgemm_ in np_helper/npdot.c and vhf/optimizer.c)."""
    import site
    for sp in site.getsitepackages():
        for p in glob.glob(os.path.join(sp, '*.libs', 'libopenblas*.so*')):
            try:
                syms = _run(['nm', '-D', '--defined-only', p])
            except RuntimeError:
                continue
            if ' dgemm_\n' in syms:
                return p
    return None


def build_oracle(force=False):
    """Compile oracle/liboracle.so (restated integrals + restated driver)."""
    srcs = [os.path.join(HERE, 'cint', 'cint_shim.c'), os.path.join(HERE, 'jk_direct.c'),
            os.path.join(HERE, 'cint', 'cint.h')]
    out = os.path.join(HERE, 'liboracle.so')
    if not force and _newer(out, srcs):
        return out
    _run(['gcc'] + CFLAGS + ['-shared', '-I', HERE, '-o', out, srcs[0], srcs[1], '-lm'])
    return out


REF_GROUPS = {
    'np_helper': ['np_helper/' + f for f in (
        'transpose.c', 'pack_tril.c', 'npdot.c', 'condense.c', 'omp_reduce.c',
        'np_helper.c', 'imatcopy.c', 'np_broadcast.c')],
    'cgto': ['gto/' + f for f in (
        'fill_int2c.c', 'fill_nr_3c.c', 'fill_r_3c.c', 'fill_int2e.c', 'fill_r_4c.c',
        'ft_ao.c', 'ft_ao_deriv.c', 'ft_ao_ppnl.c', 'fill_grids_int2c.c',
        'grid_ao_drv.c', 'nr_ecp.c', 'nr_ecp_deriv.c')],
    'cvhf': ['vhf/' + f for f in (
        'fill_nr_s8.c', 'nr_incore.c', 'nr_direct.c', 'optimizer.c', 'nr_direct_dot.c',
        'time_rev.c', 'r_direct_o1.c', 'rkb_screen.c', 'r_direct_dot.c',
        'rah_direct_dot.c', 'rha_direct_dot.c', 'hessian_screen.c', 'nr_sgx_direct.c')],
    'ao2mo': ['ao2mo/' + f for f in (
        'restore_eri.c', 'nr_ao2mo.c', 'nr_incore.c', 'r_ao2mo.c', 'nrr_ao2mo.c')],
}
LINK_ORDER = ['np_helper', 'cint', 'cgto', 'cvhf', 'ao2mo']
DEPS = {'np_helper': [], 'cint': [], 'cgto': ['cint', 'np_helper'],
        'cvhf': ['cgto', 'np_helper', 'cint'], 'ao2mo': ['cvhf', 'cint', 'np_helper']}


def ref_available():
    return os.path.isfile(os.path.join(REF_LIB, 'vhf', 'nr_direct.c'))


def build_ref(force=False):
    """Compile the reference drivers into oracle/_ref (needs the reference tree)."""
    if not ref_available():
        return None
    blas = find_blas()
    if blas is None:
        raise RuntimeError('no BLAS exporting dgemm_ found')
    os.makedirs(OUT_LIBDIR, exist_ok=True)
    with open(os.path.join(OUT_REF, 'reference_root'), 'w') as fh:
        fh.write(os.path.abspath(REF_ROOT))
    objdir = os.path.join(OUT_REF, 'obj')
    os.makedirs(objdir, exist_ok=True)
    stamp = os.path.join(OUT_LIBDIR, 'libcvhf.so')
    mine = [os.path.join(HERE, 'cint', 'cint_shim.c'), os.path.join(HERE, 'cint', 'cint.h'),
            os.path.abspath(__file__)]
    if not force and _newer(stamp, mine):
        return OUT_LIBDIR
    # config.h normally generated by CMake from pyscf/lib/config.h.in
    with open(os.path.join(OUT_REF, 'config.h'), 'w') as f:
        f.write('#if defined _OPENMP\n#include <omp.h>\n#else\n'
                '#define omp_get_thread_num() 0\n#define omp_get_num_threads() 1\n#endif\n'
                '#define XCFUN_MAX_DERIV_ORDER 3\n')
    inc = ['-I', OUT_REF, '-I', os.path.join(HERE, 'cint'), '-I', REF_LIB]
    objs = {}
    for grp, files in REF_GROUPS.items():
        objs[grp] = []
        for rel in files:
            src = os.path.join(REF_LIB, rel)
            obj = os.path.join(objdir, rel.replace('/', '__') + '.o')
            _run(['gcc'] + CFLAGS + inc + ['-c', src, '-o', obj])
            objs[grp].append(obj)
    shim_obj = os.path.join(objdir, 'cint_shim.o')
    _run(['gcc'] + CFLAGS + ['-I', os.path.join(HERE, 'cint'), '-c',
                             os.path.join(HERE, 'cint', 'cint_shim.c'), '-o', shim_obj])
    # stubs for every symbol still undefined after linking everything together
    defined = set()
    undefined = set()
    all_objs = [shim_obj] + [o for g in objs.values() for o in g]
    for o in all_objs:
        for line in _run(['nm', o]).splitlines():
            parts = line.split()
            if len(parts) == 2 and parts[0] == 'U':
                undefined.add(parts[1])
            elif len(parts) == 3 and parts[1] in 'TDBRVWCG':
                defined.add(parts[2])
    system = set()
    libs = [blas, '/lib/x86_64-linux-gnu/libc.so.6', '/lib/x86_64-linux-gnu/libm.so.6']
    libs += glob.glob('/usr/lib/gcc/x86_64-linux-gnu/*/libgomp.so')
    libs += glob.glob('/lib/x86_64-linux-gnu/libgomp.so*')
    for lib in libs:
        if not os.path.exists(lib):
            continue
        for line in _run(['nm', '-D', '--defined-only', lib]).splitlines():
            parts = line.split()
            if parts:
                system.add(parts[-1].split('@')[0])
    missing = sorted(s for s in undefined - defined - system
                     if not s.startswith('_') and not s.startswith('GOMP_') and not s.startswith('omp_'))
    stub_c = os.path.join(OUT_REF, 'cint_stubs.c')
    with open(stub_c, 'w') as f:
        f.write('#include <stdio.h>\n#include <stdlib.h>\n')
        for s in missing:
            f.write('int %s() { fprintf(stderr, "oracle: libcint symbol %s is not '
                    'available (outside the direct-SCF path)\\n"); abort(); return 0; }\n' % (s, s))
    stub_obj = os.path.join(objdir, 'cint_stubs.o')
    _run(['gcc'] + CFLAGS + ['-c', stub_c, '-o', stub_obj])
    objs['cint'] = [shim_obj, stub_obj]
    blasdir = os.path.dirname(blas)
    for grp in LINK_ORDER:
        out = os.path.join(OUT_LIBDIR, 'lib%s.so' % grp)
        cmd = ['gcc', '-shared', '-fopenmp', '-o', out] + objs[grp]
        cmd += ['-L', OUT_LIBDIR] + ['-l' + d for d in DEPS[grp]]
        # DT_RPATH (not RUNPATH) so that the BLAS's own dependency
        # (libgfortran next to it) resolves through this search path too
        cmd += [blas, '-lm', '-Wl,--disable-new-dtags', '-Wl,-rpath,$ORIGIN', '-Wl,-rpath,' + blasdir]
        _run(cmd)
    # Libraries of subsystems outside the J/K path (post-HF, DFT, PBC, ...)
    # are loaded at import time by modules that `pyscf.grad` pulls in.  Empty
    # placeholders let those imports succeed; any call into one fails loudly
    # with an AttributeError for the missing symbol.
    # Module-level code in those modules sets restype/argtypes on a few
    # symbols (e.g. pyscf/dft/libxc.py:47-90), so each placeholder defines
    # every name the Python sources access through the handle bound to it.
    import re
    handles = {}
    pyroot = os.path.join(REF_ROOT, 'pyscf')
    for dirpath, _, files in os.walk(pyroot):
        for fn in files:
            if not fn.endswith('.py'):
                continue
            try:
                text = open(os.path.join(dirpath, fn)).read()
            except (OSError, UnicodeDecodeError):
                continue
            for var, lib in re.findall(r"(\w+)\s*=\s*lib\.load_library\(['\"]lib(\w+)['\"]\)", text):
                if lib in PLACEHOLDER_LIBS:
                    syms = handles.setdefault(lib, set())
                    syms.update(re.findall(r"\b%s\.([A-Za-z_]\w*)" % re.escape(var), text))
    for name in PLACEHOLDER_LIBS:
        src = os.path.join(OUT_REF, 'placeholder_%s.c' % name)
        with open(src, 'w') as f:
            f.write('/* placeholder for a PySCF library outside the J/K path */\n'
                    'int oracle_placeholder_library(void) { return 0; }\n')
            for sym in sorted(handles.get(name, ())):
                if re.search(r'version|reference|doi|_name|splash|authors', sym):
                    # read as c_char_p at import time (pyscf/dft/libxc.py:83-113)
                    f.write('const char *%s(void) { return "0.0.0"; }\n' % sym)
                else:
                    f.write('int %s(void) { return 0; }\n' % sym)
        _run(['gcc', '-shared', '-fPIC', '-w', '-o', os.path.join(OUT_LIBDIR, 'lib%s.so' % name), src])
    return OUT_LIBDIR


PLACEHOLDER_LIBS = ['pbc', 'dft', 'ccsdt', 'mcscf', 'xcfun_itrf', 'xc_itrf', 'solvent', 'ri',
                    'pdft', 'mp', 'fft', 'fci', 'cc', 'agf2']


def write_pystub():
    """Import-time stand-ins for the reference.

    h5py is not installed; pyscf/lib/misc.py:39 imports it unconditionally
    and reads h5py.version.  A stub package in oracle/_ref/pystub satisfies
    the import (chkfiles are muted, so it is never used)."""
    d = os.path.join(OUT_REF, 'pystub', 'h5py')
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, '__init__.py'), 'w') as f:
        f.write('"""Import-only stand-in for h5py; the oracle never writes chkfiles."""\n'
                'class _V:\n    version = "3.0.0"\n    hdf5_version = "1.12.0"\n'
                'version = _V()\n__version__ = "3.0.0"\n'
                'class File:\n    def __init__(self, *a, **k):\n'
                '        raise RuntimeError("h5py is not available")\n'
                'class Group: pass\nclass Dataset: pass\n')
    # pyscf/lib/misc.py:47-80 inspects pyscf/lib/libnp_helper.so with pyelftools
    # when it is importable; the libraries live elsewhere here, so the stub
    # makes that optional probe take its ImportError branch.
    d = os.path.join(OUT_REF, 'pystub', 'elftools')
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, '__init__.py'), 'w') as f:
        f.write('raise ImportError("elftools probe disabled for the oracle")\n')
    with open(os.path.join(OUT_REF, 'pyext', 'pyscf', '__init__.py'), 'w') as f:
        f.write('')
    # chkfiles muted as in .github/workflows/run_tests.sh:9
    with open(os.path.join(OUT_REF, 'pyscf_conf.py'), 'w') as f:
        f.write('scf_hf_SCF_mute_chkfile = True\n')
    return os.path.join(OUT_REF, 'pystub')


def reference_env():
    """Environment variables that make the reference importable here."""
    env = dict(os.environ)
    env['PYSCF_EXT_PATH'] = os.path.join(OUT_REF, 'pyext')
    env['PYSCF_CONFIG_FILE'] = os.path.join(OUT_REF, 'pyscf_conf.py')
    # the reference drivers call dgemm_ inside OpenMP regions; PySCF itself
    # pins a pthreads OpenBLAS to one thread for that reason
    # (pyscf/lib/misc.py:69-80)
    env['OPENBLAS_NUM_THREADS'] = '1'
    pp = [REF_ROOT, os.path.join(OUT_REF, 'pystub')]
    if env.get('PYTHONPATH'):
        pp.append(env['PYTHONPATH'])
    env['PYTHONPATH'] = ':'.join(pp)
    return env


def build_all(force=False):
    build_oracle(force)
    if ref_available():
        build_ref(force)
        write_pystub()


if __name__ == '__main__':
    build_all(force='--force' in sys.argv)
    print('oracle built:', os.path.join(HERE, 'liboracle.so'))
    if ref_available():
        print('reference drivers built:', OUT_LIBDIR)
