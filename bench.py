"""Benchmark of the direct-SCF J/K build on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config h2o64_vtz|c20h42_vdz|h2o8_vdz]

One step = one FP64 J/K build (hermi=1) of the workload's density.  Default
workload: the synthetic (H2O)64 cluster (4x4x4 lattice, 3.0 A, +-0.3 A
jitter, seed 303) in cc-pVTZ, nao = 3712, with D = C C^T, C (nao x 320) of
N(0,1)/sqrt(nao) entries (seed 304).  Metric: shell quartets per second
(s8-unique quartets of PySCF _bas shells surviving the direct_scf_tol=1e-13
screen) with seconds per build alongside.

N > 1 (torchrun): every rank builds J/K of the same workload on its own GPU
(replicas, weak scaling); the time is the max over ranks.

--impl reference times the reference's own CPU implementation of the path
(PySCF's CVHFnr_direct_drv compiled from the reference sources, oracle/_ref,
on the oracle integral library) on all host cores, one step = one J/K build
of a bounded sample of the workload (its first 8 waters).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, 'tests', 'golden')
METRIC = 's per J/K build & shell quartets/s; mixed-prec vs FP64 at |dE|<=1e-6 Eh, 1 B200'
SAMPLES = {'h2o64_vtz': 'h2o64_vtz_sub8', 'c20h42_vdz': 'h2o8_vdz', 'h2o8_vdz': 'h2o8_vdz'}
L2_BYTES = 126 * 1024 * 1024


def load_workload(name):
    f = dict(numpy.load(os.path.join(GOLDEN, 'mol_%s.npz' % name)))
    nao = int(f['nao'])
    rng = numpy.random.default_rng(304)
    c = rng.standard_normal((nao, min(320, nao))) / numpy.sqrt(nao)
    f['dm'] = c @ c.T
    return f


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons while running."""

    FIELDS = ('clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in self.lines:
            p = [x.strip() for x in l.split(',')]
            if len(p) < 8:
                continue
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except ValueError:
                continue
            for nm, v in zip(names, p[4:8]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': float(numpy.median(sm)), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


def dist_init(n):
    import torch
    import torch.distributed as dist
    if n <= 1 or 'RANK' not in os.environ:
        return 0, 1, 0, None
    import datetime
    dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    rank, world = dist.get_rank(), dist.get_world_size()
    local = int(os.environ.get('LOCAL_RANK', rank))
    torch.cuda.set_device(local)
    return rank, world, local, dist


def cpu_reference(workload, steps, warmup):
    """The reference's CPU J/K build on a bounded sample of the workload."""
    os.environ.setdefault('OPENBLAS_NUM_THREADS', '1')
    from oracle import ref_driver
    sample = SAMPLES.get(workload, workload)
    f = load_workload(sample)
    cores = len(os.sched_getaffinity(0))
    if not ref_driver.available():
        return None, sample, cores, 'oracle/_ref not built'
    opt = ref_driver.RefVHFOpt(f['atm'], f['bas'], f['env'], 1e-13)
    # unit count: quartets the per-quartet screen keeps (the reference's block
    # screen may drop a few more, so the CPU rate is, if anything, flattered)
    import oracle
    from oracle.count import count_quartets
    nq = count_quartets(opt.q_cond, oracle.dm_cond(f['dm'], f['bas']), 1e-13)
    for _ in range(warmup):
        ref_driver.direct(f['dm'], opt, hermi=1)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ref_driver.direct(f['dm'], opt, hermi=1)
        times.append(time.perf_counter() - t0)
    t = float(numpy.median(times))
    return nq / t, sample, cores, (nq, t)


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    os.environ['OMP_NUM_THREADS'] = str(len(os.sched_getaffinity(0)))
    v, sample, cores, info = cpu_reference(args.config, max(1, args.steps), max(0, min(args.warmup, 1)))
    if v is None:
        print(json.dumps({'impl': 'reference', 'unavailable': info}))
        return
    nq, t = info
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'shell quartets/s', 'n_gpus': args.gpus,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t * 1e3, 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic',
        'config': {'workload': args.config, 'sample': sample, 'precision': 'fp64', 'direct_scf_tol': 1e-13},
        'cpu_baseline': {'value': v, 'unit': 'shell quartets/s', 'cores': cores, 'kind': 'reference',
                         'sample': '%s: one J/K build (%d quartets, %.2f s), PySCF CVHFnr_direct_drv from the '
                                   'reference sources on the oracle integral library (upstream libcint absent)'
                                   % (sample, nq, t)},
        'e2e': {'value': v, 'unit': 'shell quartets/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line))


def run_gpu(args):
    import torch
    from pyscf_b200 import lib, flops
    from pyscf_b200 import _vhf
    rank, world, local, dist = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    f = load_workload(args.config)
    nao = int(f['nao'])
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=local)
    d = torch.tensor(f['dm'], device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        plan.get_jk_device(d, hermi=1)
    torch.cuda.synchronize(dev)
    plan.set_profiling(True)
    class_ms = {}
    times = []
    nq = npq = launches = 0
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)    # evict L2 between timed builds
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            vj, vk = plan.get_jk_device(d, hermi=1)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
            st = plan.stats()
            nq += st['quartets']
            npq += st['prim_quartets']
            launches += st['kernel_launches']
            for c in plan.class_stats():
                k = (c['la'], c['lb'], c['lc'], c['ld'])
                acc = class_ms.setdefault(k, dict(c, ms=0.0, quartets=0, prim_quartets=0))
                acc['ms'] += c['ms']
                acc['quartets'] += c['quartets']
                acc['prim_quartets'] += c['prim_quartets']
        torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    t_total = sum(times)
    if dist is not None:
        tt = torch.tensor([t_total], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_total = float(tt.item())
    plan.set_profiling(False)
    q_per_build = nq / args.steps
    value = world * nq / t_total
    # roofline: FP64 pipe (the recurrences are scalar FP64, no tensor-core form)
    fp64_peak = lib.measure_fp64_peak(local)
    cls = list(class_ms.values())
    build_flops = flops.build_flops(cls) / args.steps
    dom = max(cls, key=lambda c: c['ms'])
    dom_ms = dom['ms'] / args.steps
    dom_flops = flops.class_flops(dom) / args.steps
    achieved = dom_flops / (dom_ms * 1e-3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, 'profiles', 'traffic.json')
    key = 'jk_%d%d%d%d_%s' % (dom['la'], dom['lb'], dom['lc'], dom['ld'], args.config)
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(key)
    # end to end through the public API, host arrays in pinned memory
    dm_host = torch.from_numpy(f['dm']).pin_memory().numpy()
    out = torch.empty((2, nao, nao), dtype=torch.float64).pin_memory().numpy()
    vhfopt = _vhf.VHFOpt(_Mol(f), direct_scf_tol=1e-13, device=local)
    _vhf.direct(dm_host, f['atm'], f['bas'], f['env'], vhfopt, hermi=1, out=out)
    e2e_times = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _vhf.direct(dm_host, f['atm'], f['bas'], f['env'], vhfopt, hermi=1, out=out)
        e2e_times.append(time.perf_counter() - t0)
    t_e2e = float(numpy.mean(e2e_times))
    if dist is not None:
        tt = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    clocks = clk.summary()
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': 'shell quartets/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t_total / args.steps * 1e3,
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
            'data': 'synthetic',
            'config': {'workload': args.config, 'nao': nao, 'nbas': int(f['bas'].shape[0]),
                       'density': 'C C^T, C nao x 320 N(0,1)/sqrt(nao), seed 304', 'hermi': 1,
                       'precision': 'fp64', 'direct_scf_tol': 1e-13, 'parallelism': 'replicas' if world > 1 else 'single',
                       'l2': 'flushed (256 MB write) before every timed build'},
            's_per_build': t_total / args.steps,
            'quartets_per_build': q_per_build, 'prim_quartets_per_build': npq / args.steps,
            'fp64_tflops_build': build_flops / (t_total / args.steps) / 1e12,
            'roofline': {'bound': 'fp64', 'kernel': 'jk_%s_kernel<%d,%d,%d,%d>' % (
                             'thread' if dom['family'] == 0 else 'warp', dom['la'], dom['lb'], dom['lc'], dom['ld']),
                         'achieved': achieved, 'peak': fp64_peak, 'unit': 'TFLOP/s', 'frac': achieved / fp64_peak,
                         'peak_source': 'measured FP64 FMA loop on this GPU (b200jk_measure_fp64_peak)',
                         'share': dom_ms * 1e-3 / (t_total / args.steps), 'traffic': traffic},
            'e2e': {'value': world * q_per_build / t_e2e, 'unit': 'shell quartets/s',
                    's_per_build': t_e2e, 'h2d_bytes_per_step': int(nao * nao * 8),
                    'd2h_bytes_per_step': int(2 * nao * nao * 8),
                    'timing': 'wall clock around pyscf_b200._vhf.direct with pinned host arrays'},
            'classes': [{'class': '(%d%d|%d%d)' % (c['la'], c['lb'], c['lc'], c['ld']),
                         'family': 'thread' if c['family'] == 0 else 'group',
                         'ms_per_build': c['ms'] / args.steps,
                         'share': c['ms'] * 1e-3 / t_total,
                         'quartets_per_build': c['quartets'] / args.steps,
                         'tflops': flops.class_flops(c) / (c['ms'] * 1e-3) / 1e12 if c['ms'] > 0 else None}
                        for c in sorted(cls, key=lambda c: -c['ms'])[:12]],
            'gpu_launches': int(launches),
            'clocks': clocks,
        }
        cb = None
        if world == 1 and not args.no_cpu_baseline:
            try:
                os.environ['OMP_NUM_THREADS'] = str(len(os.sched_getaffinity(0)))
                v, sample, cores, info = cpu_reference(args.config, 1, 0)
                if v is not None:
                    nq_s, t_s = info
                    cb = {'value': v, 'unit': 'shell quartets/s', 'cores': cores, 'kind': 'reference',
                          'sample': '%s: one J/K build (%d quartets, %.2f s), PySCF CVHFnr_direct_drv from the '
                                    'reference sources on the oracle integral library' % (sample, nq_s, t_s)}
            except Exception as e:  # the baseline must not sink the GPU measurement
                cb = {'value': None, 'error': str(e)[:200]}
        line['cpu_baseline'] = cb
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


class _Mol:
    def __init__(self, f):
        self._atm, self._bas, self._env = f['atm'], f['bas'], f['env']
        self.cart = bool(f['cart'])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--config', default='h2o64_vtz')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
