"""Benchmark of the direct-SCF J/K build on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--config h2o64_vtz|c20h42_vdz|h2o8_vdz]

One step = one FP64 J/K build (hermi=1) of the workload's density.  Default
workload: the synthetic (H2O)64 cluster (4x4x4 lattice, 3.0 A, +-0.3 A
jitter, seed 303) in cc-pVTZ, nao = 3712, with D = C C^T, C (nao x 320) of
N(0,1)/sqrt(nao) entries (seed 304).  Metric: shell quartets per second
(s8-unique quartets of PySCF _bas shells surviving the direct_scf_tol=1e-13
screen) with seconds per build alongside.

N > 1 (torchrun): the quartets of the one workload are sharded over the ranks
by bra shell pair (b200jk_set_shard) and every step ends with one NCCL
all-reduce of [J; K] inside the timed region (strong scaling); the time is the
max over ranks and the value counts the quartets of all ranks.

Besides the FP64 headline the line carries, measured in the same run:
  mixed   the mixed-precision build (float32 quartets below tau, float64
          accumulation) of the same density, its time, speed-up over FP64,
          float32 fraction and error against the FP64 build (max |dJ|, |dK|,
          dE = 1/2 tr(D dJ) - 1/4 tr(D dK)), and the same for a
          difference-density build (dD = 1e-4 C2 C2^T, the late-SCF regime);
  grad    the nuclear-gradient J/K (int2e_ip1) of (H2O)16/cc-pVDZ;
  batch   512 molecules (H2O)n, n ~ U{1..16}, cc-pVDZ (tests/golden/
          batch_h2o_vdz512.npz) in one batched build (one launch per quartet
          class for all molecules), FP64 and mixed, against the same 512
          builds run one molecule after another;
  scf     C20H42/cc-pVDZ RHF with incremental builds, FP64 and mixed: per
          build the mixed J/K against the FP64 J/K of the same density change
          and per iteration the energy against the FP64 SCF; final energies
          against the reference's RHF energy (tests/golden/mol_c20h42_vdz.npz);
  batch_scf  whole SCF iterations of the 512 molecules as one CUDA-graph
          replay, and the convergence of the first 64 against the reference
          energies of tests/golden/batch_scf_sample.npz;
  incore  the in-core path of (H2O)8/cc-pVDZ: GPU fill of the s8 integral
          tensor and J/K contracted from it (HBM roofline of the contraction)
          against the direct build of the same density.

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


def _max_over_ranks(v, dist, dev):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(v, dist, dev):
    if dist is None:
        return v
    import torch
    t = torch.tensor([float(v)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _timed_builds(plan, d, flush, stream, steps, dist, build):
    """steps builds of `build()` on the device, L2 flushed before each;
    returns (list of seconds, summed plan stats)."""
    import torch
    times = []
    nq = npq = nq32 = launches = 0
    for _ in range(steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = build()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) * 1e-3)
        st = plan.stats()
        nq += st['quartets']
        npq += st['prim_quartets']
        nq32 += st['fp32_quartets']
        launches += st['kernel_launches']
    return times, dict(quartets=nq, prim_quartets=npq, fp32_quartets=nq32, kernel_launches=launches), out


def batch_report(local, flush, stream, steps, tau, dist=None):
    """Batched J/K of the 512-molecule workload vs one-by-one builds.  With
    several ranks each GPU takes whole molecules (pyscf_b200.dist.
    shard_molecules, no collective on the data path) and only the batched
    FP64 build is timed; the caller combines the ranks' numbers."""
    import torch
    from pyscf_b200 import lib
    from pyscf_b200 import dist as b2dist
    f = dict(numpy.load(os.path.join(GOLDEN, 'batch_h2o_vdz512.npz')))
    dev = torch.device('cuda', local)
    nmol = len(f['nao'])
    mine = set(b2dist.my_molecules(list(numpy.diff(f['bas_off'])))) if dist is not None else set(range(nmol))
    plans, dms = [], []
    rng = numpy.random.default_rng(405)
    for m in range(nmol):
        nao, nocc = int(f['nao'][m]), 5 * int(f['nwater'][m])
        c = rng.standard_normal((nao, nocc)) / numpy.sqrt(nao)
        if m not in mine:
            continue
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        b0, b1 = f['bas_off'][m], f['bas_off'][m + 1]
        e0, e1 = f['env_off'][m], f['env_off'][m + 1]
        p = lib.Plan(f['atm'][a0:a1], f['bas'][b0:b1], f['env'][e0:e1], direct_scf_tol=1e-13, device=local)
        p.set_mixed_threshold(tau)
        plans.append(p)
        dms.append(torch.tensor(c @ c.T, device=dev))
    batch = lib.Batch(plans)

    def timed(fn, n):
        fn()
        t = []
        for _ in range(n):
            flush.fill_(1.0)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            t.append(e0.elapsed_time(e1))
        return float(numpy.median(t))
    ms_b64 = timed(lambda: batch.get_jk_device(dms, hermi=1), steps)
    q = batch.stats()['quartets']
    launches = batch.stats()['kernel_launches']
    if dist is not None:
        # this rank's numbers; the caller combines them over the ranks
        return {'batched_fp64_ms': ms_b64, 'quartets_per_build': q}
    ms_b32 = timed(lambda: batch.get_jk_device(dms, hermi=1, precision=lib.PREC_MIXED), steps)
    f32 = batch.stats()['fp32_quartets'] / max(1, batch.stats()['quartets'])

    def one_by_one():
        for p, d in zip(plans, dms):
            p.get_jk_device(d, hermi=1)
    ms_seq = timed(one_by_one, 1)
    # the batched build captured once in a CUDA graph and replayed
    graph_ms = None
    try:
        batch.get_jk_device(dms, hermi=1)
        vj = [torch.empty_like(d) for d in dms]
        vk = [torch.empty_like(d) for d in dms]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            batch.get_jk_device_async(dms, vj, vk, hermi=1)
        torch.cuda.current_stream(dev).wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            batch.get_jk_device_async(dms, vj, vk, hermi=1)
        graph_ms = timed(g.replay, steps)
    except Exception as e:  # the graph number must not sink the batch line
        graph_ms = 'error: %s' % str(e)[:120]
    return {'workload': '512 x (H2O)n, n ~ U{1..16} (seed 404), 3x3x2 lattice sites, cc-pVDZ',
            'molecules': len(plans), 'total_nao': int(f['nao'].sum()), 'quartets_per_build': q,
            'batched_fp64_ms': ms_b64, 'batched_fp64_quartets_per_s': q / (ms_b64 * 1e-3),
            'batched_mixed_ms': ms_b32, 'mixed_tau': tau, 'mixed_fp32_fraction': f32,
            'one_by_one_fp64_ms': ms_seq, 'batching_speedup': ms_seq / ms_b64,
            'cuda_graph_replay_fp64_ms': graph_ms,
            'kernel_launches_per_batched_build': launches,
            'density': 'per molecule C C^T, C nao x 5n N(0,1)/sqrt(nao), seed 405'}


def _fp(a):
    """PySCF's lib.fp fingerprint (pyscf/lib/misc.py:1259-1263), on the GPU."""
    import torch
    a = a.reshape(-1)
    w = torch.cos(torch.arange(a.numel(), device=a.device, dtype=torch.float64))
    return float(torch.dot(w, a))


def vs_oracle(workload, d, vj64, vk64, plan, tau):
    """FP64 and mixed J/K against the reference drivers' J/K of the same
    density (sampled rows, E2, fingerprints); None without the fixture."""
    import torch
    from pyscf_b200 import lib
    path = os.path.join(GOLDEN, 'jk_%s.npz' % workload)
    if not os.path.exists(path):
        return {'error': 'no reference fixture %s' % os.path.basename(path)}
    g = dict(numpy.load(path))
    rows = torch.tensor(g['rows'], device=d.device, dtype=torch.long)
    rj = torch.tensor(g['vj_rows'], device=d.device)
    rk = torch.tensor(g['vk_rows'], device=d.device)
    e2_ref = float(g['e2'])

    def cmp(vj, vk):
        e2 = float(0.5 * torch.sum(d * vj) - 0.25 * torch.sum(d * vk))
        return {'max_dJ_rows': float((vj[rows] - rj).abs().max()), 'max_dK_rows': float((vk[rows] - rk).abs().max()),
                'dE2_Eh': e2 - e2_ref, 'dfp_J': _fp(vj) - float(g['fp_j']), 'dfp_K': _fp(vk) - float(g['fp_k'])}
    out = {'reference': 'PySCF CVHFnr_direct_drv (reference sources, oracle integral library), %d sampled rows '
                        'of %d shells, E2 = %.10f' % (len(g['rows']), len(g['shells']), e2_ref),
           'fp64': cmp(vj64, vk64)}
    plan.set_mixed_threshold(tau)
    vj, vk = plan.get_jk_device(d, hermi=1, precision=lib.PREC_MIXED)
    plan.set_mixed_threshold(0.0)
    out['mixed'] = cmp(vj, vk)
    out['mixed']['tau'] = tau
    return out


def batch_scf_report(local, steps):
    """Whole SCF iterations of the 512-molecule workload as one CUDA graph:
    batched J/K, Fock, DIIS and purified density of every molecule."""
    import torch
    from pyscf_b200 import lib, batch_scf
    f = dict(numpy.load(os.path.join(GOLDEN, 'batch_h2o_vdz512.npz')))
    plans, nelec, enuc = [], [], []
    for m in range(len(f['nao'])):
        a0, a1 = f['atm_off'][m], f['atm_off'][m + 1]
        b0, b1 = f['bas_off'][m], f['bas_off'][m + 1]
        e0, e1 = f['env_off'][m], f['env_off'][m + 1]
        atm, env = f['atm'][a0:a1], f['env'][e0:e1]
        plans.append(lib.Plan(atm, f['bas'][b0:b1], env, direct_scf_tol=1e-13, device=local))
        nelec.append(10 * int(f['nwater'][m]))
        z = atm[:, 0].astype(float)
        xyz = numpy.array([env[q:q + 3] for q in atm[:, 1]])
        r = numpy.linalg.norm(xyz[:, None] - xyz[None], axis=-1)
        iu = numpy.triu_indices(len(z), 1)
        enuc.append(float((z[:, None] * z[None] / numpy.where(r > 0, r, 1.0))[iu].sum()))
    t0 = time.perf_counter()
    scf = batch_scf.BatchRHF(plans, nelec, enuc)
    scf.start()
    scf.capture()
    setup = time.perf_counter() - t0
    stream = torch.cuda.current_stream(torch.device('cuda', local))
    e0_ = torch.cuda.Event(enable_timing=True)
    e1_ = torch.cuda.Event(enable_timing=True)
    e0_.record(stream)
    for _ in range(steps):
        scf.graph.replay()
    e1_.record(stream)
    e1_.synchronize()
    ms = e0_.elapsed_time(e1_) / steps
    done = steps + 2      # the start() and capture() iterations
    del scf
    # convergence of the first 64 molecules (they hold the 8 with reference
    # energies) to the reference's conv_tol, from the same core guess
    ref = dict(numpy.load(os.path.join(GOLDEN, 'batch_scf_sample.npz')))
    sub = batch_scf.BatchRHF(plans[:64], nelec[:64], enuc[:64])
    sub.start()
    sub.capture()
    it = 2
    while True:
        e, de = sub.run(5)
        it += 5
        if (de < 1e-10).all() or it >= 60:
            break
    conv = {'molecules': 64, 'iterations': it, 'max_dE_last_iteration': float(de.max()),
            'max_idempotency_error': float(sub.idem_err.max()),
            'max_abs_E_minus_reference': float(max(abs(e[m] - er) for m, er in zip(ref['sample'], ref['e_rhf']))),
            'reference_molecules': [int(m) for m in ref['sample']]}
    return {'workload': '512 x (H2O)n cc-pVDZ, one SCF iteration of all molecules per CUDA-graph replay '
                        '(batched J/K, Fock, CDIIS, purified density)', 'molecules': len(plans),
            'ms_per_iteration': ms, 'replays_timed': steps, 'iterations_before_timing': done - steps,
            'setup_s': setup, 'convergence_first_64': conv}


def incore_report(local, steps):
    """The in-core path on the reference's CPU-runnable workload, (H2O)8/
    cc-pVDZ (the reference's RHF.get_jk goes in core there): GPU fill of the
    s8 tensor, then J/K builds contracted from it (tensor 1.37 GB > L2, so no
    flush is needed), against the direct build of the same density."""
    import torch
    from pyscf_b200 import lib, incore
    f = dict(numpy.load(os.path.join(GOLDEN, 'mol_h2o8_vdz.npz')))
    dev = torch.device('cuda', local)
    stream = torch.cuda.current_stream(dev)
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=local)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn, n):
        ev[0].record(stream)
        for _ in range(n):
            r = fn()
        ev[1].record(stream)
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1]) / n, r

    t0 = time.perf_counter()
    eri = plan.int2e_s8(device=True)
    torch.cuda.synchronize(dev)
    first_fill = time.perf_counter() - t0
    del eri
    fill_ms, eri = timed(lambda: plan.int2e_s8(device=True), 1)
    d = torch.as_tensor(f['dm_conv'], device=dev)
    for _ in range(3):
        incore.incore(eri, d, hermi=1)
    jk_ms, (vj, vk) = timed(lambda: incore.incore(eri, d, hermi=1), max(steps, 3))
    err = max(float(abs(vj.cpu().numpy() - f['vj_conv']).max()), float(abs(vk.cpu().numpy() - f['vk_conv']).max()))
    for _ in range(3):
        plan.get_jk_device(d, hermi=1)
    direct_ms, _ = timed(lambda: plan.get_jk_device(d, hermi=1), max(steps, 3))
    nbytes = eri.numel() * 8
    gbs = nbytes / (jk_ms * 1e-3) / 1e9
    peak = _hbm_peak()
    return {'workload': 'h2o8_vdz (nao 192), RHF.get_jk in-core branch: s8 tensor filled on the GPU, J/K contracted '
                        'from it', 'tensor_bytes': nbytes, 'fill_ms': fill_ms, 'first_fill_s': first_fill,
            'jk_ms_per_build': jk_ms, 'direct_jk_ms_per_build': direct_ms,
            'speedup_vs_direct': direct_ms / jk_ms, 'max_abs_err_vs_reference': err,
            'roofline': {'bound': 'hbm', 'kernel': 'incore_fast_kernel<8,true>', 'achieved': gbs, 'peak': peak,
                         'unit': 'GB/s', 'frac': gbs / peak if peak else None,
                         'bytes': 'the s8 tensor read once per build (8 bytes an entry), over the time of the whole '
                                  'in-core call (its small pair-density, unpack and finish kernels included)',
                         'peak_source': 'MEASURED_PEAKS.json hbm_gbs'}}


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            return float(json.load(fh)['hbm_gbs'])
    except (OSError, KeyError, ValueError):
        return 6650.0


def scf_report(local, tau):
    """Per-iteration errors of a mixed-precision RHF on C20H42/cc-pVDZ."""
    from pyscf_b200 import lib, rhf
    f = dict(numpy.load(os.path.join(GOLDEN, 'mol_c20h42_vdz.npz')))
    if 'hcore' not in f:
        return {'error': 'fixture without hcore'}
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=local)
    t0 = time.perf_counter()
    rows, e64, e32, c64, c32 = rhf.mixed_precision_report(f['hcore'], f['ovlp'], int(f['nelec']), float(f['e_nuc']),
                                                          plan, tau=tau, conv_tol=1e-10)
    ref = float(f['e_rhf'])
    return {'workload': 'C20H42/cc-pVDZ RHF, conv_tol 1e-10, incremental builds on dD', 'tau': tau,
            'converged': [bool(c64), bool(c32)], 'e_reference': ref,
            'dE_fp64_vs_reference': e64 - ref, 'dE_mixed_vs_reference': e32 - ref,
            'builds': len(rows), 'wall_s': time.perf_counter() - t0,
            'per_build': [{k: (round(v, 15) if isinstance(v, float) else v) for k, v in r.items()
                           if k in ('build', 'max_dJ', 'max_dK', 'fp32_fraction', 'dE')} for r in rows]}


def run_gpu(args):
    import torch
    from pyscf_b200 import lib, flops
    from pyscf_b200 import _vhf
    from pyscf_b200 import dist as b2dist
    rank, world, local, dist = dist_init(args.gpus)
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    f = load_workload(args.config)
    nao = int(f['nao'])
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13, device=local)
    if world > 1:
        plan.set_shard(rank, world)
    d = torch.tensor(f['dm'], device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def build64():
        vj, vk = plan.get_jk_device(d, hermi=1)
        if dist is not None:
            b2dist.reduce_jk(vj, vk)
        return vj, vk

    # the per-class launch variants (kets per lane of the register family,
    # lanes per quartet of the shared-memory family; float64 quartets and the
    # float32 pass of mixed builds) are tuned once per plan on the workload's
    # density, like the planning
    tuning = plan.autotune(d)
    for _ in range(args.warmup):
        build64()
    torch.cuda.synchronize(dev)
    plan.set_profiling(True)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        times, tot, (vj64, vk64) = _timed_builds(plan, d, flush, stream, args.steps, dist, build64)
        torch.cuda.synchronize(dev)
    if dist is not None:
        dist.barrier()
    plan.set_profiling(False)
    class_ms = {}
    # per-class times of the last build (profiling was on for all timed builds)
    for c in plan.class_stats():
        class_ms[(c['la'], c['lb'], c['lc'], c['ld'])] = dict(c)
    t_total = _max_over_ranks(sum(times), dist, dev)
    nq_all = _sum_over_ranks(tot['quartets'], dist, dev)
    q_per_build = nq_all / args.steps
    value = nq_all / t_total
    # roofline: FP64 pipe (the recurrences are scalar FP64, no tensor-core form)
    fp64_peak = lib.measure_fp64_peak(local)
    cls = list(class_ms.values())
    build_flops = flops.build_flops(cls)
    dom = max(cls, key=lambda c: c['ms'])
    dom_ms = dom['ms']
    dom_flops = flops.class_flops(dom)
    achieved = dom_flops / (dom_ms * 1e-3) / 1e12
    traffic = None
    tpath = os.path.join(ROOT, 'profiles', 'traffic.json')
    key = 'jk_%d%d%d%d_%s' % (dom['la'], dom['lb'], dom['lc'], dom['ld'], args.config)
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get(key)

    # mixed precision on the same density, error against the FP64 build
    def mixed_report(dens, tag, steps):
        plan.set_mixed_threshold(args.tau)

        def build32():
            vj, vk = plan.get_jk_device(dens, hermi=1, precision=lib.PREC_MIXED)
            if dist is not None:
                b2dist.reduce_jk(vj, vk)
            return vj, vk

        def build64d():
            vj, vk = plan.get_jk_device(dens, hermi=1)
            if dist is not None:
                b2dist.reduce_jk(vj, vk)
            return vj, vk
        build32()
        t32, s32, (vj, vk) = _timed_builds(plan, dens, flush, stream, steps, dist, build32)
        if tag == 'D':
            t64, j64, k64 = times, vj64, vk64
        else:
            build64d()
            t64, _, (j64, k64) = _timed_builds(plan, dens, flush, stream, steps, dist, build64d)
        ms32 = _max_over_ranks(sum(t32), dist, dev) / steps * 1e3
        ms64 = _max_over_ranks(sum(t64), dist, dev) / len(t64) * 1e3
        dj = float((vj - j64).abs().max())
        dk = float((vk - k64).abs().max())
        de = float(0.5 * torch.sum(dens * ((vj - j64) - 0.5 * (vk - k64))))
        return {'density': tag, 'tau': args.tau, 'ms_per_build': ms32, 'fp64_ms_per_build': ms64,
                'speedup_vs_fp64': ms64 / ms32, 'fp32_quartet_fraction': s32['fp32_quartets'] / max(1, s32['quartets']),
                'max_dJ': dj, 'max_dK': dk, 'dE_Eh': de}
    mixed = [mixed_report(d, 'D', args.steps)]
    # FP64 and mixed J/K of the workload density against the reference's
    # driver (tests/golden/jk_<workload>.npz, written by
    # tests/golden/make_h2o64_golden.py): sampled rows element-wise, the
    # two-electron energy E2 = 1/2 tr(D J) - 1/4 tr(D K) and the fingerprints
    oracle_cmp = vs_oracle(args.config, d, vj64, vk64, plan, args.tau) if world == 1 else None
    rng = numpy.random.default_rng(305)
    c2 = rng.standard_normal((nao, 64)) / numpy.sqrt(nao)
    dd = torch.tensor(1e-4 * (c2 @ c2.T), device=dev)
    mixed.append(mixed_report(dd, 'dD = 1e-4 C2 C2^T (C2 nao x 64, seed 305)', 1))
    plan.set_mixed_threshold(0.0)

    # nuclear-gradient J/K of the (H2O)16/cc-pVDZ workload
    grad_line = None
    try:
        fg = load_workload('h2o16_vdz')
        gplan = lib.Plan(fg['atm'], fg['bas'], fg['env'], direct_scf_tol=1e-13, device=local)
        if world > 1:
            gplan.set_shard(rank, world)
        dg = torch.tensor(fg['dm'], device=dev)

        def gbuild():
            vj, vk = gplan.grad_jk_device(dg)
            if dist is not None:
                b2dist.reduce_jk(vj, vk)
            return vj, vk
        gbuild()
        gt = []
        gq = 0
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            gbuild()
            e1.record(stream)
            e1.synchronize()
            gt.append(e0.elapsed_time(e1) * 1e-3)
            gq += gplan.grad_stats()['quartets']
        tg = _max_over_ranks(sum(gt), dist, dev)
        gq = _sum_over_ranks(gq, dist, dev)
        grad_line = {'workload': 'h2o16_vdz', 'nao': int(fg['nao']), 'ms_per_build': tg / args.steps * 1e3,
                     'quartet_sides_per_build': gq / args.steps, 'quartet_sides_per_s': gq / tg,
                     'screen': 'CVHFgrad_jk_prescreen, tol 1e-14'}
        if world == 1:
            # the two-electron force as the RHF gradient computes it: the
            # fused contraction with D x D, no vj/vk (b200jk_grad_contract)
            gplan.grad_contract(dg)
            ft = []
            for _ in range(args.steps):
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                gplan.grad_contract(dg)
                e1.record(stream)
                e1.synchronize()
                ft.append(e0.elapsed_time(e1))
            grad_line['fused_force_ms_per_build'] = float(numpy.mean(ft))
    except Exception as e:  # the gradient line must not sink the J/K measurement
        grad_line = {'error': str(e)[:200]}

    batch_line = None
    if world == 1:
        try:
            batch_line = batch_report(local, flush, stream, args.steps, args.tau)
        except Exception as e:  # the batch line must not sink the J/K measurement
            batch_line = {'error': str(e)[:200]}
    else:
        # whole molecules per GPU; every rank takes part in the two
        # reductions whatever its local outcome
        try:
            part = batch_report(local, flush, stream, args.steps, args.tau, dist=dist)
        except Exception as e:  # the batch line must not sink the J/K measurement
            part = {'batched_fp64_ms': float('nan'), 'quartets_per_build': 0, 'error': str(e)[:200]}
        ms_b = _max_over_ranks(part['batched_fp64_ms'], dist, dev)
        q_b = _sum_over_ranks(part['quartets_per_build'], dist, dev)
        batch_line = {'workload': '512 x (H2O)n, n ~ U{1..16} (seed 404), 3x3x2 lattice sites, cc-pVDZ',
                      'sharding': 'whole molecules per GPU (longest processing time first), no data-path '
                                  'collective', 'n_gpus': world, 'quartets_per_build': q_b,
                      'batched_fp64_ms_max_over_ranks': ms_b,
                      'batched_fp64_quartets_per_s': q_b / (ms_b * 1e-3) if ms_b == ms_b and ms_b > 0 else None}
        if 'error' in part:
            batch_line['error_rank%d' % rank] = part['error']

    scf_line = None
    if world == 1:
        try:
            scf_line = scf_report(local, args.tau)
        except Exception as e:  # the SCF line must not sink the J/K measurement
            scf_line = {'error': str(e)[:200]}

    batch_scf_line = None
    if world == 1:
        try:
            batch_scf_line = batch_scf_report(local, max(1, min(args.steps, 3)))
        except Exception as e:  # the batched-SCF line must not sink the J/K measurement
            batch_scf_line = {'error': str(e)[:200]}

    incore_line = None
    if world == 1:
        try:
            incore_line = incore_report(local, args.steps)
        except Exception as e:  # the in-core line must not sink the J/K measurement
            incore_line = {'error': str(e)[:200]}

    # end to end through the public API, host arrays in pinned memory
    dm_host = torch.from_numpy(f['dm']).pin_memory().numpy()
    out = torch.empty((2, nao, nao), dtype=torch.float64).pin_memory().numpy()
    vhfopt = _vhf.VHFOpt(_Mol(f), direct_scf_tol=1e-13, device=local)
    if world > 1:
        vhfopt.plan.set_shard(rank, world)
    e2e_times = []
    for it in range(1 + max(1, min(args.steps, 3))):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _vhf.direct(dm_host, f['atm'], f['bas'], f['env'], vhfopt, hermi=1, out=out)
        if dist is not None:
            o = torch.from_numpy(out).to(dev)
            dist.all_reduce(o)
            out[...] = o.cpu().numpy()
        if it > 0:
            e2e_times.append(time.perf_counter() - t0)
    t_e2e = _max_over_ranks(float(numpy.mean(e2e_times)), dist, dev)
    clocks = clk.summary()
    if rank == 0:
        line = {
            'metric': METRIC, 'value': value, 'unit': 'shell quartets/s', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t_total / args.steps * 1e3,
            'higher_is_better': True, 'scaling': 'strong' if world > 1 else 'weak', 'vs_baseline': None,
            'dtype': 'f64', 'data': 'synthetic',
            'config': {'workload': args.config, 'nao': nao, 'nbas': int(f['bas'].shape[0]),
                       'density': 'C C^T, C nao x 320 N(0,1)/sqrt(nao), seed 304', 'hermi': 1,
                       'precision': 'fp64', 'direct_scf_tol': 1e-13,
                       'parallelism': ('bra-pair shards + NCCL all-reduce of [J;K], %d GPUs' % world) if world > 1
                       else 'single',
                       'l2': 'flushed (256 MB write) before every timed build',
                       'autotuned_classes': int(sum(tuning)),
                       'autotuned_classes_fp32_pass': int(sum(plan.tuning(lib.PREC_MIXED)))},
            's_per_build': t_total / args.steps,
            'quartets_per_build': q_per_build, 'prim_quartets_per_build': _sum_over_ranks(tot['prim_quartets'], dist, dev) / args.steps,
            'fp64_tflops_build': build_flops / (t_total / args.steps) / 1e12 if world == 1 else None,
            'roofline': {'bound': 'fp64', 'kernel': 'jk_%s_kernel<%d,%d,%d,%d>' % (
                             'thread' if dom['family'] == 0 else 'warp', dom['la'], dom['lb'], dom['lc'], dom['ld']),
                         'achieved': achieved, 'peak': fp64_peak, 'unit': 'TFLOP/s', 'frac': achieved / fp64_peak,
                         'peak_source': 'measured FP64 FMA loop on this GPU (b200jk_measure_fp64_peak)',
                         'share': dom_ms * 1e-3 / (sum(times) / args.steps), 'traffic': traffic},
            'grad': grad_line,
            'batch': batch_line,
            'scf': scf_line,
            'batch_scf': batch_scf_line,
            'incore': incore_line,
            'e2e': {'value': q_per_build / t_e2e, 'unit': 'shell quartets/s',
                    's_per_build': t_e2e, 'h2d_bytes_per_step': int(nao * nao * 8),
                    'd2h_bytes_per_step': int(2 * nao * nao * 8),
                    'timing': 'wall clock around pyscf_b200._vhf.direct with pinned host arrays'},
            'classes': [{'class': '(%d%d|%d%d)' % (c['la'], c['lb'], c['lc'], c['ld']),
                         'family': 'thread' if c['family'] == 0 else 'group',
                         'ms_per_build': c['ms'],
                         'share': c['ms'] * 1e-3 / (sum(times) / args.steps),
                         'quartets_per_build': c['quartets'],
                         'tflops': flops.class_flops(c) / (c['ms'] * 1e-3) / 1e12 if c['ms'] > 0 else None}
                        for c in sorted(cls, key=lambda c: -c['ms'])[:8]],
            'gpu_launches': int(tot['kernel_launches']),
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
        # last, so that a truncated log still shows them: the mixed-precision
        # builds (speed-up over FP64, float32 fraction, errors) and both
        # precisions against the reference drivers' J/K
        line['vs_oracle'] = oracle_cmp
        line['mixed'] = mixed
        m0 = mixed[0]
        line['mixed_summary'] = {'speedup_vs_fp64': m0['speedup_vs_fp64'], 'ms_per_build': m0['ms_per_build'],
                                 'fp64_ms_per_build': m0['fp64_ms_per_build'],
                                 'fp32_quartet_fraction': m0['fp32_quartet_fraction'], 'tau': m0['tau'],
                                 'dE2_vs_oracle_Eh': (oracle_cmp or {}).get('mixed', {}).get('dE2_Eh'),
                                 'max_dJ_vs_oracle': (oracle_cmp or {}).get('mixed', {}).get('max_dJ_rows'),
                                 'max_dK_vs_oracle': (oracle_cmp or {}).get('mixed', {}).get('max_dK_rows'),
                                 'dD_speedup_vs_fp64': mixed[1]['speedup_vs_fp64'] if len(mixed) > 1 else None}
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_one_build(args):
    from pyscf_b200 import lib
    f = load_workload(args.config)
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    if args.autotune:
        plan.autotune(f['dm'])
    if args.variants is not None:
        # the FP64 variants of an earlier tuning, replayed without timing:
        # class index, or class:variant
        tun = [0] * 55
        for x in args.variants.split(','):
            if x:
                t, _, v = x.partition(':')
                tun[int(t)] = int(v) if v else 1
        plan.set_tuning(tun)
    plan.get_jk(f['dm'], hermi=1)
    st = plan.stats()
    print(json.dumps({'workload': args.config, 'ms': st['last_build_ms'], 'quartets': st['quartets'],
                      'variants': ','.join('%d:%d' % (t, v) for t, v in enumerate(plan.tuning()) if v)}))


def run_one_incore():
    import torch
    from pyscf_b200 import lib, incore
    f = dict(numpy.load(os.path.join(GOLDEN, 'mol_h2o8_vdz.npz')))
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    eri = plan.int2e_s8(device=True)
    d = torch.as_tensor(f['dm_conv'], device='cuda:0')
    for _ in range(2):
        vj, vk = incore.incore(eri, d, hermi=1)
    torch.cuda.synchronize()
    print(json.dumps({'workload': 'h2o8_vdz in-core', 'max_dJ': float(abs(vj.cpu().numpy() - f['vj_conv']).max()),
                      'max_dK': float(abs(vk.cpu().numpy() - f['vk_conv']).max())}))


def run_one_grad():
    """Plan of (H2O)16/cc-pVDZ, then one gradient J/K build and two fused force
    contractions of its density (the case profiled under ncu)."""
    from pyscf_b200 import lib
    f = dict(numpy.load(os.path.join(GOLDEN, 'grad_h2o16_vdz.npz')))
    plan = lib.Plan(f['atm'], f['bas'], f['env'], direct_scf_tol=1e-13)
    plan.grad_jk(f['dm0'])
    jk_ms = plan.grad_stats()['last_build_ms']
    for _ in range(2):
        de = plan.grad_contract(f['dm0'])
    print(json.dumps({'workload': 'h2o16_vdz gradient', 'grad_jk_ms': jk_ms,
                      'fused_force_ms': plan.grad_stats()['last_build_ms'],
                      'sum_de': float(numpy.asarray(de).sum())}))


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
    ap.add_argument('--tau', type=float, default=1e-6, help='float32 threshold of the mixed-precision line')
    ap.add_argument('--one-build', action='store_true',
                    help='plan + one FP64 J/K build of the workload, nothing else (the case profiled under ncu)')
    ap.add_argument('--one-incore', action='store_true',
                    help='fill the s8 tensor of (H2O)8/cc-pVDZ and run two in-core J/K builds, nothing else '
                         '(the case profiled under ncu)')
    ap.add_argument('--one-grad', action='store_true',
                    help='one gradient J/K build and two fused force contractions of (H2O)16/cc-pVDZ, nothing '
                         'else (the case profiled under ncu)')
    ap.add_argument('--autotune', action='store_true', help='--one-build: run the autotuner first')
    ap.add_argument('--variants', default=None,
                    help='--one-build: comma-separated class:variant pairs (a bare class index means variant 1), '
                         'as printed by --autotune')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.one_build:
        run_one_build(args)
    elif args.one_incore:
        run_one_incore()
    elif args.one_grad:
        run_one_grad()
    else:
        run_gpu(args)


if __name__ == '__main__':
    main()
