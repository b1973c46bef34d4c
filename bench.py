#!/usr/bin/env python3
"""Factor + solve benchmark of the SPR numeric phase on B200.

Workload (one step): the numeric phase of SPR on the 48^3 hex8 elasticity box
(E=1, nu=0.3, face x=0 clamped, 345,744 equations), i.e. the LDL'
factorisation of SM plus forward/diagonal/back solves of 4 right-hand sides
U[-1,1] (seed 1).  The symbolic structure is the reference's own (its MMD
ordering, supernodes and symbolic factorisation, committed as
sam_lib_b200/structures/hex48.npz); SM is assembled by the library's SPRADM
main add.  Synthetic, seeded data; no dataset is involved.

  value  : GFLOP/s of factor+solve = (RINFO(3) + NRHS*RINFO(4)) / t, with SM
           and B resident in HBM (device API), CUDA events on the engine's
           stream, max over ranks; N>1 runs independent replicas (weak).
  e2e    : the same metric through the Fortran-ABI call sprsol_(IOP=3) with
           pinned host SM and B (H2D of SM, factor, D2H of the factor into SM,
           H2D/D2H of B inside the timed region).
  --impl reference : the reference's own CPU implementation (the translated
           Fortran SPR from the oracle build) on all host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'factor+solve s & GFLOP/s, 350k-DOF hex elasticity; mixed+IR vs FP64 @1e-12'
UNIT = 'GFLOP/s'
N_MESH = 48
NRHS = 4
SAMPLE_N = 20          # bounded CPU sample: the 20^3 box of the same family


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--n', type=int, default=N_MESH)
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--case', choices=['fp64', 'mixed', 'batched'], default=None,
                    help='profiling case: only WARMUP+STEPS factorisations of the n^3 box in that mode')
    ap.add_argument('--phases', action='store_true',
                    help='with --case: CUDA events between launch groups, time by phase')
    ap.add_argument('--no-forms', action='store_true',
                    help='skip the mixed+IR, batched and adjoint measurements')
    return ap.parse_args()


def config(n=N_MESH):
    return {'workload': 'SPR numeric phase, %d^3 hex8 elasticity (E=1, nu=0.3, x=0 clamped), '
                        'LDL\' factor + %d RHS solve' % (n, NRHS),
            'mesh': '%dx%dx%d' % (n, n, n), 'nrhs': NRHS, 'rhs': 'U[-1,1] seed 1',
            'ordering': 'reference MMD + supernodes (bit-exact structure)',
            'l2': 'inputs larger than L2 (SM is %s)' % ('9.1 GB' if n == 48 else 'n^3-sized'),
            'parallelism': 'replicas'}


# ---------------------------------------------------------------------------
# CPU: the reference SPR path on a bounded sample (oracle build; baseline only)
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    n, reps = args
    from oracle.refpipe import RefSystem
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    rs = RefSystem(HexBox(n))
    ke = hex8_stiffness()
    sm0 = rs.assemble(lambda e: ke)
    b0 = np.asfortranarray(np.random.default_rng(1).uniform(-1.0, 1.0, size=(rs.neq, NRHS)))
    # RINFO(3) + NRHS * RINFO(4); RINFO(4) is already 2*sum + NEQ (sprtrs.f:2019)
    flops = float(rs.rinfo[2] + NRHS * rs.rinfo[3])
    times = []
    for _ in range(reps):
        sm = sm0.copy()
        b = b0.copy(order='F')
        t = time.perf_counter()
        ierr, _, _ = rs.sprsol(3, sm, b)
        times.append(time.perf_counter() - t)
        assert ierr == 0
    return flops, times


def cpu_sample(nproc, reps):
    """GFLOP/s of the reference SPRSOL(IOP=3) on the 20^3 sample, nproc processes."""
    import multiprocessing as mp
    if nproc == 1:
        flops, times = _cpu_worker((SAMPLE_N, reps))
        return flops, [times]
    ctx = mp.get_context('spawn')
    with ctx.Pool(nproc) as pool:
        res = pool.map(_cpu_worker, [(SAMPLE_N, reps)] * nproc)
    return res[0][0], [r[1] for r in res]


def sample_desc(cores):
    return ('reference SPRSOL IOP=3 (factor + %d-RHS solve) on the %d^3 hex8 box (26,460 eq, RINFO(3) '
            '4.37e10) of the same family, machine-translated Fortran SPR built with gcc -O2, %d process%s%s' %
            (NRHS, SAMPLE_N, cores, '' if cores == 1 else 'es',
             ' (the reference is single-threaded: one system runs on one core)' if cores == 1 else
             ', one independent system each'))


def sample_config():
    return {'workload': 'bounded sample of the %d^3 workload: the %d^3 box of the same hex8 family, LDL\' '
                        'factor + %d RHS solve' % (N_MESH, SAMPLE_N, NRHS),
            'mesh': '%dx%dx%d' % (SAMPLE_N, SAMPLE_N, SAMPLE_N), 'neq': 26460, 'nrhs': NRHS}


def _ladder_worker(n):
    """One SPRSOL IOP=1 factorisation of the n^3 box: (n, NEQ, RINFO(3), seconds)."""
    from oracle.refpipe import RefSystem
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    rs = RefSystem(HexBox(n))
    ke = hex8_stiffness()
    sm = rs.assemble(lambda e: ke)
    b = np.zeros((rs.neq, 1), order='F')
    t = time.perf_counter()
    ierr, _, _ = rs.sprsol(1, sm, b)
    dt = time.perf_counter() - t
    assert ierr == 0
    return n, rs.neq, float(rs.rinfo[2]), dt


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
             'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
             'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.QUERY,
                                       '--format=csv,noheader,nounits', '-lms', '200'],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(',') for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == 'active':
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm)}


def dgemm_peak(torch):
    """Measured cuBLAS DGEMM throughput (TFLOP/s): the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device='cuda')
    b = torch.randn(n, n, dtype=torch.float64, device='cuda')
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        a @ b
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / ms / 1e9


def tf32_peak():
    """Dense TF32 tensor peak: half the measured bf16 burst rate (tcgen05 kind::tf32
    runs at half the kind::f16 rate), else half the fallback bf16 figure."""
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(p) as f:
            bf16 = float(json.load(f)['bf16_tflops'])
        return bf16 / 2.0, 'measured bf16 burst %.1f TFLOP/s (MEASURED_PEAKS.json) / 2' % bf16
    except Exception:
        return 1590.0 / 2.0, 'fallback bf16 1590 TFLOP/s / 2'


def read_traffic():
    """dram bytes per Schur-update flop from the committed ncu summary, if any."""
    p = os.path.join(ROOT, 'profiles', 'k_gemm_traffic.txt')
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith('dram_bytes_per_flop'):
            return float(line.split('=')[1])
    return None


# ---------------------------------------------------------------------------
# the three further forms (each one timed with CUDA events on its stream)
# ---------------------------------------------------------------------------
def _ev(torch):
    return torch.cuda.Event(enable_timing=True)


def form_mixed_ir(torch, spr, n, emod, reps=2):
    """FP64 factor+solve against mixed (3xTF32 Schur updates) factor + FP64
    iterative refinement to a normwise backward error of 1e-12, same system."""
    from sam_lib_b200.adjoint import ElementOps
    from sam_lib_b200.fe import element_moduli
    from sam_lib_b200.system import HexSystem
    hs = HexSystem(n, moduli=element_moduli(n ** 3, emod, seed=2))
    ops = ElementOps(hs)
    d_sm0 = torch.empty(hs.neq + hs.nzerol, dtype=torch.float64, device='cuda')
    ops.assemble(d_sm0, torch.from_numpy(hs.ke.ravel(order='F').copy()).cuda(),
                 torch.from_numpy(hs.moduli).cuda())
    ops.close()
    ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
    st = torch.cuda.Stream()
    ds.set_stream(st.cuda_stream)
    ds.build_residual(d_sm0)
    b = torch.from_numpy(np.random.default_rng(1).uniform(-1.0, 1.0, size=(NRHS, hs.neq))).cuda()
    d_sm, x, x64 = torch.empty_like(d_sm0), torch.empty_like(b), torch.empty_like(b)
    tuned = ds.autotune(d_sm0)            # mixed-mode engine choice, timed on a copy
    out = {}
    for mode in (0, 1):
        ds.set_mode(bool(mode))
        ts = []
        for r in range(reps + 1):
            with torch.cuda.stream(st):
                d_sm.copy_(d_sm0)
            st.synchronize()
            e0, e1 = _ev(torch), _ev(torch)
            e0.record(st)
            fr = ds.factor(d_sm)
            fac_ms = ds.info()['factor_ms']
            if mode == 0:
                with torch.cuda.stream(st):
                    x64.copy_(b)
                ds.solve(d_sm, x64, NRHS)
                e1.record(st)
                e1.synchronize()
                it, berr, _ = ds.refine(d_sm, b, x, NRHS, tol=1e-12, maxit=0)
            else:
                it, berr, _ = ds.refine(d_sm, b, x, NRHS, tol=1e-12, maxit=30)
                e1.record(st)
                e1.synchronize()
            assert fr['lierr'] == 0, fr
            if r > 0:
                ts.append(e0.elapsed_time(e1))
        out[mode] = {'factor_solve_s': float(np.mean(ts)) / 1e3, 'factor_s': fac_ms / 1e3,
                     'ir_corrections': it, 'backward_error': berr, 'numneg': fr['numneg']}
    # roofline of the tensor-core update (split + k_gemm_tc launches, CUDA
    # events around each launch pair) in one more mixed factorisation
    ds.set_mode(1)
    ds.set_profile(True)
    with torch.cuda.stream(st):
        d_sm.copy_(d_sm0)
    st.synchronize()
    ds.factor(d_sm)
    tc_flops, tc_ms = ds.tc_stats()
    inf = ds.info()
    ds.set_profile(False)
    ds.set_mode(False)
    tf32_flops = 3.0 * tc_flops
    peak, src = tf32_peak()
    achieved = tf32_flops / (tc_ms / 1e3) / 1e12
    roof_tc = {'bound': 'tensor', 'kernel': 'k_split_tc + k_gemm_tc: 3xTF32 Schur update (tcgen05.mma kind::tf32, '
                                            'TMA, TMEM accumulators)',
               'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s', 'frac': achieved / peak,
               'flops': 'TF32 tensor flops = 3 products x the algorithmic flops of the tensor-core updates '
                        '(far trailing columns, next super-panels and K = S updates above the autotuned '
                        'threshold: %.4g of %.4g)' % (tc_flops, inf['gemm_flops']),
               'peak_source': src, 'time_s': tc_ms / 1e3}
    rel = float(torch.linalg.norm(x - x64) / torch.linalg.norm(x64))
    del ds
    torch.cuda.empty_cache()
    return {'system': '%d^3 hex8, E %s (seed 2), %d RHS U[-1,1] seed 1' % (
                n, 'log-uniform [1,1e4]' if emod == 'loguniform' else '= 1', NRHS),
            'fp64': out[0], 'mixed_ir': out[1], 'tol': 1e-12, 'roofline_tc': roof_tc, 'autotune': tuned,
            'speedup_mixed_ir_vs_fp64': out[0]['factor_solve_s'] / out[1]['factor_solve_s'],
            'numneg_equal': out[0]['numneg'] == out[1]['numneg'],
            'rel_diff_vs_fp64_gpu_solution': rel}


def form_mixed_vs_reference(torch, spr, n=20, emod='loguniform'):
    """Mixed + refinement against the reference's own FP64 CPU solve (the
    translated SPR SPRSOL) on a size the CPU affords: the n^3 box with the
    config-3 moduli, 4 RHS.  Reports the relative difference of the refined
    solution from the reference's, NUMNEG of both and the refinement."""
    from oracle.refpipe import RefSystem
    from sam_lib_b200.fe import HexBox, hex8_stiffness, element_moduli
    from sam_lib_b200.system import HexSystem
    moduli = element_moduli(n ** 3, emod, seed=2)
    hs = HexSystem(n, moduli=moduli)
    sm = hs.assemble()
    f = np.random.default_rng(1).uniform(-1.0, 1.0, size=(NRHS, hs.neq))
    rs = RefSystem(HexBox(n))
    ke = hex8_stiffness()
    rsm = rs.assemble(lambda e: ke * moduli[e])
    same = bool(np.array_equal(rsm, sm))                 # SPRADM and the library's assembly agree
    rb = np.asfortranarray(f.T.copy())
    t0 = time.perf_counter()
    ierr, _, rneg = rs.sprsol(3, rsm, rb)
    t_ref = time.perf_counter() - t0
    ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
    d_sm0 = torch.from_numpy(sm).cuda()
    ds.build_residual(d_sm0)
    ds.set_mode(1)
    d_sm = d_sm0.clone()
    fr = ds.factor(d_sm)
    d_b = torch.from_numpy(f).cuda()
    d_x = torch.empty_like(d_b)
    it, berr, _ = ds.refine(d_sm, d_b, d_x, NRHS, tol=1e-12, maxit=30)
    x = d_x.cpu().numpy().T
    ds.close()
    del d_sm0, d_sm, d_b, d_x
    torch.cuda.empty_cache()
    return {'system': '%d^3 hex8, E %s (seed 2), %d RHS U[-1,1] seed 1' % (n, emod, NRHS),
            'reference': 'translated SPR SPRSOL IOP=3 (FP64, 1 core, %.1f s)' % t_ref,
            'rel_diff_vs_reference_solution': float(np.linalg.norm(x - rb) / np.linalg.norm(rb)),
            'numneg': fr['numneg'], 'numneg_reference': int(rneg), 'ir_corrections': it, 'backward_error': berr,
            'same_assembled_matrix': same}


def form_batched(torch, reps=3, cpu_procs=0):
    """512 uneven shifted (indefinite) systems, 16 RHS each, as one forest."""
    from sam_lib_b200.batch import BatchSolver
    from sam_lib_b200.workloads import config4
    bs = BatchSolver(config4())
    ds = bs.ds
    st = torch.cuda.Stream()
    ds.set_stream(st.cuda_stream)
    ds.build_residual(bs.sm0)
    x = torch.empty_like(bs.b0)
    out = {'tile_autotune': ds.autotune_tiles(bs.sm0)}
    ts = []
    for r in range(reps + 1):
        with torch.cuda.stream(st):
            bs.sm.copy_(bs.sm0)
            bs.b.copy_(bs.b0)
        st.synchronize()
        e0, e1 = _ev(torch), _ev(torch)
        e0.record(st)
        fr = ds.factor(bs.sm)
        ds.solve(bs.sm, bs.b, bs.nrhs)
        e1.record(st)
        e1.synchronize()
        if r > 0:
            ts.append(e0.elapsed_time(e1))
    it, berr, _ = ds.refine(bs.sm, bs.b0, x, bs.nrhs, tol=1e-12, maxit=0)
    t = float(np.mean(ts)) / 1e3
    out['fp64'] = {'systems_per_s': bs.forest.nsys / t, 's_per_batch': t, 'backward_error': berr,
                   'numneg_total': fr['numneg'], 'indefinite_systems': int(np.count_nonzero(bs.numneg() > 0))}
    del bs, ds
    torch.cuda.empty_cache()
    out['workload'] = ('512 boxes n~U{3..12} (seed 3), K - sigma M, sigma = U[0.5,2] x lambda1, '
                       '16 RHS each, merged forest (%s)' % 'one launch per kernel per tree level')
    out['note'] = ('FP64 only: the tensor-core form changes only the Schur updates of fronts larger than 176, a '
                   'small part of these systems, and 318 of them are indefinite, so its inertia guard redoes the '
                   'factorisation in FP64')
    if cpu_procs:
        out['cpu_reference'] = batched_cpu_sample(cpu_procs)
    return out


def _batched_cpu_worker(idx):
    """Reference SPRSOL(IOP=3), 16 RHS, on systems idx of the 512-system workload (CPU)."""
    import time as _t
    from oracle.refpipe import lib as reflib, _p, _i
    import ctypes as _C
    from sam_lib_b200.workloads import config4_system_sm
    R = reflib()
    done, t = 0, 0.0
    for i in idx:
        _, _, sm, hs = config4_system_sm(i)
        sm = sm.copy()
        b = np.asfortranarray(np.random.default_rng(i).uniform(-1.0, 1.0, size=(hs.neq, 16)))
        msp = hs.mspar.copy()
        tol = np.array([1e-12, 0.0, 0.0])
        iw = np.zeros(int(hs.mspar[13]) + int(hs.mspar[12]) + 8, dtype=np.int64)
        rw = np.zeros(int(hs.mspar[16]) + int(hs.mspar[13]) + 8)
        ierr = _C.c_int64(0)
        t0 = _t.perf_counter()
        R.sprsol_(_i(3), _p(msp), _p(hs.mtrees), _p(hs.msifa), _p(sm), _p(b), _i(hs.neq), _i(16), _p(tol),
                  _p(iw), _p(rw), _i(-1), _C.byref(ierr))
        t += _t.perf_counter() - t0
        done += 1
    return done, t


def batched_cpu_sample(nproc, per_proc=8):
    """Systems/s of the reference on the 512-system workload, one process per
    host core, each factoring and solving its own share of a bounded sample
    (the first nproc*per_proc systems; sizes are drawn i.i.d., so the sample
    has the workload's size mix)."""
    import multiprocessing as mp
    n = min(512, nproc * per_proc)
    shares = [list(range(k, n, nproc)) for k in range(nproc)]
    ctx = mp.get_context('spawn')
    t0 = time.perf_counter()
    with ctx.Pool(nproc) as pool:
        res = pool.map(_batched_cpu_worker, shares)
    wall = time.perf_counter() - t0
    busy = max(r[1] for r in res)
    return {'systems_per_s': n / busy, 'unit': 'systems/s', 'cores': nproc, 'kind': 'reference',
            'sample': 'reference SPRSOL IOP=3 (16 RHS) on the first %d of the 512 systems, %d processes '
                      '(one per core, each timing its own systems; rate = systems / the slowest process time)' % (n, nproc),
            'wall_s_incl_setup': wall}


def form_batched_sharded(torch, rank, world, dist, reps=3):
    """The 512-system workload sharded over the ranks (round robin by system,
    no exchange on the data path): each rank factors and solves its share as
    one forest; the batch time is the maximum over ranks (CUDA events on each
    rank's stream)."""
    from sam_lib_b200.batch import BatchSolver
    from sam_lib_b200.replicas import max_over_ranks, shard
    from sam_lib_b200.workloads import config4
    systems = config4()
    mine = [systems[i] for i in shard(len(systems), rank, world)]
    bs = BatchSolver(mine)
    st = torch.cuda.Stream()
    bs.ds.set_stream(st.cuda_stream)
    ts = []
    for r in range(reps + 1):
        with torch.cuda.stream(st):
            bs.sm.copy_(bs.sm0)
            bs.b.copy_(bs.b0)
        st.synchronize()
        dist.barrier()
        e0, e1 = _ev(torch), _ev(torch)
        e0.record(st)
        fr = bs.ds.factor(bs.sm)
        bs.ds.solve(bs.sm, bs.b, bs.nrhs)
        e1.record(st)
        e1.synchronize()
        if r > 0:
            ts.append(e0.elapsed_time(e1))
    t = max_over_ranks(float(np.mean(ts)) / 1e3, dist, 'cuda')
    neg = bs.numneg()
    total_neg = max_over_ranks(float(neg.sum()), None)
    del bs
    torch.cuda.empty_cache()
    return {'systems_per_s': len(systems) / t, 's_per_batch': t, 'ranks': world,
            'systems_this_rank': len(mine), 'numneg_rank0': int(total_neg), 'lierr_rank0': fr['lierr'],
            'workload': '512 boxes n~U{3..12} (seed 3), K - sigma M, 16 RHS each, sharded round robin '
                        '(strong scaling: the same 512 systems for any number of ranks), FP64'}


def form_adjoint(torch, reps=3):
    """32^3 SIMP compliance: forward (assemble + factor + solve) vs forward + backward."""
    from sam_lib_b200.adjoint import SimpModel, simp_solve, simp_workload
    hs, theta, f = simp_workload(32, seed=4)
    model = SimpModel(hs)
    th = torch.tensor(theta, device='cuda', requires_grad=True)
    ft = torch.tensor(f, device='cuda')
    fw, fb = [], []
    for r in range(reps + 1):
        torch.cuda.synchronize()
        e0, e1 = _ev(torch), _ev(torch)
        e0.record()
        with torch.no_grad():
            torch.dot(ft, simp_solve(th, ft, model))
        e1.record()
        e1.synchronize()
        th.grad = None
        torch.cuda.synchronize()
        e2, e3 = _ev(torch), _ev(torch)
        e2.record()
        torch.dot(ft, simp_solve(th, ft, model)).backward()
        e3.record()
        e3.synchronize()
        if r > 0:
            fw.append(e0.elapsed_time(e1))
            fb.append(e2.elapsed_time(e3))
    res = {'workload': '32^3 hex8 SIMP E=theta^3, theta~U[0.2,1] seed 4, tip load, L = f^T u',
           'forward_s': float(np.mean(fw)) / 1e3, 'forward_backward_s': float(np.mean(fb)) / 1e3}
    res['backward_over_forward'] = res['forward_backward_s'] / res['forward_s'] - 1.0
    del model
    torch.cuda.empty_cache()
    return res


def form_assembly(torch, n=N_MESH, reps=3, ref_elements=1024):
    """Element stiffness + SPRADM on the device at n^3 (distorted mesh, seed 5;
    log-uniform moduli, seed 2), against the library's host SPRADM
    restatement (one core) and the translated reference SPRADM on a sample of
    elements (per-call ctypes overhead included).  Device SM must equal the
    host SM bit for bit."""
    import ctypes
    import sam_lib_b200 as spr
    from sam_lib_b200.adjoint import ElementOps
    from sam_lib_b200.fe import element_moduli
    from sam_lib_b200.system import HexSystem
    hs = HexSystem(n)
    box = hs.box
    ops = ElementOps(hs)
    d_xyz = torch.from_numpy(box.distorted_coords(5)).cuda()
    d_E = torch.from_numpy(element_moduli(box.nel, 'loguniform', seed=2)).cuda()
    d_em = torch.empty((box.nel, 24, 24), dtype=torch.float64, device='cuda')
    d_sm = torch.empty(hs.neq + hs.nzerol, dtype=torch.float64, device='cuda')
    flush = torch.empty(256 << 20, dtype=torch.uint8, device='cuda')
    tk, ta = [], []
    for r in range(reps + 1):
        flush.zero_()
        e0, e1, e2 = _ev(torch), _ev(torch), _ev(torch)
        e0.record()
        ops.hex8(d_xyz, d_E, 0.3, out=d_em)
        e1.record()
        ops.assemble(d_sm, d_em)
        e2.record()
        e2.synchronize()
        if r > 0:
            tk.append(e0.elapsed_time(e1))
            ta.append(e1.elapsed_time(e2))
    em = d_em.cpu().numpy().reshape(-1)
    sm = np.zeros(hs.neq + hs.nzerol)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)     # noqa: E731
    i8 = ctypes.c_int64
    t0 = time.perf_counter()
    rc = spr.load(8).spr_b200_assemble(p(hs.mspar), p(hs.mtrees), p(hs.msifa), p(hs.meqn), p(box.madof),
                                       p(box.mpmnpc), p(box.mmnpc), i8(box.nel), i8(24), p(em), None, p(sm))
    t_host = time.perf_counter() - t0
    assert rc == 0
    same = bool(np.array_equal(d_sm.cpu().numpy(), sm))
    try:
        ref = _reference_spradm_sample(ref_elements, box.nel)
    except Exception as exc:       # the reference library is test infrastructure; report its absence
        ref = {'unavailable': str(exc)[:200]}
    t_k, t_a = float(np.mean(tk)) / 1e3, float(np.mean(ta)) / 1e3
    em_bytes = 576 * 8 * box.nel
    del d_em, d_sm, d_xyz, d_E, flush, ops
    torch.cuda.empty_cache()
    return {'workload': '%d^3 hex8 box, nodes moved U[-0.15,0.15] (seed 5), E log-uniform (seed 2), nu 0.3' % n,
            'elements': box.nel, 'hex8_s': t_k, 'assemble_s': t_a, 'device_s': t_k + t_a,
            'hex8_write_gbs': em_bytes / t_k / 1e9, 'host_restatement_s': t_host,
            'host_over_device': t_host / (t_k + t_a), 'device_sm_equals_host_sm': same,
            'reference_spradm': ref}


def _reference_spradm_sample(count, nel_full, n=12):
    """The translated reference SPRADM, one call per element for the first
    `count` elements of the n^3 box (its symbolic inputs from the reference
    pipeline; the per-element work does not depend on the mesh size):
    seconds per element, and that rate times nel_full."""
    import ctypes
    from oracle.refpipe import RefSystem, lib, _p, _i
    from sam_lib_b200.fe import HexBox, hex8_stiffness
    L = lib()
    b = HexBox(n)
    rs = RefSystem(b)
    sm = np.zeros(rs.neq + rs.nzerol)
    sv = np.zeros(1)
    tt = np.zeros(1)
    iw = np.zeros(int(rs.mspar[38]) + 64, dtype=np.int64)
    ierr = ctypes.c_int64(0)
    ke = np.asfortranarray(hex8_stiffness())
    count = min(count, b.nel)
    t0 = time.perf_counter()
    for e in range(count):
        L.spradm_(_p(ke), _p(tt), _p(rs.mpar), _p(rs.mspar), _p(b.madof), _p(rs.meqn), _p(b.mpmnpc),
                  _p(b.mmnpc), _p(b.mpmceq), _p(b.mmceq), _p(rs.msica), _p(rs.mtrees), _p(rs.msifa),
                  _p(rs.mdofnc), _p(sm), _p(sv), _p(iw), _i(e + 1), _i(24), _i(-1), _i(0), ctypes.byref(ierr))
    dt = time.perf_counter() - t0
    return {'elements_timed': count, 'mesh': '%d^3' % n, 's_per_element': dt / count,
            'extrapolated_s': dt / count * nel_full,
            'note': 'one SPRADM call per element through ctypes (call overhead included), 1 core; '
                    'element matrices formed beforehand (not timed)'}


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    """The reference's own CPU implementation of the path (the machine-translated
    SPR Fortran) on this host.  The reference is single-threaded and has no way
    to spread one system over cores, so `value` is its rate on one core; each
    step is one SPRSOL(IOP=3) of the bounded 20^3 sample (about 5-7 s).  Also
    reported: a size ladder (one factorisation each of 12^3..24^3, so that the
    rate's size dependence is visible before anyone extrapolates it to 48^3),
    the RINFO(3)-based extrapolation to the 48^3 factorisation, and the
    all-core aggregate of independent sample systems (one process per core)."""
    if rank != 0:
        return
    ladder = []
    for n in (12, 16, 20, 24):
        nn, neq, r3, dt = _ladder_worker(n)
        ladder.append({'mesh': '%d^3' % nn, 'neq': neq, 'rinfo3': r3, 'factor_s': dt,
                       'gflops': r3 / dt / 1e9})
    flops, times = cpu_sample(1, args.warmup + args.steps)
    per_step = times[0][args.warmup:]
    t = float(np.mean(per_step))
    value = flops / t / 1e9
    nproc = os.cpu_count() or 1
    agg_flops, agg_times = cpu_sample(nproc, 1)
    agg = nproc * agg_flops / max(tt[0] for tt in agg_times) / 1e9
    rinfo3_48 = 1.419e13
    line = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': args.gpus,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': t * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded hex8 meshes)',
            'config': config(args.n), 'sample_config': sample_config(),
            'cpu_baseline': {'value': value, 'unit': UNIT, 'cores': 1, 'kind': 'reference',
                             'sample': sample_desc(1)},
            'e2e': {'value': value, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
            'ladder': ladder,
            'extrapolated_48_factor_s': rinfo3_48 / (value * 1e9),
            'extrapolation_note': '48^3 RINFO(3) 1.419e13 at the 1-core sample rate; the ladder shows the '
                                  'rate at 12^3..24^3, the 48^3 top fronts are larger still',
            'aggregate_all_cores': {'value': agg, 'unit': UNIT, 'cores': nproc,
                                    'sample': sample_desc(nproc),
                                    'note': 'independent systems only; not a rate for one system'},
            'host_cpu': _cpu_model()}
    print(json.dumps(line), flush=True)


def _cpu_model():
    try:
        for line in open('/proc/cpuinfo'):
            if line.startswith('model name'):
                return line.split(':', 1)[1].strip()
    except OSError:
        pass
    return None


def run_ours(args, rank, world, local_rank):
    from sam_lib_b200.replicas import max_over_ranks, whole_job_rate
    # CPU baseline first (rank 0, N=1 only), before the GPU is touched
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        flops_s, times = cpu_sample(1, 1)
        t = times[0][0]
        cpu = {'value': flops_s / t / 1e9, 'unit': UNIT, 'cores': 1, 'kind': 'reference',
               'sample': sample_desc(1), 'sample_s': t}
    import torch
    import sam_lib_b200 as spr
    from sam_lib_b200.system import HexSystem
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    hs = HexSystem(args.n)
    sm = hs.assemble()
    neq, nzerol = hs.neq, hs.nzerol
    f = np.random.default_rng(1).uniform(-1.0, 1.0, size=(NRHS, neq))
    ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
    stream = torch.cuda.Stream()
    ds.set_stream(stream.cuda_stream)
    d_sm0 = torch.from_numpy(sm).cuda()
    d_sm = torch.empty_like(d_sm0)
    d_b0 = torch.from_numpy(f).cuda()
    d_b = torch.empty_like(d_b0)
    info = ds.info()
    flops = info['factor_flops'] + NRHS * info['solve_flops']

    def step(timed):
        with torch.cuda.stream(stream):
            d_sm.copy_(d_sm0)
            d_b.copy_(d_b0)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = ds.factor(d_sm)
        ds.solve(d_sm, d_b, NRHS)
        e1.record(stream)
        e1.synchronize()
        assert r['lierr'] == 0 and r['numneg'] == 0, r
        inf = ds.info()
        return e0.elapsed_time(e1), inf

    for _ in range(args.warmup):
        step(False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    times, fac_ms, sol_ms, launches = [], [], [], 0
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        ms, inf = step(True)
        times.append(ms)
        fac_ms.append(inf['factor_ms'])
        sol_ms.append(inf['solve_ms'])
        launches += int(inf['launches'] + inf['solve_launches'])
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    # one more step, untimed, in profile mode: CUDA events around every
    # Schur-update launch and between the launch groups of the factorisation
    ds.set_profile(True)
    prof_ms, inf = step(False)
    gemm_ms = [inf['gemm_ms']]
    phases = ds.phase_ms()
    ds.set_profile(False)
    ms_step = max_over_ranks(float(np.mean(times)), dist, 'cuda')
    value = whole_job_rate(flops, world, ms_step / 1e3) / 1e9
    # accuracy of the last step: ||K x - f|| / ||f|| per RHS
    x = d_b.cpu().numpy()
    res = [float(np.linalg.norm(hs.matvec(x[r]) - f[r]) / np.linalg.norm(f[r])) for r in range(NRHS)]
    # end to end through the Fortran ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        sm_pin0 = torch.from_numpy(sm).pin_memory()
        sm_pin = torch.empty(sm.shape, dtype=torch.float64, pin_memory=True)
        b_pin0 = torch.from_numpy(f.copy()).pin_memory()           # (NRHS, NEQ) == B(NEQ, NRHS)
        b_pin = torch.empty(f.shape, dtype=torch.float64, pin_memory=True)
        mspar = hs.mspar.copy()
        e2e_t = []
        for k in range(1 + min(args.steps, 3)):
            sm_pin.copy_(sm_pin0)
            b_pin.copy_(b_pin0)
            smv, bv = sm_pin.numpy(), b_pin.numpy().T
            tol = np.array([1.0e-12, 0.0, 0.0])
            mspar[:] = hs.mspar
            t = time.perf_counter()
            ierr = spr.sprsol(3, mspar, hs.mtrees, hs.msifa, smv, bv, neq, NRHS, tol)
            dt = time.perf_counter() - t
            assert ierr == 0, ierr
            if k > 0:                 # the first call also builds the context (plan, buffers)
                e2e_t.append(dt)
        cs = np.zeros(3)
        spr.load(8).spr_b200_copy_stats(cs.ctypes.data_as(__import__('ctypes').c_void_p))
        spr.release_all()
        xe = b_pin.numpy()
        assert np.allclose(xe, x, rtol=1e-9, atol=1e-12)
        te = max_over_ranks(float(np.mean(e2e_t)), dist, 'cuda')
        bytes_io = 8 * (neq + nzerol) + 8 * neq * NRHS
        e2e = {'value': whole_job_rate(flops, world, te) / 1e9, 'unit': UNIT, 'h2d_bytes_per_step': bytes_io,
               'd2h_bytes_per_step': bytes_io, 's_per_step': te,
               'copies': {'upload_before_factor_ms': cs[0], 'factor_ms': cs[1], 'download_after_factor_ms': cs[2],
                          'note': 'last step: SM is pinned, so LNZ goes up and comes back level group by level '
                                  'group while the factorisation runs; these are the parts not overlapped'}}
    peak = dgemm_peak(torch)
    gemm_s = float(np.mean(gemm_ms)) / 1e3
    achieved = info['gemm_flops'] / gemm_s / 1e12
    tpf = read_traffic()
    launches_per_step = inf['gemm_launches']
    roof = {'bound': 'tensor', 'achieved': achieved, 'peak': peak, 'unit': 'TFLOP/s',
            'frac': achieved / peak,
            'traffic': (tpf * info['gemm_flops'] / launches_per_step) if tpf else None,
            'kernel': 'k_gemm: FP64 Schur update C -= L D L\' (mma.sync m8n8k4 f64)',
            'flops_per_launch': info['gemm_flops'] / launches_per_step,
            'peak_source': 'measured in-run: cuBLAS DGEMM 8192^3 via torch.matmul float64 '
                           '(MEASURED_PEAKS.json has no FP64 figure)',
            'time_share': gemm_s / (prof_ms / 1e3),
            'timing': 'Schur-update launches timed with CUDA events in one extra profiled step (%.1f ms)' % prof_ms}
    del ds, d_sm0, d_sm, d_b0, d_b
    torch.cuda.empty_cache()
    forms = None
    if world > 1 and not args.no_forms:
        # every rank takes part (the same collective steps on all ranks)
        bs = form_batched_sharded(torch, rank, world, dist)
        if rank == 0:
            forms = {'batched_sharded': bs}
    if rank == 0 and world == 1 and not args.no_forms and args.n == N_MESH:
        forms = {'mixed_ir_vs_reference_cpu': form_mixed_vs_reference(torch, spr),
                 'mixed_ir_loguniform': form_mixed_ir(torch, spr, N_MESH, 'loguniform'),
                 'mixed_ir_uniform': form_mixed_ir(torch, spr, N_MESH, 'uniform'),
                 'batched': form_batched(torch, cpu_procs=os.cpu_count() or 1), 'adjoint': form_adjoint(torch),
                 'assembly': form_assembly(torch)}
    if rank == 0:
        line = {'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': args.steps,
                'warmup': args.warmup, 'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'weak',
                'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded hex8 mesh, reference structure)',
                'config': config(args.n),
                'factor_s': float(np.mean(fac_ms)) / 1e3, 'solve_s': float(np.mean(sol_ms)) / 1e3,
                'factor_solve_s': ms_step / 1e3, 'factor_flops': info['factor_flops'],
                'solve_flops_per_rhs': info['solve_flops'], 'residual': max(res),
                'roofline': roof, 'factor_phase_ms': phases, 'cpu_baseline': cpu, 'e2e': e2e,
                'gpu_launches': launches,
                'clocks': clocks, 'wall_s_timed': t_wall, 'forms': forms}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_case(args):
    """Factorisations only (no solve, e2e, CPU leg or forms): the command the
    committed ncu summaries were captured with."""
    import torch
    import sam_lib_b200 as spr
    if args.case == 'batched':
        from sam_lib_b200.batch import BatchSolver
        from sam_lib_b200.workloads import config4
        bs = BatchSolver(config4())
        ds, d_sm0, nrhs, neq = bs.ds, bs.sm0, bs.nrhs, bs.forest.neq
    else:
        from sam_lib_b200.system import HexSystem
        hs = HexSystem(args.n)
        ds = spr.DeviceSolver(hs.mspar, hs.mtrees, hs.msifa)
        d_sm0 = torch.from_numpy(hs.assemble()).cuda()
        nrhs, neq = NRHS, hs.neq
    st = torch.cuda.Stream()
    ds.set_stream(st.cuda_stream)
    ds.set_mode(1 if args.case == 'mixed' else 0)
    ds.set_profile(args.phases)
    d_sm = torch.empty_like(d_sm0)
    ms = []
    for k in range(args.warmup + args.steps):
        with torch.cuda.stream(st):
            d_sm.copy_(d_sm0)
        st.synchronize()
        r = ds.factor(d_sm)
        assert r['lierr'] == 0, r
        if k >= args.warmup:
            ms.append(ds.info()['factor_ms'])
    line = {'case': args.case, 'n': args.n, 'factor_ms': ms}
    if args.phases:
        b = torch.from_numpy(np.random.default_rng(1).uniform(-1.0, 1.0, size=(nrhs, neq))).cuda()
        ds.solve(d_sm, b, nrhs)
        line['solve_ms'] = ds.info()['solve_ms']
    if args.phases:
        line['phase_ms'] = ds.phase_ms()
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.case:
        run_case(args)
        return
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local_rank = int(os.environ.get('LOCAL_RANK', '0'))
    if args.impl == 'reference':
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == '__main__':
    main()
