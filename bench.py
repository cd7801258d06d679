"""Benchmark: tangent-linear + adjoint gradients per second of the MPAS shallow-water RK4 model.

Workload (default): level-7 bisected-icosahedron TRiSK mesh (163842 cells, 491520 edges, 327680
vertices), seeded balanced flow (seed 0) over 8 seeded mountains (h reduced by the topography),
dt = 75 s, a 288-step (6 h) window, trajectory checkpointed every 16 steps, perturbations
h' ~ N(0, 1 m), u' ~ N(0, 0.1 m/s), B = 64 members.  One bench step is one gradient batch:
the nonlinear window with checkpoints, the B-member tangent-linear sweep and the B-member
adjoint sweep (seeded with the tangent-linear output, i.e. the gradient of 1/2 |L dx|^2).
`value` counts gradients of the batched FP32-stencil / FP64-accumulation form; the plain FP64
single-member form is timed beside it, with the relative L2 error of the batched result against
the FP64 window.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--batch B]
                  [--level L] [--nsteps T]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'mpas-sw-tl-ad_b200'))

METRIC = 'TL+AD gradients/s, batched FP32 vs plain FP64 (rel err<=1e-4)'
UNIT = 'gradients/s'
KERNELS = ['tl_vertex', 'tl_cell', 'tl_edge_diag', 'tl_edge_tend', 'ad_edge', 'ad_cell',
           'ad_vertex', 'ad_final', 'tl_stage', 'ad_stage']


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=3)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='mpsw', choices=['mpsw', 'reference'])
    p.add_argument('--workload', default='tlad', choices=['tlad', 'fwd', 'costs', 'long'],
                   help='tlad: batched TL+AD gradients (level 7, 288 steps of 75 s, B=64); '
                        'fwd: nonlinear forward with mountains (level 7, 1152 steps of 75 s), sim-days/s; '
                        'costs: 64 cost-function gradients by one batched adjoint (level 6, 1152 steps of 150 s); '
                        'long: TL+AD gradients over a day on level 8 (2160 steps of 40 s, B=16) with binomial '
                        'checkpointing of 32 snapshots')
    p.add_argument('--batch', type=int, default=None)
    p.add_argument('--snapshots', type=int, default=None, help='binomial checkpointing snapshots (long: 32)')
    p.add_argument('--level', type=int, default=None)
    p.add_argument('--nsteps', type=int, default=None)
    p.add_argument('--dt', type=float, default=None)
    p.add_argument('--ckpt', type=int, default=16)
    p.add_argument('--storage', type=int, default=-1,
                   help='stage storage mode of the window: -1 auto, 0 checkpoints only, 1 FP64, 2 FP32, 3 both')
    p.add_argument('--no-plain', action='store_true', help='skip the plain FP64 arm')
    p.add_argument('--profile-kernels', action='store_true',
                   help='one small window, then each member kernel once (twice with its warm-up) inside '
                        'the NVTX range "mpsw_kernels", as mpsw_time_kernel launches them; no JSON line')
    p.add_argument('--profile', action='store_true',
                   help='only the timed batched windows (for profiler launch lists); no JSON line')
    a = p.parse_args()
    dflt = {'tlad': (7, 288, 75.0), 'fwd': (7, 1152, 75.0), 'costs': (6, 1152, 150.0), 'long': (8, 2160, 40.0)}[a.workload]
    a.batch = a.batch or (16 if a.workload == 'long' else 64)
    a.snapshots = (32 if a.workload == 'long' else 0) if a.snapshots is None else a.snapshots
    a.level = dflt[0] if a.level is None else a.level
    a.nsteps = dflt[1] if a.nsteps is None else a.nsteps
    a.dt = dflt[2] if a.dt is None else a.dt
    return a


def workload(level, dt):
    """Seeded balanced flow (config-0 initial condition) loaded through the module surface."""
    import numpy as np
    from mpsw import ic
    from mpsw.mesh import icosahedral_mesh
    unit = icosahedral_mesh(level)
    mesh = ic.scale_mesh(unit)
    st = ic.balanced_flow(mesh, seed=0)
    return unit, mesh, st


def load_module(mod, unit, mesh, st, dt):
    import numpy as np
    mod.nvertlevels = 1
    mod.ncells, mod.nedges, mod.nvertices = unit['nCells'], unit['nEdges'], unit['nVertices']
    mod.maxedges, mod.maxedges2, mod.vertexdegree = unit['maxEdges'], unit['maxEdges2'], unit['vertexDegree']
    mod.r3 = 3
    mod.ntracers = 1
    mod.var_allocation()
    mod.on_a_sphere = True
    for k in ('latCell', 'lonCell', 'xCell', 'yCell', 'zCell', 'latEdge', 'lonEdge', 'xEdge',
              'yEdge', 'zEdge', 'latVertex', 'lonVertex', 'xVertex', 'yVertex', 'zVertex',
              'cellsOnEdge', 'nEdgesOnCell', 'nEdgesOnEdge', 'edgesOnCell', 'edgesOnEdge',
              'weightsOnEdge', 'dvEdge', 'dcEdge', 'angleEdge', 'areaCell', 'areaTriangle',
              'cellsOnCell', 'verticesOnCell', 'verticesOnEdge', 'edgesOnVertex', 'cellsOnVertex',
              'kiteAreasOnVertex', 'meshDensity'):
        setattr(mod, k.lower(), np.asarray(mesh[k]).T)
    mod.fvertex = st['fVertex']
    mod.fedge = st['fEdge']
    mod.u[0, 0] = st['u']
    mod.h[0, 0] = st['h']
    mod.config_dt = dt
    mod.config_test_case = 7
    mod.config_apvm_upwinding = 0.5


def perturbations(unit, B, seed=1):
    from mpsw import ic
    return ic.perturbation(unit, seed, count=B)


# ---- reference arm and CPU baseline: the oracle (serial C restatement of the Fortran) -------
class OracleMember:
    """One member's oracle instance on the host: the workload's mesh, balanced flow over
    mountains and a seeded perturbation, built once; sample(n) times n forward, n
    tangent-linear and n adjoint steps."""

    def __init__(self, level, dt, seed):
        sys.path.insert(0, os.path.join(ROOT, 'oracle'))
        import oracle as O
        m = O.OracleModule()
        unit = forward_module(m, level, dt)
        m.var_allocation_tlm()
        m.var_allocation_adj()
        m.sw_mpas_init_block()
        dh, du = perturbations(unit, 1, seed)
        self.m, self.du, self.dh = m, du[:, 0].copy(), dh[:, 0].copy()
        self.u0, self.h0 = m.u[0, 0].copy(), m.h[0, 0].copy()

    def sample(self, n):
        """Seconds per step of the forward, tangent-linear and adjoint sweeps (n steps each)."""
        m = self.m
        m.u[0, 0], m.h[0, 0] = self.u0, self.h0
        m.u_tl[0, 0], m.h_tl[0, 0] = self.du, self.dh
        t0 = time.perf_counter()
        for _ in range(n):
            m.sw_rk4()
        t1 = time.perf_counter()
        m.u[0, 0], m.h[0, 0] = self.u0, self.h0
        for _ in range(n):
            m.sw_rk4_tlm()
        t2 = time.perf_counter()
        m.u_ad[0, 0], m.h_ad[0, 0] = m.u_tl[0, 0], m.h_tl[0, 0]
        for _ in range(n):
            m.u[0, 0], m.h[0, 0] = self.u0, self.h0
            m.sw_rk4_adj()
        t3 = time.perf_counter()
        return (t1 - t0) / n, (t2 - t1) / n, (t3 - t2) / n


def _oracle_worker(conn, level, dt, seed):
    """Host process of the reference arm: builds its member once, then runs one sample per
    request (n steps of each sweep) and answers with the per-step seconds."""
    try:
        om = OracleMember(level, dt, seed)
        conn.send('ready')
        while True:
            n = conn.recv()
            if n is None:
                break
            conn.send(om.sample(n))
    except Exception as e:  # reported to the parent, which raises
        conn.send('error: %r' % (e,))


class OracleWorkers:
    """`count` host processes (spawned, before any GPU use), each with its own member; one
    bench step sends every process one sample request at once and waits for all answers."""

    def __init__(self, count, level, dt):
        import multiprocessing as mp
        ctx = mp.get_context('spawn')
        self.procs, self.conns = [], []
        for i in range(count):
            a, b = ctx.Pipe()
            p = ctx.Process(target=_oracle_worker, args=(b, level, dt, 1 + i), daemon=True)
            p.start()
            self.procs.append(p)
            self.conns.append(a)
        for c in self.conns:
            r = c.recv()
            if r != 'ready':
                raise RuntimeError('oracle worker failed: %s' % r)

    def step(self, n):
        """One sample on every process at once: (wall seconds, per-process per-step seconds)."""
        t0 = time.perf_counter()
        for c in self.conns:
            c.send(n)
        per = [c.recv() for c in self.conns]
        wall = time.perf_counter() - t0
        bad = [r for r in per if isinstance(r, str)]
        if bad:
            raise RuntimeError('oracle worker failed: %s' % bad[0])
        return wall, per

    def close(self):
        for c in self.conns:
            try:
                c.send(None)
            except Exception:
                pass
        for p in self.procs:
            p.join(timeout=10)


def run_reference(a, rank, world):
    """The reference's CPU path (the serial oracle, one member per host process on every host
    core at once).  One bench step is one sample: each process runs one forward, one
    tangent-linear and one adjoint step of its member; `ms_per_step` is that sample's wall time
    and `value` the gradients per second it implies for the full window (linear in steps)."""
    if rank != 0:  # rank 0 alone times the host baseline; other ranks exit without work
        return
    workers = os.cpu_count() or 1
    pool = OracleWorkers(workers, a.level, a.dt)
    try:
        for _ in range(a.warmup):
            pool.step(1)
        walls, grads = [], []
        for _ in range(a.steps):
            wall, per = pool.step(1)
            walls.append(wall)
            step_s = max(f + t + d for f, t, d in per)  # the slowest process's fwd + TL + AD step
            grads.append(workers / (step_s * a.nsteps))
    finally:
        pool.close()
    v = statistics.median(grads)
    ms = 1e3 * statistics.mean(walls)
    line = {
        'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': UNIT, 'n_gpus': a.gpus,
        'steps': a.steps, 'warmup': a.warmup, 'ms_per_step': ms,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic (seeded balanced flow over 8 seeded mountains, level-%d TRiSK mesh)' % a.level,
        'config': workload_config(a),
        'sample_ms': [round(1e3 * w, 1) for w in walls],
        'extrapolation': {'steps_per_sample': 1, 'window_steps': a.nsteps,
                          'seconds_per_gradient_per_process': workers / v,
                          'note': 'value = processes / (slowest process fwd+TL+AD step seconds x window steps)'},
        'cpu_baseline': {'value': v, 'unit': UNIT, 'cores': workers, 'kind': 'port',
                         'sample': '1 forward + 1 TL + 1 AD step per process on %d processes, extrapolated to %d steps' % (workers, a.nsteps)},
        'e2e': {'value': v, 'unit': UNIT, 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def cpu_gradient_seconds(level, dt, nsteps, target_s=15.0):
    """Seconds per gradient of the serial reference restatement on one host core, from a bounded
    sample (about target_s seconds of host work) extrapolated to the window; and the sample's
    step count."""
    om = OracleMember(level, dt, 1)
    f, t, d = om.sample(1)
    n = max(1, min(30, int(target_s / max(f + t + d, 1e-6)) - 1))
    f, t, d = om.sample(n)
    return (f + t + d) * nsteps, n


def workload_config(a):
    """`config` of the TL+AD bench line (both arms)."""
    nC = 10 * 4 ** a.level + 2
    return {'workload': 'TL+AD window: level-%d mesh (%d cells), %d RK4 steps of %g s, %d members, checkpoint every %d'
                        % (a.level, nC, a.nsteps, a.dt, a.batch, a.ckpt),
            'members_per_gpu': a.batch, 'parallelism': 'replicas x%d' % a.gpus,
            'l2': 'GPU arm: flushed (256 MB write) between timed steps; working set far above L2'}


# ---- host jitter ----------------------------------------------------------------------------------
class host_quiet:
    """Python's cyclic garbage collector paused over the timed steps (after one collection and
    with the set-up's objects frozen), so a full collection cannot stall the host thread that
    feeds the GPU in the middle of a timed step.  close() restores it."""

    def __init__(self):
        import gc
        self.gc = gc
        gc.collect()
        gc.freeze()
        self.was = gc.isenabled()
        gc.disable()

    def close(self):
        if self.was:
            self.gc.enable()
        self.gc.unfreeze()


# ---- clocks -------------------------------------------------------------------------------------
class Clocks:
    FIELDS = 'index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap'

    def __init__(self, index):
        self.index = index
        self.proc = None
        # the raw samples; MPSW_CLOCKS_DIR keeps them somewhere chosen by the caller
        out = os.environ.get('MPSW_CLOCKS_DIR') or tempfile.gettempdir()
        self.path = os.path.join(out, 'mpsw_clocks_%d.csv' % os.getpid())

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + self.FIELDS,
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()
            self.f.close()

    def summary(self):
        if not self.proc:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for line in open(self.path):
            parts = [x.strip() for x in line.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(n)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': mx, 'reasons': sorted(reasons), 'samples': len(sm)}


# ---- algorithmic bytes of the member kernels ------------------------------------------------------
def kernel_bytes(name, nC, nE, nV, sum_eoe, B, s):
    """Bytes a launch must move if every array element it touches is read or written once
    (viscosity, drag and wind off, as in the benchmark workload: the sweeps then neither write
    divergence' / vorticity' nor form divergence_ad, which feed only the viscosity terms).

    s: bytes of a member value, a linearisation-point value and a mesh metric (4 in FP32);
    accumulators and member RK states are a = 8 bytes; connectivity words 4 bytes, edge signs
    1 byte.  E, C, V: edges, cells, vertices.  RK bookkeeping of a middle stage, as the sweeps
    and mpsw_time_kernel run it, reads the step's input state (FP32 members: its rounding, s
    bytes; FP64: x0 itself) and writes the next provisional state and the stage's tendency
    (3 s per member value); ad_final likewise reads x2 (rounded for FP32 members) and writes the
    next tendency adjoint and its stage contribution (3 s)."""
    a, i, E, C, V, S = 8, 4, nE, nC, nV, sum_eoe
    eoe = i * (E + S) + s * S                              # nEdgesOnEdge, edgesOnEdge, weights
    kb = {
        'tl_vertex': (3 * i + 3 + 3 * i + 3 * s) * V + 2 * s * V + s * E   # v_es,esg,v_c,kites; area,f; dc
                     + 2 * s * V                                          # base h_vertex, vorticity
                     + B * s * (E + C + V),                               # u,h in; pv out
        'tl_cell': (i + 3 * 6 * i + 6 + 6 * s + s) * C + (2 * i + 2 * s) * E  # c_n,es,eoc,vs,esg,kites,area; c1,c2,dc,dv
                   + 2 * s * E                                                  # base u, h_edge
                   + B * (s * (E + C + V + 2 * C) + 3 * s * C),                # u,h,pv in; ke,pc out; RK
        'tl_edge_diag': eoe + (6 * i + 2 * s) * E + 4 * s * E                  # ends; dc,dv; base gradPVt,v,gradPVn,u
                        + (2 * s * E if s == 4 else 0)                         # FP32: base h_edge, pv_edge
                        + B * s * (E + C + V + C + 2 * E)                      # u,h,pv,pc in; pv_edge,h_edge out
                        + (B * s * E if s == 4 else 0),                        # FP32: h_edge -> u h_edge, + PV flux
        'tl_edge_tend': eoe + (2 * i + s) * E + 3 * s * E                      # c1,c2,dc; base pv_edge,u,h_edge
                        + B * (s * (3 * E + 2 * C) + 3 * s * E),               # u,pe,he,ke,h in; RK
        'ad_edge': eoe + s * S + (2 * i + s) * E + 6 * s * E                   # wrev; c1,c2,dv; 6 base fields
                   + B * s * (E + C + 3 * E),                                  # tu,th in; pe_ad,he_ad,ud out
        'ad_cell': (i + 6 * i + 6 + s) * C + 2 * s * E                         # c_n,es,esg,area; dc; base u
                   + B * s * (3 * E + 3 * C),                                  # tu,pe_ad,he_ad in; 3 out
        'ad_vertex': (3 * i + 3 * s + 3 * i + 3 * i + 3 + 2 * s) * V + s * C + 2 * s * E + 2 * s * V
                     + B * s * (C + E + 2 * V),                                # pc_ad,pe_ad in; 2 out
        'ad_final': (i + 6 * i + 6 * s + s) * C + i * (E + S) + s * S + (4 * i + 2 * s) * E + 2 * s * E
                    + B * (s * (C + 2 * V + 2 * E + C) + 3 * s * (C + E)),
    }
    kb['tl_stage'] = sum(kb[k] for k in ('tl_vertex', 'tl_cell', 'tl_edge_diag', 'tl_edge_tend'))
    kb['ad_stage'] = sum(kb[k] for k in ('ad_edge', 'ad_cell', 'ad_vertex', 'ad_final'))
    return kb[name]


def fused_bytes(name, nC, nE, nV, B, s=4, a=8):
    """Bytes a fused stage launch must move (a middle stage as the sweeps and mpsw_time_kernel run
    it; default physics): every mesh coefficient, linearisation-point value and member value it
    touches, once.  Members: the stage's inputs (s), and the RK bookkeeping, which reads the
    step's rounded input state (s) and writes the next provisional state and the stage's tendency
    (tangent linear) or its contribution and the next tendency adjoint (adjoint) (2 s): 4 s per
    member value.
    Mesh, tangent linear: vertex 3+3 coefficients and f, cell 3 x 6 coefficients, edge 10 weights
    and two reciprocals; adjoint: both weight lists, dvEdge, dcEdge, cell 3 x 6 coefficients and
    areaCell, vertex 2 x 3 coefficients, areaTriangle and f.  Base: 6 edge and 2 vertex fields."""
    E, C, V = nE, nC, nV
    mesh = s * (7 * V + 18 * C + 12 * E) if name == 'tl_stage' else s * (22 * E + 19 * C + 8 * V)
    base = s * (6 * E + 2 * V)
    return mesh + base + B * (E + C) * 4 * s


def model_stage_bytes(nC, nE, nV, sum_eoe, B, s=4, a=8):
    """The per-stage bytes M + B S of the path's algorithmic model: mesh read once per stage and,
    per member, x_k read and x_k+1 written at s, x0 read and the accumulator read and written at
    a: S = (N + E)(2 s + 3 a)."""
    E, N, V, S = nE, nC, nV, sum_eoe
    mesh = 4 * (2 * E + 2 * E + S + E + 2 * E + N + 3 * V + 3 * V) + s * (S + 2 * E + 2 * N + 3 * V + 2 * V)
    return mesh + B * (N + E) * (2 * s + 3 * a)


def traffic_of(kernel, level, B):
    """DRAM bytes (read + write) of one launch of `kernel`, from the committed ncu summary of
    that kernel on this workload (profiles/k_<kernel>_l<level>_b<B>_fp32.md: the read and write
    sums, or the bytes derived from the DRAM rate and the duration), or None."""
    import re
    path = os.path.join(ROOT, 'profiles', 'k_%s_l%d_b%d_fp32.md' % (kernel, level, B))
    if not os.path.exists(path):
        return None
    unit = {'byte': 1, 'Kbyte': 1e3, 'Mbyte': 1e6, 'Gbyte': 1e9}
    total, found = 0.0, 0
    derived = None
    for line in open(path):
        m = re.search(r'dram__bytes_(read|write)\.sum`?\)?\s*\|\s*([0-9.]+)\s*(\w+)', line)
        if m and m.group(3) in unit:
            total += float(m.group(2)) * unit[m.group(3)]
            found += 1
        # captures with sections only: bytes = dram__bytes.sum.per_second x duration
        m = re.search(r'derived \(`dram__bytes\.sum\.per_second` . `gpu__time_duration\.sum`\)\s*\|\s*([0-9.]+)\s*(\w+)', line)
        if m and m.group(2) in unit:
            derived = float(m.group(1)) * unit[m.group(2)]
    return total if found == 2 else derived


def run_mpsw(a, rank, world):
    import numpy as np
    import torch
    from module_sw_mpas import MpasSwModule
    from mpsw import _lib
    from mpsw import replicas
    from mpsw.torch_api import FP32, FP64, Engine, Window

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    mod = MpasSwModule()
    unit = forward_module(mod, a.level, a.dt)
    mod.var_allocation_tlm()
    mod.var_allocation_adj()
    mod.sw_mpas_init_block()
    eng = Engine(mod)
    L = _lib.load()
    B = a.batch
    nC, nE, nV = unit['nCells'], unit['nEdges'], unit['nVertices']
    dh_h, du_h = perturbations(unit, B, seed=replicas.member_seed(1, rank))
    du = torch.tensor(du_h, device='cuda')
    dh = torch.tensor(dh_h, device='cuda')
    du_i, dh_i = eng.to_internal(du, 1), eng.to_internal(dh, 0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')

    def gradient_batch(prec, Bm, u0, h0, ev=None):
        """One bench step on device-resident members: window, TL, AD seeded with the TL output.
        With `ev` (four CUDA events) the phase boundaries are recorded on the stream."""
        rec = (lambda i: ev[i].record(stream)) if ev else (lambda i: None)
        rec(0)
        w = Window(eng, a.nsteps, a.ckpt, a.storage)
        xu, xh = u0.clone(), h0.clone()
        rec(1)
        w.tl_internal(xu, xh, prec)
        rec(2)
        w.ad_internal(xu, xh, prec)
        rec(3)
        return xu, xh

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, n_warm, n_time):
        for _ in range(n_warm):
            fn()
        times = []
        launches0 = L.mpsw_launch_count()
        quiet = host_quiet()
        for _ in range(n_time):
            flush.zero_()  # L2 flush between timed iterations, outside the timed region
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            barrier()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            times.append(e0.elapsed_time(e1))
        quiet.close()
        return times, (L.mpsw_launch_count() - launches0) / n_time

    if world > 1:
        import torch.distributed as dist
        dist.barrier()

    # batched FP32 stencils / FP64 accumulation: the headline
    if a.profile_kernels:
        import ctypes
        gradient_batch(FP32, B, du_i, dh_i)
        torch.cuda.synchronize()
        fm, fk = ctypes.c_int(), ctypes.c_int()
        eng.h.check(L.mpsw_window_fused(eng.h.ptr, FP32, B, ctypes.byref(fm), ctypes.byref(fk)), 'window_fused')
        # the kernels the sweeps launch: the two fused stages (8, 9) or the eight split kernels
        which = [8, 9] if fm.value else list(range(len(KERNELS) - 2))
        torch.cuda.nvtx.range_push('mpsw_kernels')
        for i in which:
            out = ctypes.c_double()
            eng.h.check(L.mpsw_time_kernel(eng.h.ptr, i, FP32, B, 1, ctypes.byref(out)), 'time_kernel')
        torch.cuda.nvtx.range_pop()
        return
    if a.profile:
        timed(lambda: gradient_batch(FP32, B, du_i, dh_i), a.warmup, a.steps)
        return
    with Clocks(dev) as clk:
        t32, launches = timed(lambda: gradient_batch(FP32, B, du_i, dh_i), a.warmup, a.steps)
    clocks = clk.summary()
    # the job's time is its slowest replica's
    ms = replicas.max_over_ranks(sum(t32) / len(t32), device='cuda')
    value = world * B / (ms / 1e3)

    # phases of one step (window forward, TL sweep, AD sweep), after an L2 flush
    flush.zero_()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    gradient_batch(FP32, B, du_i, dh_i, ev)
    torch.cuda.synchronize()
    phases = {k: ev[i].elapsed_time(ev[i + 1]) for i, k in enumerate(('window', 'tl', 'ad'))}

    # accuracy of the batched FP32 form against the FP64 window on the same members
    ru32, rh32 = gradient_batch(FP32, B, du_i, dh_i)
    ru64, rh64 = gradient_batch(FP64, B, du_i, dh_i)
    num = torch.sqrt(((ru32 - ru64) ** 2).sum(0) + ((rh32 - rh64) ** 2).sum(0))
    den = torch.sqrt((ru64 ** 2).sum(0) + (rh64 ** 2).sum(0))
    rel_err = float((num / den).max())

    # plain FP64 single-member form (the drop-in numerics, one gradient per sweep)
    plain = None
    if not a.no_plain:
        tp, _ = timed(lambda: gradient_batch(FP64, 1, du_i[:, :1].contiguous(), dh_i[:, :1].contiguous()),
                      1, max(1, min(a.steps, 2)))
        plain = 1.0 / (sum(tp) / len(tp) / 1e3)

    # end to end through the public API with host buffers (pinned), copies inside
    du_host = torch.tensor(du_h).pin_memory()
    dh_host = torch.tensor(dh_h).pin_memory()
    out_u = torch.empty_like(du_host).pin_memory()
    out_h = torch.empty_like(dh_host).pin_memory()

    # device buffers of the public-API path, allocated once: a step allocates nothing
    xu, xh = torch.empty_like(du), torch.empty_like(dh)
    work = (torch.empty_like(du), torch.empty_like(dh))
    res = (torch.empty_like(du), torch.empty_like(dh))

    def e2e_step():
        w = Window(eng, a.nsteps, a.ckpt, a.storage)
        xu.copy_(du_host, non_blocking=True)
        xh.copy_(dh_host, non_blocking=True)
        tu, th = w.tl(xu, xh, FP32, work=work, out=res)
        gu, gh = w.ad(tu, th, FP32, work=work, out=(xu, xh))
        out_u.copy_(gu, non_blocking=True)
        out_h.copy_(gh, non_blocking=True)

    te, _ = timed(e2e_step, 1, a.steps)
    e2e_val = world * B / (sum(te) / len(te) / 1e3)

    # roofline of the dominant member kernel, timed alone with CUDA events
    roof = None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        pass
    hbm = peaks.get('hbm_gbs')
    peak_kind = 'measured' if hbm else 'fallback'
    hbm = hbm or 6650.0
    gradient_batch(FP32, B, du_i, dh_i)  # leaves the buffers of this configuration in place
    sum_eoe = int(unit['nEdgesOnEdge'].sum())
    import ctypes
    fm, fk = ctypes.c_int(), ctypes.c_int()
    eng.h.check(L.mpsw_window_fused(eng.h.ptr, FP32, B, ctypes.byref(fm), ctypes.byref(fk)), 'window_fused')
    fused = fm.value > 0
    # the kernels the sweeps launch: the two fused stage kernels, or the eight split ones
    timed_k = ['tl_stage', 'ad_stage'] if fused else KERNELS
    kt = {}
    for name in timed_k:
        out = ctypes.c_double()
        eng.h.check(L.mpsw_time_kernel(eng.h.ptr, KERNELS.index(name), FP32, B, 20, ctypes.byref(out)), 'time_kernel')
        kt[name] = out.value

    def kbytes(k):
        return fused_bytes(k, nC, nE, nV, B) if fused else kernel_bytes(k, nC, nE, nV, sum_eoe, B, 4)
    cand = ['tl_stage', 'ad_stage'] if fused else KERNELS[:8]
    top = max(cand, key=lambda k: kt[k])  # every candidate launches once per stage
    bytes_ = kbytes(top)
    ach = bytes_ / (kt[top] / 1e3) / 1e9
    s8d = model_stage_bytes(nC, nE, nV, sum_eoe, B)
    stages = {k: {'ms': kt[k], 'algorithmic_bytes': kbytes(k), 'achieved_gbs': kbytes(k) / (kt[k] / 1e3) / 1e9,
                  'frac': kbytes(k) / (kt[k] / 1e3) / 1e9 / hbm,
                  'frac_of_M_plus_BS': s8d / (kt[k] / 1e3) / 1e9 / hbm}
              for k in ('tl_stage', 'ad_stage')}
    roof = {'bound': 'hbm', 'kernel': ('k_tl_fused' if top == 'tl_stage' else 'k_ad_fused') if fused else top,
            'achieved': ach, 'peak': hbm, 'unit': 'GB/s', 'frac': ach / hbm, 'peak_source': peak_kind,
            'traffic': traffic_of(('tl_fused' if top == 'tl_stage' else 'ad_fused') if fused else top, a.level, B),
            'algorithmic_bytes': bytes_, 'ms_per_launch': kt[top], 'timing': 'each launch alone after a 256 MB L2 flush',
            'stage_bytes_M_plus_BS': s8d, 'kernel_ms': kt, 'stages': stages,
            'fused': {'members_per_block': fm.value, 'tile_cells': fk.value} if fused else None}
    if not fused:
        vb = (ctypes.c_int * 16)()
        eng.h.check(L.mpsw_window_tuning(eng.h.ptr, FP32, B, vb), 'window_tuning')
        roof['tuning'] = {k: {'v': vb[2 * i], 'block': vb[2 * i + 1]} for i, k in enumerate(KERNELS[:8])}

    # host baseline: serial oracle on one core, bounded sample
    cpu = None
    if rank == 0:
        sec, sample = cpu_gradient_seconds(a.level, a.dt, a.nsteps)
        cpu = {'value': 1.0 / sec, 'unit': UNIT, 'cores': 1, 'kind': 'port',
               'sample': '%d forward + %d TL + %d AD steps of one member, extrapolated to %d steps' % (sample, sample, sample, a.nsteps)}

    if rank == 0:
        wset = (B * (nE + nC) * (8 * 3 + 4 * 12) + 8 * (nE + nC) * 60) / 1e6
        line = {
            'metric': METRIC, 'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': a.steps,
            'warmup': a.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32 stencils + f64 accumulation',
            'data': 'synthetic (seeded balanced flow over 8 seeded mountains, level-%d TRiSK mesh, seeded perturbations)' % a.level,
            'config': workload_config(a),
            'stage_storage': {-1: 'auto (FP64+FP32 stage linearisation points when they fit 40%% of free HBM)', 0: 'none: stages recomputed from checkpoints', 1: 'FP64', 2: 'FP32', 3: 'FP64+FP32'}[a.storage],
            'working_set_mb': round(wset),
            'step_ms': [round(t, 3) for t in t32],
            'phase_ms': phases,
            'fp64_plain_gradients_per_s': plain,
            'batched_vs_plain': (value / world / plain) if plain else None,
            'rel_err_fp32_vs_fp64': rel_err,
            'e2e': {'value': e2e_val, 'unit': UNIT, 'h2d_bytes_per_step': int(du_host.numel() * 8 + dh_host.numel() * 8),
                    'd2h_bytes_per_step': int(out_u.numel() * 8 + out_h.numel() * 8),
                    'step_ms': [round(t, 3) for t in te]},
            'roofline': roof,
            'cpu_baseline': cpu,
            'clocks': clocks,
            'gpu_launches': int(launches),
        }
        print(json.dumps(line), flush=True)


def forward_bytes(nC, nE, nV, sum_eoe, s, a=8):
    """Algorithmic bytes of one RK4 step of one trajectory: per stage the mesh once,
    M(s) = 4 (2E + 2E + S + E + 2E + N + 3V + 3V) + s (S + 2E + 2N + 3V + 2V), and the state
    S = (N + E)(2s + 3a) (read x_k, write x_k+1 at s; x0 and the accumulator at a)."""
    E, N, V, S = nE, nC, nV, sum_eoe
    mesh = 4 * (2 * E + 2 * E + S + E + 2 * E + N + 3 * V + 3 * V) + s * (S + 2 * E + 2 * N + 3 * V + 2 * V)
    return 4 * (mesh + (N + E) * (2 * s + 3 * a))


def _oracle_forward_sample(args):
    """Seconds per sw_rk4 step of the oracle on the forward workload (host, one core)."""
    level, dt, n = args
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    m = O.OracleModule()
    forward_module(m, level, dt)
    m.sw_mpas_init_block()
    m.sw_rk4()
    t0 = time.perf_counter()
    for _ in range(n):
        m.sw_rk4()
    return (time.perf_counter() - t0) / n


def forward_module(mod, level, dt):
    """Seeded balanced flow over seeded mountains (h reduced by the topography)."""
    from mpsw import ic
    unit, mesh, st = workload(level, dt)
    load_module(mod, unit, mesh, st, dt)
    b = ic.mountains(mesh, 1000)
    mod.h_s = b[None, :]
    mod.h[0, 0] = st['h'] - b
    return unit


def run_forward(a, rank, world):
    """Nonlinear forward over one day: FP32 stencils + FP64 accumulation (the value) beside the
    plain FP64 form, each timed on the engine's stream; errors against the FP64 GPU run."""
    import ctypes
    import numpy as np
    import torch
    from module_sw_mpas import MpasSwModule
    from mpsw import _lib, replicas

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    mod = MpasSwModule()
    unit = forward_module(mod, a.level, a.dt)
    mod.sw_mpas_init_block()
    L = _lib.load()
    h = mod.handle
    sp = ctypes.c_void_p()
    h.check(L.mpsw_get_stream(h.ptr, ctypes.byref(sp)), 'get_stream')
    stream = torch.cuda.ExternalStream(sp.value)
    nC, nE, nV = unit['nCells'], unit['nEdges'], unit['nVertices']
    u0 = torch.tensor(np.ascontiguousarray(mod.u[0, 0]), device='cuda')
    h0 = torch.tensor(np.ascontiguousarray(mod.h[0, 0]), device='cuda')
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')

    def reset():
        torch.cuda.synchronize()
        h.check(L.mpsw_state_from_device(h.ptr, ctypes.c_void_p(u0.data_ptr()), ctypes.c_void_p(h0.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), 'state')

    def run(prec, n_warm, n_time):
        times = []
        launches0 = L.mpsw_launch_count()
        for i in range(n_warm + n_time):
            reset()
            flush.zero_()
            torch.cuda.synchronize()
            replicas_barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.check(L.mpsw_forward(h.ptr, prec, a.nsteps), 'forward')
            e1.record(stream)
            torch.cuda.synchronize()
            replicas_barrier()
            if i >= n_warm:
                times.append(e0.elapsed_time(e1))
            else:
                launches0 = L.mpsw_launch_count()
        return sum(times) / len(times), (L.mpsw_launch_count() - launches0) / max(1, n_time)

    def replicas_barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def state():
        out_u = torch.empty(nE, dtype=torch.float64, device='cuda')
        out_h = torch.empty(nC, dtype=torch.float64, device='cuda')
        h.check(L.mpsw_state_to_device(h.ptr, ctypes.c_void_p(out_u.data_ptr()), ctypes.c_void_p(out_h.data_ptr()),
                                       ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), 'state')
        torch.cuda.synchronize()
        return out_u, out_h

    days = a.nsteps * a.dt / 86400.0
    with Clocks(dev) as clk:
        ms32, launches = run(1, a.warmup, a.steps)
    clocks = clk.summary()
    ms32 = replicas.max_over_ranks(ms32, device='cuda')
    u32, h32 = state()
    ms64, _ = run(0, 1, max(1, min(a.steps, 2)))
    ms64 = replicas.max_over_ranks(ms64, device='cuda')
    u64, h64 = state()
    err = {'u': float(torch.linalg.norm(u32 - u64) / torch.linalg.norm(u64)),
           'h': float(torch.linalg.norm(h32 - h64) / torch.linalg.norm(h64))}
    value = world * days / (ms32 / 1e3)

    # end to end through the module surface: host state in, host state out, every run
    hu, hh = u0.cpu().numpy(), h0.cpu().numpy()
    te = []
    for i in range(1 + a.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        mod.u[0, 0] = hu
        mod.h[0, 0] = hh
        mod.sw_rk4_steps(a.nsteps, 1)
        out = mod.h[0, 0].copy(), mod.u[0, 0].copy()
        if i:
            te.append(time.perf_counter() - t0)
    e2e = world * days / (sum(te) / len(te))

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        pass
    hbm = peaks.get('hbm_gbs') or 6650.0
    sum_eoe = int(unit['nEdgesOnEdge'].sum())
    bytes_step = forward_bytes(nC, nE, nV, sum_eoe, 4)
    ach = bytes_step / (ms32 / 1e3 / a.nsteps) / 1e9
    cpu = None
    if rank == 0:
        sample = 3
        per = _oracle_forward_sample((a.level, a.dt, sample))
        cpu = {'value': days / (per * a.nsteps), 'unit': 'sim-days/s', 'cores': 1, 'kind': 'port',
               'sample': '%d sw_rk4 steps of the oracle, extrapolated to %d steps' % (sample, a.nsteps)}
    if rank == 0:
        line = {
            'metric': 'sim-days/s, nonlinear forward, FP32 stencils + FP64 accumulation (error vs FP64 GPU)',
            'value': value, 'unit': 'sim-days/s', 'n_gpus': world, 'steps': a.steps, 'warmup': a.warmup,
            'ms_per_step': ms32, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f32 stencils + f64 accumulation',
            'data': 'synthetic (seeded balanced flow over 8 seeded mountains, level-%d TRiSK mesh)' % a.level,
            'config': {'workload': 'forward: level-%d mesh (%d cells), %d RK4 steps of %g s (%.2f days)' % (a.level, nC, a.nsteps, a.dt, days),
                       'parallelism': 'replicas x%d' % world,
                       'l2': 'flushed (256 MB write) between timed runs; state + mesh ~%.0f MB' % ((nC + nE) * 8 * 10 / 1e6 + 300 * nC / 1e6)},
            'fp64_sim_days_per_s': world * days / (ms64 / 1e3),
            'rel_err_fp32_vs_fp64': err,
            'e2e': {'value': e2e, 'unit': 'sim-days/s', 'h2d_bytes_per_step': int((nC + nE) * 8),
                    'd2h_bytes_per_step': int((nC + nE) * 8)},
            'roofline': {'bound': 'hbm', 'kernel': 'one RK4 step (20 launches)', 'achieved': ach, 'peak': hbm,
                         'unit': 'GB/s', 'frac': ach / hbm, 'traffic': None, 'algorithmic_bytes': bytes_step,
                         'peak_source': 'measured' if peaks.get('hbm_gbs') else 'fallback'},
            'cpu_baseline': cpu,
            'clocks': clocks,
            'gpu_launches': int(launches),
        }
        print(json.dumps(line), flush=True)


def _oracle_costs_sample(args):
    """Seconds per step of the oracle's forward and adjoint (one cost function) on the host."""
    level, dt, n = args
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    unit, mesh, st = workload(level, dt)
    m = O.OracleModule()
    load_module(m, unit, mesh, st, dt)
    m.var_allocation_adj()
    m.sw_mpas_init_block()
    u0, h0 = m.u[0, 0].copy(), m.h[0, 0].copy()
    t0 = time.perf_counter()
    for _ in range(n):
        m.sw_rk4()
    t1 = time.perf_counter()
    m.h_ad[0, 0] = m.h[0, 0]
    for _ in range(n):
        m.u[0, 0], m.h[0, 0] = u0, h0
        m.sw_rk4_adj()
    t2 = time.perf_counter()
    return (t1 - t0) / n, (t2 - t1) / n


def run_costs(a, rank, world):
    """Gradients of B quadratic costs J_k = 1/2 |M_k h(T)|^2 (M_k: seeded spherical-cap masks)
    with respect to the initial state: one window forward, then one batched adjoint sweep seeded
    with M_k^T M_k h(T); FP32 stencils with FP64 accumulation, beside sequential plain FP64
    adjoint runs (one cost per window)."""
    import ctypes
    import torch
    from module_sw_mpas import MpasSwModule
    from mpsw import _lib, ic, replicas
    from mpsw.torch_api import FP32, FP64, Engine, Window

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    unit, mesh, st = workload(a.level, a.dt)
    mod = MpasSwModule()
    load_module(mod, unit, mesh, st, a.dt)
    mod.var_allocation_adj()
    mod.sw_mpas_init_block()
    eng = Engine(mod)
    L = _lib.load()
    B = a.batch
    nC, nE, nV = unit['nCells'], unit['nEdges'], unit['nVertices']
    masks = torch.tensor(ic.cap_masks(mesh, replicas.member_seed(3, rank), B), device='cuda')
    masks_i = eng.to_internal(masks, 0)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device='cuda')

    def gradients(prec, mk):
        """One bench step: window forward, seeds from h(T), batched adjoint; internal order."""
        w = Window(eng, a.nsteps, a.ckpt, a.storage)
        uT = torch.empty(nE, 1, dtype=torch.float64, device='cuda')
        hT = torch.empty(nC, 1, dtype=torch.float64, device='cuda')
        eng.h.call('mpsw_window_final_state', ctypes.c_void_p(uT.data_ptr()), ctypes.c_void_p(hT.data_ptr()),
                   ctypes.c_void_p(stream.cuda_stream))
        au = torch.zeros(nE, mk.shape[1], dtype=torch.float64, device='cuda')
        ah = (mk * mk * hT).contiguous()
        w.ad_internal(au, ah, prec)
        return au, ah

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def timed(fn, n_warm, n_time):
        for _ in range(n_warm):
            fn()
        times = []
        launches0 = L.mpsw_launch_count()
        quiet = host_quiet()
        for _ in range(n_time):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            barrier()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            times.append(e0.elapsed_time(e1))
        quiet.close()
        return times, (L.mpsw_launch_count() - launches0) / n_time

    with Clocks(dev) as clk:
        t32, launches = timed(lambda: gradients(FP32, masks_i), a.warmup, a.steps)
    clocks = clk.summary()
    ms = replicas.max_over_ranks(sum(t32) / len(t32), device='cuda')
    value = world * B / (ms / 1e3)
    gu32, gh32 = gradients(FP32, masks_i)
    gu64, gh64 = gradients(FP64, masks_i)
    num = torch.sqrt(((gu32 - gu64) ** 2).sum(0) + ((gh32 - gh64) ** 2).sum(0))
    den = torch.sqrt((gu64 ** 2).sum(0) + (gh64 ** 2).sum(0))
    rel_err = float((num / den).max())
    # sequential plain FP64 adjoint runs: one cost per window
    tp, _ = timed(lambda: gradients(FP64, masks_i[:, :1].contiguous()), 1, 1)
    seq = 1.0 / (tp[0] / 1e3)

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, 'MEASURED_PEAKS.json')))
    except Exception:
        pass
    hbm = peaks.get('hbm_gbs') or 6650.0
    gradients(FP32, masks_i)  # leaves the buffers of this configuration in place
    out = ctypes.c_double()
    eng.h.check(L.mpsw_time_kernel(eng.h.ptr, 9, FP32, B, 10, ctypes.byref(out)), 'time_kernel')
    sum_eoe = int(unit['nEdgesOnEdge'].sum())
    sb = kernel_bytes('ad_stage', nC, nE, nV, sum_eoe, B, 4)
    ach = sb / (out.value / 1e3) / 1e9
    cpu = None
    if rank == 0:
        sample = 3
        f, adj = _oracle_costs_sample((a.level, a.dt, sample))
        cpu = {'value': 1.0 / ((f + adj) * a.nsteps), 'unit': 'gradients/s', 'cores': 1, 'kind': 'port',
               'sample': '%d forward + %d adjoint steps of the oracle (one cost), extrapolated to %d steps' % (sample, sample, a.nsteps)}
    if rank == 0:
        line = {
            'metric': 'cost-function gradients/s, batched FP32 adjoint vs sequential plain FP64 (rel err<=1e-4)',
            'value': value, 'unit': 'gradients/s', 'n_gpus': world, 'steps': a.steps, 'warmup': a.warmup,
            'ms_per_step': ms, 'step_ms': [round(t, 3) for t in t32], 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32 stencils + f64 accumulation',
            'data': 'synthetic (seeded balanced flow, level-%d TRiSK mesh, %d seeded spherical-cap masks)' % (a.level, B),
            'config': {'workload': 'costs: level-%d mesh (%d cells), %d RK4 steps of %g s, %d costs J_k = 1/2 |M_k h(T)|^2' % (a.level, nC, a.nsteps, a.dt, B),
                       'parallelism': 'replicas x%d' % world, 'l2': 'flushed (256 MB write) between timed steps'},
            'sequential_fp64_gradients_per_s': seq,
            'batched_vs_sequential': value / world / seq,
            'rel_err_fp32_vs_fp64': rel_err,
            'roofline': {'bound': 'hbm', 'kernel': 'one adjoint stage (ad_edge, ad_cell, ad_vertex, ad_final)',
                         'achieved': ach, 'peak': hbm, 'unit': 'GB/s', 'frac': ach / hbm, 'traffic': None,
                         'algorithmic_bytes': sb, 'ms_per_launch': out.value,
                         'peak_source': 'measured' if peaks.get('hbm_gbs') else 'fallback'},
            'cpu_baseline': cpu,
            'clocks': clocks,
            'gpu_launches': int(launches),
        }
        print(json.dumps(line), flush=True)


def spawn_ranks(n, script=None, argv=None):
    """`bench.py --gpus N` started without a launcher: start N rank processes of this script (one
    per GPU, as torchrun would: RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT set), pass rank 0's
    output through, and return the first nonzero exit status (0 when all succeed).  script / argv
    default to this file and its command line."""
    import socket
    with socket.socket() as sk:
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    procs = []
    for r in range(n):
        env = dict(os.environ, RANK=str(r), LOCAL_RANK=str(r), WORLD_SIZE=str(n), LOCAL_WORLD_SIZE=str(n),
                   MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
        cmd = [sys.executable, script or os.path.abspath(__file__)] + (sys.argv[1:] if argv is None else argv)
        procs.append(subprocess.Popen(cmd, env=env, stdout=None if r == 0 else subprocess.DEVNULL))
    rcs = [p.wait() for p in procs]
    return next((rc for rc in rcs if rc), 0)


def run_long(a, rank, world):
    """Long-window gradients (level 8 by default): the window's stages are not stored (they would
    take hundreds of GB), so the tangent-linear sweep recomputes the trajectory alongside and the
    adjoint sweep reverses it by binomial checkpointing with `snapshots` snapshot states,
    recomputing each step's RK stages.  One bench step is one gradient batch (B members); the
    FP64 window's dot-product test and the FP32 form's error against it are reported."""
    import torch
    from module_sw_mpas import MpasSwModule
    from mpsw import _lib, replicas
    from mpsw.torch_api import FP32, FP64, Engine, Window

    dev = rank % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    unit, mesh, st = workload(a.level, a.dt)
    from mpsw import ic
    b = ic.mountains(mesh, 1000)
    mod = MpasSwModule()
    load_module(mod, unit, mesh, st, a.dt)
    mod.h_s = b[None, :]
    mod.h[0, 0] = st['h'] - b
    mod.sw_mpas_init_block()
    eng = Engine(mod)
    L = _lib.load()
    B = a.batch
    nC, nE = unit['nCells'], unit['nEdges']
    dh_h, du_h = perturbations(unit, B, seed=replicas.member_seed(4, rank))
    du_i = eng.to_internal(torch.tensor(du_h, device='cuda'), 1)
    dh_i = eng.to_internal(torch.tensor(dh_h, device='cuda'), 0)
    stream = torch.cuda.current_stream()

    def batch(prec, keep=False):
        w = Window(eng, a.nsteps, a.ckpt, 0, 0.0, a.snapshots)
        xu, xh = du_i.clone(), dh_i.clone()
        w.tl_internal(xu, xh, prec)
        tl = (xu.clone(), xh.clone()) if keep else None
        w.ad_internal(xu, xh, prec)
        return tl, (xu, xh), w.forward_steps()

    batch(FP32)  # warm-up (graph capture)
    times = []
    launches0 = L.mpsw_launch_count()
    with Clocks(dev) as clk:
        for _ in range(a.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            _, _, fsteps = batch(FP32)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    launches = (L.mpsw_launch_count() - launches0) / a.steps
    ms = replicas.max_over_ranks(sum(times) / len(times), device='cuda')
    value = world * B / (ms / 1e3)
    tl32, ad32, _ = batch(FP32, keep=True)
    tl64, ad64, _ = batch(FP64, keep=True)
    # dot-product test of the FP64 window: <L dx, L dx> = <dx, L^T L dx> (the adjoint is seeded
    # with the tangent-linear output)
    lhs = (tl64[0] * tl64[0]).sum(0) + (tl64[1] * tl64[1]).sum(0)
    rhs = (du_i * ad64[0]).sum(0) + (dh_i * ad64[1]).sum(0)
    dot = float(((lhs - rhs).abs() / lhs.abs()).max())
    num = torch.sqrt(((ad32[0] - ad64[0]) ** 2).sum(0) + ((ad32[1] - ad64[1]) ** 2).sum(0))
    den = torch.sqrt((ad64[0] ** 2).sum(0) + (ad64[1] ** 2).sum(0))
    rel_err = float((num / den).max())
    if rank == 0:
        line = {
            'metric': 'TL+AD gradients/s, long window, binomial checkpointing (FP32 stencils, FP64 accumulation)',
            'value': value, 'unit': UNIT, 'n_gpus': world, 'steps': a.steps, 'warmup': 1, 'ms_per_step': ms,
            'step_ms': [round(t, 1) for t in times], 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f32 stencils + f64 accumulation',
            'data': 'synthetic (seeded balanced flow over 8 seeded mountains, level-%d TRiSK mesh)' % a.level,
            'config': {'workload': 'long TL+AD window: level-%d mesh (%d cells), %d RK4 steps of %g s, %d members, '
                                   'binomial checkpointing with %d snapshots' % (a.level, nC, a.nsteps, a.dt, B, a.snapshots),
                       'parallelism': 'replicas x%d' % world},
            'recomputed_forward_steps_in_adjoint': fsteps,
            'fp64_dot_product_rel': dot,
            'rel_err_fp32_vs_fp64': rel_err,
            'clocks': clk.summary(),
            'gpu_launches': int(launches),
        }
        print(json.dumps(line), flush=True)


def main():
    a = parse()
    if 'WORLD_SIZE' not in os.environ and a.gpus > 1 and a.impl == 'mpsw':
        sys.exit(spawn_ranks(a.gpus))
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if a.impl == 'mpsw':
            torch.cuda.set_device(int(os.environ.get('LOCAL_RANK', '0')))
            dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=600))
    if a.impl == 'reference':
        run_reference(a, rank, world)
    elif a.workload == 'fwd':
        run_forward(a, rank, world)
    elif a.workload == 'costs':
        run_costs(a, rank, world)
    elif a.workload == 'long':
        run_long(a, rank, world)
    else:
        run_mpsw(a, rank, world)
    if world > 1 and a.impl == 'mpsw':
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
