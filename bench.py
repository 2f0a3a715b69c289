"""Benchmark of the dense statevector engine (one JSON line on rank 0).

Headline workload (metric "gate-layer HBM GB/s at 30q c64"): a 30-qubit
complex64 random circuit of 40 layers -- U3(theta, phi, lambda) on every qubit
with angles U[0, 2pi) from the seed, then a brick wall of CZ -- fused into tile
passes.  One step = the whole 40-layer circuit applied to the 8 GiB state that
stays resident in HBM (inputs far larger than the 126 MB L2).
value = fused passes x 2 x 2^30 x 8 B / step time (algorithmic bytes: one read
and one write of the state per pass).

Secondary block "vqe" (metric "VQE grads/s adjoint vs parameter-shift"): the
24-qubit complex64 hardware-efficient ansatz of 10 layers (480 parameters)
with the open-chain transverse-field Ising Hamiltonian; adjoint gradients per
second against parameter-shift gradients (2 x 480 forward runs) on the same
kernels.

Multi-GPU: replicas only -- every rank runs the same workload on its own GPU,
value is the sum over ranks, time the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'dense-evolution_b200'))
sys.path.insert(0, ROOT)

N_QUBITS, LAYERS, SEED = 30, 40, 2024
VQE_N, VQE_LAYERS = 24, 10
METRIC = 'gate-layer HBM GB/s at 30q c64; VQE grads/s adjoint vs parameter-shift'


def _peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured (MEASURED_PEAKS.json hbm_gbs)'
    except (OSError, KeyError, ValueError):
        return 6650.0, 'fallback 6.65 TB/s'


def _profile_traffic():
    """DRAM bytes per 30-qubit rotation-pass launch from the committed ncu summary
    (a 28-qubit capture scaled by the state size), or None."""
    path = os.path.join(ROOT, 'profiles', 'rotation_pass_28q_c64.txt')
    try:
        with open(path) as f:
            for line in f:
                if line.startswith('dram_bytes_per_launch_full_size:'):
                    return float(line.split(':', 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                          '-lms', '200', '-i', str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
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
        for ln in self.lines:
            f = [x.strip() for x in ln.split(',')]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower() == 'active':
                    reasons.add(name)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['unsampled'], 'samples': 0}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


def _dist():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return ws, rank, local


def _max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device='cuda')
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (a NumPy restatement of the reference's eager path)
# ---------------------------------------------------------------------------

def _fused_schedule(n, layers):
    """(transpiled gate count, fused pass count) of the headline circuit -- host
    code only (lowering + fusion), used to put both arms on one byte rule."""
    import torch
    from dense_evolution.circuits import fusion
    from dense_evolution.circuits.compiler import QuantumTranspiler, default_tile_bits
    from dense_evolution.workloads import brick_u3_circuit
    target = QuantumTranspiler.transpile(brick_u3_circuit(n, layers, SEED))
    _, _, packed = fusion.build(target, n, default_tile_bits(n, torch.complex64))
    return len(target), len(packed.passes)


def cpu_baseline(n=N_QUBITS, layers=LAYERS, gates=2, npasses=None):
    """The CPU path of the reference algorithm (the NumPy oracle, complex64 like
    the workload) on a bounded sample: `gates` transpiled gates of the headline
    circuit, one full-state pass each.  The whole-circuit time is extrapolated
    as (mean time per gate) x (transpiled gate count), and the value uses the
    same rule as the GPU arm: fused passes x 2 x 2^n x 8 B / circuit time, so
    the ratio of the two values is the speed-up on the same circuit.  `cores`
    is measured: process CPU time / wall time over the sample."""
    from oracle import sv_oracle as O
    from dense_evolution.workloads import brick_u3_circuit
    ngates, nfused = _fused_schedule(n, layers)
    if npasses is not None:
        nfused = npasses
    circ = O.transpile(brick_u3_circuit(n, 1, SEED))[:gates]
    sv = np.zeros(1 << n, dtype=np.complex64)
    sv[0] = 1
    c0, t0 = time.process_time(), time.perf_counter()
    for cmd in circ:
        sv = O.run_circuit(sv, n, [cmd], do_transpile=False)
    dt = time.perf_counter() - t0
    cores = (time.process_time() - c0) / dt
    per_gate = dt / len(circ)
    est = per_gate * ngates
    gbs = nfused * 2 * (1 << n) * 8 / est / 1e9
    return {'value': gbs, 'unit': 'GB/s', 'cores': round(cores, 2), 'kind': 'port',
            'sample': f'{len(circ)} transpiled gates ({", ".join(c[0] for c in circ)}) of the {n}-qubit complex64 '
                      f'circuit through the NumPy oracle, {per_gate:.2f} s per gate, extrapolated to all '
                      f'{ngates} gates ({est:.0f} s per circuit); bytes counted as {nfused} fused passes',
            'est_circuit_s': est}


def config1_cpu(layers=20, n=20):
    """Config 1 whole on the host cores: the 20-qubit, 20-layer brick circuit in
    complex128 through the NumPy oracle (the reference's eager CPU path
    restated), state and <Z_i>; seconds per circuit (one run after a warm-up of
    the first layer)."""
    from oracle import sv_oracle as O
    from dense_evolution.workloads import brick_u3_circuit
    circ = brick_u3_circuit(n, layers, SEED)
    O.run_circuit(O.zero_state(n), n, circ[:n])
    c0, t0 = time.process_time(), time.perf_counter()
    sv = O.run_circuit(O.zero_state(n), n, circ)
    p = np.abs(sv) ** 2
    z = [float(np.sum(p.reshape(1 << q, 2, -1)[:, 0].sum() - p.reshape(1 << q, 2, -1)[:, 1].sum()))
         for q in range(n)]
    dt = time.perf_counter() - t0
    return {'workload': f'{n}-qubit complex128 brick circuit, {layers} layers (config 1), state + <Z_i>',
            'seconds_per_circuit': dt, 'cores': round((time.process_time() - c0) / dt, 2), 'kind': 'port',
            'z0': z[0]}


def config1_gpu(layers=20, n=20, reps=20, warm=5):
    """Config 1 whole on the GPU through the public API (DenseSVSimulator,
    complex128): seconds per circuit, state resident, <Z_i> read back.  This
    leg runs after the CPU baseline has left the GPU idle for half a minute, so
    warm-up circuits come first and the mean is over 20 circuits (one full run
    with one warm-up and three timed circuits read 17 ms; alone, 1.5 ms)."""
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import brick_u3_circuit
    circ = brick_u3_circuit(n, layers, SEED)
    sim = de.DenseSVSimulator(n)
    for _ in range(warm):
        sim.set_initial_state(None)
        sim.run_circuit(circ)
        z = sim.expectation_z()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        sim.set_initial_state(None)
        sim.run_circuit(circ)
        z = sim.expectation_z()
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / reps
    return {'seconds_per_circuit': dt, 'z0': float(z[0])}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    t0 = time.perf_counter()
    vals, cores, last = [], [], None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(args.qubits, args.layers, gates=1)
        if i >= args.warmup:
            vals.append(r['value'])
            cores.append(r['cores'])
        last = r
    v = float(np.mean(vals))
    c1 = config1_cpu()
    line = {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'GB/s', 'n_gpus': args.gpus,
            'value_kind': 'estimate: a one-gate sample of the 30-qubit circuit per step, extrapolated to all gates',
            'config1_whole_circuit': c1,
            'steps': args.steps, 'warmup': args.warmup, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'complex64', 'data': 'synthetic',
            'config': {'workload': f'{args.qubits}-qubit complex64 random circuit, {args.layers} layers of U3 on every '
                                   f'qubit + brick-wall CZ', 'seed': SEED, 'qubits': args.qubits,
                       'layers': args.layers},
            'cpu_baseline': {'value': v, 'unit': 'GB/s', 'cores': float(np.mean(cores)), 'kind': 'port',
                             'sample': 'per step: ' + last['sample']},
            'e2e': {'value': v, 'unit': 'GB/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
            'wall_s': time.perf_counter() - t0}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def fidelity_check(n=28, layers=LAYERS):
    """Config 2's accuracy check: the headline circuit structure at n qubits in
    complex64 against the same circuit in complex128 (the accuracy mode); both
    on the GPU, untimed.  Returns fidelity |<a|b>|^2 and max |a - b|."""
    import torch
    import dense_evolution as de
    from dense_evolution.circuits.compiler import CompiledCircuit
    from dense_evolution.workloads import brick_u3_circuit
    target = de.QuantumTranspiler.transpile(brick_u3_circuit(n, layers, SEED))
    out = {}
    states = []
    for dt in (torch.complex64, torch.complex128):
        sv = torch.zeros(1 << n, dtype=dt, device='cuda')
        sv[0] = 1
        CompiledCircuit(target, n, dt).run(sv)
        states.append(sv)
    a, b = states[0].to(torch.complex128), states[1]
    out['qubits'] = n
    out['fidelity_c64_vs_c128'] = float(torch.abs(torch.vdot(b, a)) ** 2)
    out['max_abs_amp_error_c64'] = float((a - b).abs().max())
    out['norm_c128'] = float(torch.vdot(b, b).real)
    del a, b, states
    torch.cuda.empty_cache()
    return out


def run_headline(args, ws, local):
    """The headline: fused passes of the brick-wall U3 circuit, timed per pass
    with CUDA events on the launching stream; then the same metric end to end
    through DenseSVSimulator."""
    import torch
    import dense_evolution as de
    from dense_evolution import _native as N
    from dense_evolution.circuits.compiler import CompiledCircuit
    from dense_evolution.circuits import jit
    from dense_evolution.workloads import brick_u3_circuit

    dev = torch.device('cuda', torch.cuda.current_device())
    st = torch.cuda.current_stream()
    n, layers = args.qubits, args.layers
    circ = brick_u3_circuit(n, layers, SEED)
    t_c = time.perf_counter()
    plan = CompiledCircuit(de.QuantumTranspiler.transpile(circ), n, torch.complex64)
    rot = plan.rotation
    compile_s = time.perf_counter() - t_c
    npasses = plan.npasses
    sv = torch.empty(1 << n, dtype=torch.complex64, device=dev)
    lib = N.lib()
    N.check(lib.desv_init_basis(ctypes.c_void_p(sv.data_ptr()), n, N.DESV_C64, 0, ctypes.c_void_p(st.cuda_stream)),
            'init')
    pass_bytes = 2 * (1 << n) * 8
    specialised = rot is None and jit.enabled(n)
    t_c = time.perf_counter()
    if rot is not None:
        blocks = rot.blocks()
        kernels = rot.prog.pass_kernels(torch.cuda.current_device(), blocks)
        rows = rot.prog.rows
    else:
        ops_t, mats_t = plan.device_arrays(dev)
        passes = plan.device_passes
        kernels = plan.specialised_kernels(dev) if specialised else None
    jit_compile_s = time.perf_counter() - t_c

    def one_pass(i):
        if rot is not None:
            N.check(lib.desv_rot_pass(kernels[i].handle, ctypes.c_void_p(sv.data_ptr()), n,
                                      ctypes.c_void_p(rows.ctypes.data + i * rows.itemsize),
                                      blocks[i].ctypes.data_as(ctypes.c_void_p), len(blocks[i]),
                                      ctypes.c_void_p(st.cuda_stream)), 'rotation pass')
            return
        if specialised:
            jit.run_passes(kernels[i:i + 1], sv.data_ptr(), n, N.DESV_C64, passes[i:i + 1], ops_t.data_ptr(),
                           mats_t.data_ptr(), st.cuda_stream)
            return
        N.check(lib.desv_apply_passes(ctypes.c_void_p(sv.data_ptr()), n, N.DESV_C64,
                                      ctypes.c_void_p(passes[i:i + 1].ctypes.data), 1,
                                      ctypes.c_void_p(ops_t.data_ptr()), ctypes.c_void_p(mats_t.data_ptr()),
                                      ctypes.c_void_p(st.cuda_stream)), 'pass')

    for _ in range(args.warmup):
        for i in range(npasses):
            one_pass(i)
    torch.cuda.synchronize()
    _barrier(ws)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps * npasses + 1)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        _barrier(ws)
        ev[0].record()
        k = 1
        for _ in range(args.steps):
            for i in range(npasses):
                one_pass(i)
                ev[k].record()
                k += 1
        torch.cuda.synchronize()
    N.device_status()
    total_ms = ev[0].elapsed_time(ev[-1])
    per_pass = np.array([ev[j].elapsed_time(ev[j + 1]) for j in range(len(ev) - 1)])
    ms_step = _max_over_ranks(total_ms / args.steps, ws)
    value = ws * npasses * pass_bytes / (ms_step / 1e3) / 1e9
    avg_pass_ms = float(per_pass.mean())
    achieved = pass_bytes / (avg_pass_ms / 1e3) / 1e9
    peak, peak_src = _peaks()
    traffic = _profile_traffic()

    # ---- end to end through the public API: fresh seeded angles every step (the
    # same brick structure, as in a variational loop): transpile, angle
    # extraction, the rotation values and their H2D copy, run, <Z_i> read back
    sim = de.DenseSVSimulator(n, use_float32=True)
    e2e_times, h2d, parts = [], 0, []
    for i in range(0 if args.skip_e2e else args.warmup + args.steps):
        c = brick_u3_circuit(n, layers, SEED + 1 + i)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.set_initial_state(None)
        plan_i = sim.compile(c)
        t1 = time.perf_counter()
        sim.run_circuit(c)
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        sim.expectation_z()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_times.append(dt)
            parts.append((t1 - t0, t2 - t1, t0 + dt - t2))
            if plan_i.rotation is not None:
                h2d = int(sum(b.nbytes for b in plan_i.rotation.blocks()))
            else:
                ops_i, mats_i = plan_i.device_arrays(dev)
                h2d = int(ops_i.numel() + mats_i.numel() * 4)
    e2e_step = _max_over_ranks(float(np.mean(e2e_times)), ws) if e2e_times else float('nan')
    e2e_value = ws * npasses * pass_bytes / e2e_step / 1e9
    steps_ms = per_pass.reshape(args.steps, npasses).mean(axis=0)
    if rot is not None:
        st_ = rot.plan.stats()['per_pass']
        table = [{'pass': i, 'rotations': r, 'stages': g_, 'diag_groups': d, 'ms': round(float(steps_ms[i]), 4)}
                 for i, (r, g_, d) in enumerate(st_)]
    else:
        table = [{'pass': i, 'ms': round(float(steps_ms[i]), 4)} for i in range(npasses)]
    del sv, sim
    torch.cuda.empty_cache()
    return {
        'metric': METRIC, 'value': value, 'unit': 'GB/s', 'n_gpus': ws, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': ms_step, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'complex64 (fp32 gate math)', 'data': 'synthetic',
        'config': {'workload': f'{n}-qubit complex64 random circuit, {layers} layers of U3 on every qubit + '
                               f'brick-wall CZ, fused into tile passes', 'seed': SEED, 'qubits': n,
                   'layers': layers, 'fused_passes': npasses, 'tile_bits': plan.tile_bits,
                   'l2': f'state ({(1 << n) * 8 / 2**30:.2f} GiB) larger than L2 (126 MB); no flush needed',
                   'parallelism': f'replicas x{ws}'},
        'passes_per_step': npasses, 'layers_per_s': ws * layers / (ms_step / 1e3),
        'ms_per_layer': ms_step / layers, 'compile_s': compile_s, 'jit_compile_s': jit_compile_s,
        'roofline': {'bound': 'hbm', 'achieved': achieved, 'peak': peak, 'unit': 'GB/s',
                     'frac': achieved / peak, 'traffic': traffic, 'peak_source': peak_src,
                     'kernel': ('desv_rot_kernel (rotation pass, NVRTC sm_100a)' if rot is not None else
                                'desv_jit_kernel (plan-specialised fused pass, NVRTC sm_100a)' if specialised
                                else f'k_fused_pass<float2,{plan.tile_bits},3>'),
                     'algorithmic_bytes_per_launch': pass_bytes,
                     'avg_launch_ms': avg_pass_ms, 'min_launch_ms': float(per_pass.min()),
                     'max_launch_ms': float(per_pass.max())},
        'e2e': {'value': e2e_value, 'unit': 'GB/s', 'h2d_bytes_per_step': h2d,
                'd2h_bytes_per_step': (n + 1) * 8, 'ms_per_step': e2e_step * 1e3,
                'breakdown_ms': ({k: float(v) * 1e3 for k, v in zip(
                    ('host_plan (transpile, plan lookup, angle values)', 'run (values upload + passes)',
                     'readout (<Z_i> pass + read back)'), np.mean(parts, axis=0))} if parts else None),
                'path': 'DenseSVSimulator.run_circuit (new angles each step: transpile, angle extraction, '
                        'rotation values and their upload; the plan is cached by circuit structure) + '
                        'expectation_z()'},
        'gpu_launches': args.steps * npasses,
        'clocks': clk.summary(),
        'pass_table': table,
    }


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    line = run_headline(args, ws, local) if not args.skip_headline else {
        'metric': METRIC, 'value': None, 'unit': 'GB/s', 'n_gpus': ws, 'steps': args.steps,
        'warmup': args.warmup, 'higher_is_better': True, 'skipped': 'headline (--skip-headline)'}
    if not args.skip_headline and args.qubits == N_QUBITS and not args.skip_fidelity:
        line['fidelity_28q'] = fidelity_check(28, args.layers)
    line['vqe'] = run_vqe(args) if not args.skip_vqe else None
    torch.cuda.empty_cache()
    line['batch'] = run_batch(args) if not args.skip_batch else None
    torch.cuda.empty_cache()
    line['large'] = run_large(args) if not args.skip_large else None
    torch.cuda.empty_cache()
    npasses = line.get('passes_per_step')
    line['cpu_baseline'] = cpu_baseline(args.qubits, args.layers, gates=2, npasses=npasses) \
        if (rank == 0 and ws == 1 and not args.skip_cpu and not args.skip_headline) else None
    if line['cpu_baseline'] is not None:
        line['cpu_baseline']['value_kind'] = 'estimate (two-gate sample of the 30-qubit circuit, extrapolated)'
        c1 = config1_cpu()
        g1 = config1_gpu()
        line['config1'] = {'cpu': c1, 'gpu_seconds_per_circuit': g1['seconds_per_circuit'],
                           'speedup_gpu_over_cpu': c1['seconds_per_circuit'] / g1['seconds_per_circuit'],
                           'z0_cpu': c1['z0'], 'z0_gpu': g1['z0']}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_vqe(args):
    """Config 3: adjoint grads/s vs parameter-shift grads/s at 24q complex64."""
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, tfim_terms
    n, layers = args.vqe_qubits, VQE_LAYERS
    fn, npar = de.circuit_to_energy_fn(hea_circuit(n, layers), n, use_float32=True)
    prog = fn.program
    op = de.PauliSumOperator(tfim_terms(n), n)
    rng = np.random.default_rng(SEED)
    theta = rng.uniform(-np.pi, np.pi, npar)
    for _ in range(max(1, args.warmup)):
        prog.value_and_grad(rng.uniform(-np.pi, np.pi, npar), op)
    torch.cuda.synchronize()
    # a VQE loop: a fresh theta every gradient (host materialisation and upload
    # of the forward and backward values inside the timed region)
    reps = max(3, args.steps)
    thetas = [rng.uniform(-np.pi, np.pi, npar) for _ in range(reps)]
    t0 = time.perf_counter()
    for th in thetas:
        e, g, _ = prog.value_and_grad(th, op)
    torch.cuda.synchronize()
    adj_s = (time.perf_counter() - t0) / reps
    # the same gradient with theta repeated: the values are cached, so this is
    # (close to) the device time of the gradient's kernels
    t0 = time.perf_counter()
    for _ in range(reps):
        prog.value_and_grad(thetas[-1], op)
    torch.cuda.synchronize()
    cached_s = (time.perf_counter() - t0) / reps
    theta = thetas[-1]
    e, g, _ = prog.value_and_grad(theta, op)
    pauli = pauli_roofline(prog, theta, n)
    # parameter shift on the same kernels: 2 * npar forward runs + <H>
    if args.vqe_no_shift:
        return {'energy': e, 'adjoint_grads_per_s': 1.0 / adj_s, 'adjoint_ms': adj_s * 1e3, 'qubits': n,
                'pauli': pauli}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ps = prog.parameter_shift_grad(theta, op)
    torch.cuda.synchronize()
    ps_s = time.perf_counter() - t0
    return {'workload': f'{n}-qubit complex64 HEA, {layers} layers (RY,RZ + CX ladder), {npar} parameters, '
                        f'TFIM open chain', 'energy': e, 'adjoint_grads_per_s': 1.0 / adj_s,
            'theta': 'fresh theta every timed gradient (a VQE loop); parameter shift changes theta on every run',
            'adjoint_ms_repeated_theta': cached_s * 1e3,
            'host_ms_per_gradient': (adj_s - cached_s) * 1e3,
            'parameter_shift_grads_per_s': 1.0 / ps_s, 'adjoint_over_parameter_shift': ps_s / adj_s,
            'max_abs_grad_diff_adjoint_vs_shift': float(np.max(np.abs(g - ps))),
            'forward_passes': int(prog.forward.npasses),
            'backward_passes': int(len(prog.back.passes)), 'adjoint_ms': adj_s * 1e3, 'shift_ms': ps_s * 1e3,
            'pauli': pauli}


def pauli_roofline(prog, theta, n, reps=10):
    """<H> and H|psi> of the TFIM chain on the VQE state, timed with CUDA events
    on the launching stream; algorithmic bytes: every Pauli pass reads psi once
    (<H>), and H|psi> also writes its output once and reads + writes it on every
    further pass."""
    import torch
    from dense_evolution.physics.observables import plan_for
    from dense_evolution.workloads import tfim_terms
    psi = prog.forward_state(np.asarray(theta, dtype=np.float64))
    plan = plan_for(tfim_terms(n), n, dtype=psi.dtype)
    out = torch.empty_like(psi)
    amp = (1 << n) * psi.element_size()
    res = {'terms': int(plan.nterms), 'passes': int(plan.npasses)}
    for name, fn, nbytes in (('expect', lambda: plan.expect(psi), plan.npasses * amp),
                             ('matvec', lambda: plan.matvec(psi, out), plan.npasses * amp + amp +
                              (plan.npasses - 1) * 2 * amp)):
        # an NVTX range per kind, so that a profiler can pick these launches out
        torch.cuda.nvtx.range_push(f'pauli_{name}')
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        ms = e0.elapsed_time(e1) / reps
        res[name] = {'ms': ms, 'algorithmic_bytes': nbytes, 'gbs': nbytes / ms / 1e6,
                     'frac_of_hbm': nbytes / ms / 1e6 / _peaks()[0]}
    del psi, out
    return res


def run_batch(args, layers=6):
    """Config 4: 4096 circuits, n ~ U{10..20}, HEA of 6 layers, XXZ chain with J_z ~ U[0.5, 1.5];
    energy + adjoint gradient of every circuit: one persistent launch over the circuits of <= 12
    qubits, the wider ones as rows groups (one launch per pass over all circuits of a width), the
    whole batch replayed from one CUDA graph.  The tile width comes from the autotuner, tuned
    first on a seeded 256-circuit sample."""
    import torch
    from dense_evolution import autotune
    from dense_evolution.batch import BatchVQE, hea_xxz_batch
    ncirc = args.batch_circuits
    rng = np.random.default_rng(SEED)
    ns = rng.integers(10, 21, ncirc)
    if args.batch_qubits:
        ns = np.full(ncirc, args.batch_qubits)      # one width only (profiling a single rows group)
    jz = rng.uniform(0.5, 1.5, ncirc)
    srng = np.random.default_rng(SEED + 7)
    sample = hea_xxz_batch(srng.integers(10, 21, 256), layers, srng.uniform(0.5, 1.5, 256))
    tune = autotune.tune_batch(sample, use_float32=True) if not args.batch_no_tune else {}
    t0 = time.perf_counter()
    b = BatchVQE(hea_xxz_batch(ns, layers, jz), use_float32=True)
    build_s = time.perf_counter() - t0
    thetas = [rng.uniform(-np.pi, np.pi, 2 * n * layers) for n in ns]
    b.set_theta(thetas)
    b.capture()
    for _ in range(max(1, args.warmup)):
        b.graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(2, args.steps)
    e0.record()
    for _ in range(reps):
        b.graph.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # end to end: host parameters in, energies + gradients out, every step
    t0 = time.perf_counter()
    for _ in range(reps):
        e, g = b.run(thetas, use_graph=True)
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) / reps * 1e3
    amps = float(np.sum(2.0 ** ns))
    # algorithmic HBM bytes of the circuits wider than 12 qubits (rows groups:
    # BatchVQE.rows_algorithmic_bytes; persistent streamed circuits: forward
    # passes 2 2^n B, backward passes 4 2^n B, lambda = H psi 2 2^n B);
    # circuits of <= 12 qubits never leave shared memory
    hbm = 0.0
    for i, (pi, _, _) in enumerate(b.circ):
        if pi < 0:
            continue
        p = b.plans[pi]
        if p.n > 12:
            hbm += (2 * len(p.fwd.passes) + 4 * len(p.bwd.passes) + 2) * (1 << p.n) * 8
    hbm += sum(b.rows_algorithmic_bytes(g) for g in b.groups)
    hbm_gbs = hbm / (ms / 1e3) / 1e9
    # device time of each part: the persistent launch (<= 12 qubits) and every
    # rows group, CUDA events on the launching stream, eager launches
    parts = {}
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(b.groups) + 2)]
    evs[0].record()
    b.launch_persistent()
    evs[1].record()
    for k, g in enumerate(b.groups):
        g.launch(b.d_theta, b.d_grad, None)
        evs[k + 2].record()
    torch.cuda.synchronize()
    parts['persistent_ms'] = evs[0].elapsed_time(evs[1])
    rows_tab = []
    for k, g in enumerate(b.groups):
        gms = evs[k + 1].elapsed_time(evs[k + 2])
        gb = b.rows_algorithmic_bytes(g)
        rows_tab.append({'qubits': g.plan.n, 'rows': g.B, 'ms': gms, 'algorithmic_bytes': gb,
                         'gbs': gb / (gms / 1e3) / 1e9, 'frac_of_hbm': gb / (gms / 1e3) / 1e9 / _peaks()[0]})
    parts['rows_groups'] = rows_tab
    widths = f'{args.batch_qubits} qubits each' if args.batch_qubits else 'qubits uniform in 10..20'
    return {'workload': f'{ncirc} circuits, {widths}, HEA {layers} layers (RY,RZ + CX ladder), '
                        f'XXZ open chain J_xy=1, J_z~U[0.5,1.5]; energy + adjoint gradient per circuit',
            'ms_per_batch': ms, 'circuits_per_s': ncirc / (ms / 1e3), 'grads_per_s': ncirc / (ms / 1e3),
            'e2e_ms_per_batch': e2e_ms, 'plans': len(b.plans) + len(b.groups),
            'launches_per_batch': b.launches_per_batch(),
            'total_amplitudes': amps, 'resident_circuits': int(np.sum(ns <= 12)),
            'rows_from_qubits': b.rows_from, 'parts': parts,
            'streamed_algorithmic_bytes': hbm, 'achieved_gbs_streamed': hbm_gbs,
            'frac_of_hbm_streamed': hbm_gbs / _peaks()[0],
            'register_bound_ctas_per_sm': int(os.environ.get('DESV_BATCH_MINB', '2')),
            'plan_build_s': build_s, 'energy_mean': float(np.mean(e)), 'tile_bits': b.tile_bits,
            'autotune_ms_per_launch_256': {str(k): v for k, v in tune.items()}}


def run_large(args, n=32, n_ref=30, layers=4):
    """Config 5: 32-qubit complex64 adjoint gradient (psi, lambda, mu: 3 x 32 GiB), HEA 4 layers
    (256 parameters), Heisenberg XXX open chain; accuracy from the same structure at 30 qubits,
    complex64 against complex128."""
    import torch
    import dense_evolution as de
    from dense_evolution.workloads import hea_circuit, xxx_terms
    out = {'workload': f'{n}-qubit complex64 HEA {layers} layers, XXX open chain; adjoint gradient'}
    free = torch.cuda.mem_get_info()[0]
    if free < 3.2 * (1 << n) * 8:
        out['skipped'] = f'needs {3 * (1 << n) * 8 / 2**30:.0f} GiB of free HBM, {free / 2**30:.0f} GiB free'
        return out
    fn, npar = de.circuit_to_energy_fn(hea_circuit(n, layers), n, use_float32=True)
    op = de.PauliSumOperator(xxx_terms(n), n)
    theta = np.random.default_rng(SEED).uniform(-np.pi, np.pi, npar)
    e, g, psi = fn.program.value_and_grad(theta, op)       # warm-up (plans, scratch)
    del psi
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e, g, psi = fn.program.value_and_grad(theta, op)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    peak = torch.cuda.max_memory_allocated() / 2**30
    del psi
    torch.cuda.empty_cache()
    # algorithmic HBM bytes of one gradient: forward passes 2 2^n B, the norm read
    # 2^n B, H psi (every Pauli pass reads psi, writes or accumulates lambda),
    # the mu = psi copy 2 2^n B, backward passes 4 2^n B
    from dense_evolution.physics.observables import plan_for
    S = (1 << n) * 8
    pp = plan_for(xxx_terms(n), n, dtype=torch.complex64)
    nb = len(fn.program.back.passes)
    gbytes = (2 * fn.program.forward.npasses + 1 + (pp.npasses + 1 + 2 * (pp.npasses - 1)) + 2 + 4 * nb) * S
    out.update({'energy': e, 'grad_norm': float(np.linalg.norm(g)), 'seconds_per_gradient': dt,
                'algorithmic_bytes_per_gradient': gbytes, 'achieved_gbs': gbytes / dt / 1e9,
                'frac_of_hbm': gbytes / dt / 1e9 / _peaks()[0],
                'grads_per_s': 1.0 / dt, 'params': npar, 'peak_hbm_gib': peak,
                'forward_passes': fn.program.forward.npasses, 'backward_passes': len(fn.program.back.passes)})
    # accuracy of complex64 against complex128, same structure at 30 qubits
    th = np.random.default_rng(SEED).uniform(-np.pi, np.pi, 2 * n_ref * layers)
    r = {}
    for f32 in (True, False):
        f, _ = de.circuit_to_energy_fn(hea_circuit(n_ref, layers), n_ref, use_float32=f32)
        ee, gg, pp = f.program.value_and_grad(th, de.PauliSumOperator(xxx_terms(n_ref), n_ref))
        r[f32] = (ee, gg)
        del pp
        torch.cuda.empty_cache()
    out.update({'ref_qubits': n_ref, 'abs_energy_error_c64_vs_c128': abs(r[True][0] - r[False][0]),
                'max_abs_grad_error_c64_vs_c128': float(np.max(np.abs(r[True][1] - r[False][1])))})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=5)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--skip-vqe', action='store_true')
    ap.add_argument('--skip-cpu', action='store_true')
    ap.add_argument('--skip-batch', action='store_true')
    ap.add_argument('--skip-large', action='store_true')
    ap.add_argument('--skip-headline', action='store_true')
    ap.add_argument('--skip-fidelity', action='store_true', help='headline without the 28-qubit accuracy check')
    ap.add_argument('--skip-e2e', action='store_true', help='headline without the end-to-end leg')
    ap.add_argument('--vqe-qubits', type=int, default=VQE_N, help='VQE block width (default 24)')
    ap.add_argument('--vqe-no-shift', action='store_true', help='VQE block without the parameter-shift leg')
    ap.add_argument('--batch-circuits', type=int, default=4096, help='batch block size (default 4096)')
    ap.add_argument('--batch-no-tune', action='store_true',
                    help='skip the batch tile-width autotuner (its cached or default width is used)')
    ap.add_argument('--batch-qubits', type=int, default=0,
                    help='give every batch circuit this width (default 0: widths uniform in 10..20)')
    ap.add_argument('--qubits', type=int, default=N_QUBITS, help='headline circuit width (default 30)')
    ap.add_argument('--layers', type=int, default=LAYERS, help='headline circuit depth (default 40)')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_ours(args)


if __name__ == '__main__':
    main()
