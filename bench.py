#!/usr/bin/env python
"""Benchmark of the spectral-transform hot path on B200.

Headline workload: the spherical-harmonic transform pair (inverse then
forward, ``Grid.to_nodal`` / ``Grid.to_modal``) on Grid.TL255 (512 x 256
nodes, 257 total wavenumbers) for a batch of 128 float32 fields (32 levels x
4 variables), seeded synthetic spectral coefficients (complex Gaussians scaled
by (l+1)^-1.5, top wavenumber zeroed).  Metric: algorithmic SHT TFLOP/s,
counting the triangular Legendre work 2 * J * N_tri per field per direction.

One JSON line is printed by rank 0.  ``--impl reference`` times the CPU
restatement of the reference's Real spherical-harmonic transform (NumPy FP32
einsums, all host threads) on a bounded sample of the same workload.
Multi-GPU runs (torchrun) are independent replicas (weak scaling).
"""

from __future__ import annotations

import argparse
import functools
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = dict(name='TL255', max_wavenumber=255, gaussian_nodes=128)
FIELDS = 128
# (longitude wavenumbers, total wavenumbers, longitude nodes, latitude nodes)
GRIDS = {'TL255': (256, 257, 512, 256), 'T85': (86, 87, 256, 128)}
FORMS = ('fp32', 'bf16x3', 'tf32x3')


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# each transform phase over the 128 TL255 fields, from one ncu capture of
# `bench.py --profile-phase <phase>` per phase.
PHASE_TRAFFIC = {
    ('bf16x3', 'legendre_inverse'): 75098880 + 17449728,
    ('bf16x3', 'fourier_inverse'): 67005440 + 22596096,
    ('bf16x3', 'fourier_forward'): 67136000 + 24715264,
    ('bf16x3', 'legendre_forward'): 103041024 + 21350656,
    ('fp32', 'legendre_inverse'): 58467584 + 19169536,
    ('fp32', 'fourier_inverse'): 67005440 + 22596096,
    ('fp32', 'fourier_forward'): 67136000 + 24715264,
    ('fp32', 'legendre_forward'): 84916224 + 27469824,
    ('tf32x3', 'legendre_inverse'): 118548480 + 34110976,
    ('tf32x3', 'legendre_forward'): 151210240 + 43932416,
}


def workload_dims(name=GRID['name']):
  lw, L, I, J = GRIDS[name]
  M = 2 * lw - 1
  n_tri = L + 2 * sum(L - m for m in range(1, lw))
  return lw, L, I, J, M, n_tri


def sht_flops(fields, name=GRID['name']):
  _, _, _, J, _, n_tri = workload_dims(name)
  return 2.0 * 2.0 * J * n_tri * fields  # 2 directions x 2 flops x J x N_tri


def modal_input(fields, seed=0, name=GRID['name']):
  """Seeded complex Gaussians (Re -> cos row, Im -> sin row) * (l+1)^-1.5."""
  lw, L, _, _, M, _ = workload_dims(name)
  rng = np.random.default_rng(seed)
  re = rng.standard_normal((fields, lw, L))
  im = rng.standard_normal((fields, lw, L))
  out = np.zeros((fields, M, L))
  out[:, 0] = re[:, 0]
  out[:, 1::2] = re[:, 1:]
  out[:, 2::2] = im[:, 1:]
  m = np.concatenate([[0], np.repeat(np.arange(1, lw), 2)])
  l = np.arange(L)
  mask = m[:, None] <= l[None, :]
  out *= mask / (l + 1.0) ** 1.5
  out[..., -1] = 0
  return out.astype(np.float32)


# ---------------------------------------------------------------------------
# Clocks
# ---------------------------------------------------------------------------

class ClockSampler:
  FIELDS = ('clocks.sm,clocks.max.sm,clocks_event_reasons.active,'
            'clocks_event_reasons.hw_slowdown,'
            'clocks_event_reasons.hw_thermal_slowdown,'
            'clocks_event_reasons.sw_thermal_slowdown,'
            'clocks_event_reasons.sw_power_cap')

  def __init__(self, device_index):
    import tempfile
    self.proc = None
    self.path = os.path.join(tempfile.gettempdir(), f'dino_clocks_{os.getpid()}.csv')
    try:
      self.proc = subprocess.Popen(
          ['nvidia-smi', f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
           '-lms', '100', '-i', str(device_index), '-f', self.path],
          stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
      time.sleep(0.3)
    except (OSError, FileNotFoundError):
      self.proc = None

  def stop(self):
    if self.proc is None:
      return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
    time.sleep(0.2)
    self.proc.terminate()
    try:
      self.proc.wait(timeout=5)
    except subprocess.TimeoutExpired:
      self.proc.kill()
      self.proc.wait()
    try:
      with open(self.path) as fh:
        out = fh.read()
      os.remove(self.path)
    except OSError:
      out = ''
    sm, smax, reasons = [], None, set()
    names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
             'sw_power_cap']
    for line in out.strip().splitlines():
      parts = [p.strip() for p in line.split(',')]
      if len(parts) < 7:
        continue
      try:
        sm.append(float(parts[0]))
        smax = float(parts[1])
      except ValueError:
        continue
      for name, val in zip(names, parts[3:7]):
        if val.lower().startswith('active'):
          reasons.add(name)
    under_load = [s for s in sm if smax and s > 0.3 * smax] or sm
    return {'sm_mhz': statistics.median(under_load) if under_load else None,
            'sm_max_mhz': smax, 'reasons': sorted(reasons),
            'samples': len(sm)}


# ---------------------------------------------------------------------------
# CPU arms (oracle port of the reference's Real SHT)
# ---------------------------------------------------------------------------

def cpu_sht_pair_fn(fields, seed=1):
  """The reference's Real SHT pair in FP32 on the host: the oracle's
  restatement of spherical_harmonic.py:262-280 in the reference's contraction
  shape (one GEMM per m with the fields as N, the Fourier sums as one GEMM),
  on all host threads.  Returns (pair, x)."""
  from oracle import sht as osht  # CPU baseline only
  og = osht.Grid.TL255(compute_dtype=np.float32)
  og._gemm_basis  # tables built outside the timed region
  x = modal_input(fields, seed=seed)
  return (lambda xx: og.to_modal(og.to_nodal(xx))), x


def cpu_sht_sample(fields=FIELDS, seconds=10.0):
  """Median seconds per pair over `seconds` of repeated pairs (at least 2)."""
  pair, x = cpu_sht_pair_fn(fields)
  pair(x)
  times = []
  t_end = time.perf_counter() + seconds
  while time.perf_counter() < t_end or len(times) < 2:
    t0 = time.perf_counter()
    pair(x)
    times.append(time.perf_counter() - t0)
  return statistics.median(times), len(times)


def cpu_threads():
  """Host threads the NumPy BLAS may use (the process's CPU affinity)."""
  try:
    return len(os.sched_getaffinity(0))
  except AttributeError:
    return os.cpu_count()


def cpu_baseline_entry(seconds=10.0):
  t, reps = cpu_sht_sample(FIELDS, seconds)
  return {'value': sht_flops(FIELDS) / t / 1e12, 'unit': 'TFLOP/s',
          'cores': cpu_threads(), 'kind': 'port', 'ms_per_pair': t * 1e3,
          'sample': f'all {FIELDS} TL255 fields per pair; FP32 NumPy restatement of the '
                    'reference Real SHT in its contraction shape (per-m GEMMs over all '
                    f'fields, DFT as a GEMM); median of {reps} pairs (~{seconds:.0f} s)'}


def cpu_pe_baseline(seconds=20.0):
  """Primitive-equation steps/s of the FP64 NumPy restatement of the
  reference's filtered imex_rk_sil3 step (time_integration.py:375-405 over
  primitive_equations.py:1126-1458) on the host: T21 / 12 levels (the
  one-day configuration, timed over its first steps) and one TL255 / 32-level
  dry step."""
  from oracle import dycore as od, sht as osht, states as ost  # CPU baseline only
  out = {}
  for name, grid_name, layers, dt_min, budget in (('T21_L12', 'T21', 12, 20, seconds / 2),
                                                   ('TL255_L32_dry', 'TL255', 32, 6,
                                                    seconds / 2)):
    og = getattr(osht.Grid, grid_name)()
    st, tref, orog, vert = ost.baroclinic_config(og, layers)
    eq = od.PrimitiveEquationsSigma(tref, orog, og, vert, od.SimUnits())
    dt = od.nondim_time(dt_min * 60.0)
    step = od.step_with_filters(od.imex_rk_sil3(eq, dt),
                                [od.exponential_step_filter(og, dt)])
    # Warm-up outside the timed region: the tables and the implicit factors
    # of the three SIL3 stages (the tableau's diagonal).
    og._gemm_basis
    a_im = od.SIL3['a_im']
    for i in range(1, len(a_im) + 1):
      eq.implicit_inverse(st, dt * a_im[i - 1][i])
    n, t0 = 0, time.perf_counter()
    while n < 1 or (time.perf_counter() - t0 < budget and n < 72):
      st = step(st)
      n += 1
    sec = (time.perf_counter() - t0) / n
    out[name] = {'steps_per_s': 1.0 / sec, 'ms_per_step': sec * 1e3, 'steps_timed': n,
                 'cores': cpu_threads(), 'kind': 'port',
                 'dtype': 'f64 (the oracle; the reference\'s float32 JAX path is not '
                          'installed)'}
  return out


def run_reference(args):
  rank = int(os.environ.get('RANK', '0'))
  if rank != 0:
    return
  pair, x = cpu_sht_pair_fn(FIELDS)
  for _ in range(args.warmup):
    pair(x)
  t0 = time.perf_counter()
  for _ in range(args.steps):
    pair(x)
  t = (time.perf_counter() - t0) / args.steps
  value = sht_flops(FIELDS) / t / 1e12
  line = {
      'metric': 'SHT TFLOP/s (TL255 fwd+inv pair, 128 fields)',
      'value': value, 'unit': 'TFLOP/s', 'n_gpus': args.gpus,
      'steps': args.steps, 'warmup': args.warmup,
      'ms_per_step': t * 1e3,
      'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
      'dtype': 'f32', 'data': 'synthetic',
      'config': {'workload': 'SHT pair TL255 x 128 fields', 'grid': 'TL255',
                 'fields': FIELDS},
      'impl': 'reference',
      'cpu_baseline': {'value': value, 'unit': 'TFLOP/s',
                       'cores': cpu_threads(), 'kind': 'port',
                       'sample': f'all {FIELDS} fields per pair, {args.steps} timed pairs; '
                                 'FP32 NumPy restatement of the reference Real SHT in '
                                 'its contraction shape (JAX is not installed)'},
      'e2e': {'value': value, 'unit': 'TFLOP/s', 'h2d_bytes_per_step': 0,
              'd2h_bytes_per_step': 0},
  }
  print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Multi-rank helpers (replicas: no collective on the data path)
# ---------------------------------------------------------------------------

def gpu_local_cpus(torch, device):
  """Host CPUs of the GPU's NUMA node (sysfs local_cpulist), or None."""
  prop = torch.cuda.get_device_properties(device)
  path = '/sys/bus/pci/devices/%04x:%02x:%02x.0/local_cpulist' % (
      prop.pci_domain_id, prop.pci_bus_id, prop.pci_device_id)
  try:
    with open(path) as fh:
      text = fh.read().strip()
  except OSError:
    return None
  cpus = set()
  for part in text.split(','):
    if '-' in part:
      lo, hi = part.split('-')
      cpus.update(range(int(lo), int(hi) + 1))
    elif part:
      cpus.add(int(part))
  return cpus or None


class on_gpu_numa_node:
  """Runs the block on the GPU's NUMA-local host CPUs, so that pinned host
  buffers allocated (and first touched) inside it sit on the node the GPU's
  PCIe link attaches to; the previous CPU affinity is restored afterwards."""

  def __init__(self, device):
    import torch
    self.cpus = gpu_local_cpus(torch, device)
    self.old = None

  def __enter__(self):
    if self.cpus and hasattr(os, 'sched_setaffinity'):
      self.old = os.sched_getaffinity(0)
      use = self.cpus & self.old
      if use:
        os.sched_setaffinity(0, use)
    return self

  def __exit__(self, *exc):
    if self.old is not None:
      os.sched_setaffinity(0, self.old)
    return False


def _measured_peaks():
  try:
    with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
      return json.load(fh)
  except OSError:
    return {}


def replica_seed(rank):
  """Each replica transforms its own seeded batch."""
  return 1000 + rank


def max_over_ranks(value, device='cpu'):
  """Max of a per-rank float over the default process group (or the value)."""
  import torch
  import torch.distributed as dist
  if not (dist.is_available() and dist.is_initialized()):
    return float(value)
  t = torch.tensor([float(value)], device=device, dtype=torch.float64)
  dist.all_reduce(t, op=dist.ReduceOp.MAX)
  return float(t.item())


def aggregate_tflops(flops_per_rank, world, ms_max):
  """Whole-job throughput: every rank does flops_per_rank in ms_max."""
  return world * flops_per_rank / (ms_max * 1e-3) / 1e12


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

def phase_bytes(phase, fields, precision, name=GRID['name']):
  lw, L, I, J, M, n_tri = workload_dims(name)
  Jh = J // 2
  table_elems = Jh * sum(L - m for m in range(lw))
  # fp32 table, bf16 hi + lo (4 bytes per entry) or tf32 hi + lo (8 bytes)
  table_bytes = table_elems * (8 if precision == 'tf32x3' else 4)
  modal = fields * M * L * 4
  fourier = fields * M * J * 4
  nodal = fields * I * J * 4
  return {'legendre_inverse': modal + fourier + table_bytes,
          'fourier_inverse': fourier + nodal,
          'fourier_forward': nodal + fourier,
          'legendre_forward': fourier + modal + table_bytes}[phase]


def host_link(torch, h_in, d_in, d_out, h_out, s_in, s_out, stream, reps=5):
  """The host link under the end-to-end loop: each direction alone, and one
  step's input copied in while one step's output is copied out (two
  streams, the same pinned buffers), CUDA events on the launching stream.
  The duplex time is the floor of a pipelined end-to-end step."""
  def timed(h2d, d2h):
    for r in range(reps + 1):
      if r == 1:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
      if h2d:
        with torch.cuda.stream(s_in):
          d_in.copy_(h_in, non_blocking=True)
      if d2h:
        with torch.cuda.stream(s_out):
          h_out.copy_(d_out, non_blocking=True)
    stream.wait_stream(s_in)
    stream.wait_stream(s_out)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps
  nbytes = h_in.numel() * h_in.element_size()
  ms_in, ms_out, ms_both = timed(True, False), timed(False, True), timed(True, True)
  return {'h2d_gbs': nbytes / (ms_in * 1e-3) / 1e9,
          'd2h_gbs': nbytes / (ms_out * 1e-3) / 1e9,
          'duplex_gbs': 2 * nbytes / (ms_both * 1e-3) / 1e9,
          'step_ms': ms_both,
          'what': 'bound_tflops = algorithmic flops per step / duplex copy time of one '
                  'step\'s input and output; frac = e2e value / bound'}


def time_phases(torch, plan, x, name, reps):
  """Milliseconds per launch of each transform phase over x's fields (CUDA
  events on the launching stream, after two untimed launches)."""
  from dinosaur_b200 import _lib
  from dinosaur_b200 import spherical_harmonic as sh
  lw, L, I, J, M, _ = workload_dims(name)
  fields = x.shape[0]
  stream = torch.cuda.current_stream()
  buf_f = torch.empty((fields, M, J), device='cuda')
  buf_n = torch.empty((fields, I, J), device='cuda')
  buf_m = torch.empty((fields, M, L), device='cuda')
  phases = [('legendre_inverse', 0, x, buf_f), ('fourier_inverse', 1, buf_f, buf_n),
            ('fourier_forward', 2, buf_n, buf_f), ('legendre_forward', 3, buf_f, buf_m)]
  phase_ms = {}
  for pname, code, src, dst in phases:
    for _ in range(2):
      _lib.check(_lib.lib().dino_sht_phase(plan.handle, code, sh.ptr(src), sh.ptr(dst),
                                           fields, sh.stream_handle()))
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(reps):
      _lib.check(_lib.lib().dino_sht_phase(plan.handle, code, sh.ptr(src), sh.ptr(dst),
                                           fields, sh.stream_handle()))
    a1.record(stream)
    torch.cuda.synchronize()
    phase_ms[pname] = a0.elapsed_time(a1) / reps
  return phase_ms


def compute_peaks(torch, measured, sm_mhz=None):
  """Compute-roofline denominators: the nominal FP32 FMA rate at the SM clock
  (148 SMs x 128 lanes x 2 flops; the SIMT Legendre's bound), a cuBLAS TF32
  GEMM measured here (the split-TF32 form's), best of three; BF16 and HBM
  from the measured-peaks file."""
  prop = torch.cuda.get_device_properties(torch.cuda.current_device())
  mhz = sm_mhz or measured.get('sm_max_mhz') or 1965.0
  fp32 = prop.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
  n = 8192
  a = torch.randn(n, n, device='cuda')
  b = torch.randn(n, n, device='cuda')
  old = torch.backends.cuda.matmul.allow_tf32
  torch.backends.cuda.matmul.allow_tf32 = True
  try:
    tf32 = []
    for _ in range(3):
      for _ in range(3):
        c = a @ b
      e0 = torch.cuda.Event(enable_timing=True)
      e1 = torch.cuda.Event(enable_timing=True)
      e0.record()
      for _ in range(10):
        c = a @ b
      e1.record()
      torch.cuda.synchronize()
      tf32.append(10 * 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
  finally:
    torch.backends.cuda.matmul.allow_tf32 = old
  del a, b, c
  return {'fp32_fma_tflops': fp32, 'tf32_gemm_tflops': max(tf32),
          'bf16_gemm_tflops': measured.get('bf16_tflops'),
          'hbm_gbs': measured.get('hbm_gbs'),
          'how': f'fp32: nominal, SMs x 128 lanes x 2 x {mhz:.0f} MHz; '
                 'tf32: cuBLAS 8192^3 GEMM via torch, allow_tf32; bf16 / hbm: '
                 'MEASURED_PEAKS.json'}


def legendre_forms(torch, args, peaks):
  """Each Legendre form (plain FP32 SIMT, split-BF16, split-TF32) on the SHT
  microbenchmark at TL255 and T85 x 128 fields: pair time and TFLOP/s,
  round-trip error, per-phase times, and each Legendre phase against the HBM
  roofline (algorithmic bytes) and its arithmetic pipe's peak (folded
  2 Jh N_tri flops per field, times the 3 products of a split form)."""
  from dinosaur_b200 import spherical_harmonic as sh
  pipes = {'fp32': ('fp32 FMA (SIMT)', peaks.get('fp32_fma_tflops'), 1),
           'bf16x3': ('bf16 tensor', peaks.get('bf16_gemm_tflops'), 3),
           'tf32x3': ('tf32 tensor', peaks.get('tf32_gemm_tflops'), 3)}
  stream = torch.cuda.current_stream()
  out = {}
  for name in ('TL255', 'T85'):
    lw, L, I, J, M, n_tri = workload_dims(name)
    x = torch.as_tensor(modal_input(FIELDS, 0, name), device='cuda')
    for form in FORMS:
      impl = functools.partial(sh.CudaSphericalHarmonics, precision=form)
      # Each form as such: the plans keep their tensor-core contraction even
      # where the autotuner would choose the FP32 SIMT one.
      os.environ['DINO_B200_TENSOR_CORES_ONLY'] = '1'
      try:
        plan = getattr(sh.Grid, name)(spherical_harmonics_impl=impl).plan
      finally:
        os.environ.pop('DINO_B200_TENSOR_CORES_ONLY', None)
      for _ in range(args.warmup):
        y = plan.forward(plan.inverse(x))
      torch.cuda.synchronize()
      rt = float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x))
      b0 = torch.cuda.Event(enable_timing=True)
      b1 = torch.cuda.Event(enable_timing=True)
      b0.record(stream)
      for _ in range(args.steps):
        y = plan.forward(plan.inverse(x))
      b1.record(stream)
      torch.cuda.synchronize()
      ms = b0.elapsed_time(b1) / args.steps
      phase_ms = time_phases(torch, plan, x, name, max(5, args.steps))
      label, peak, mult = pipes[form]
      folded = FIELDS * 2.0 * ((J + 1) // 2) * n_tri
      entry = {'ms_per_pair': ms, 'tflops': aggregate_tflops(sht_flops(FIELDS, name), 1, ms),
               'round_trip_rel_l2': rt, 'phase_ms': phase_ms, 'pipe': label}
      for ph in ('legendre_inverse', 'legendre_forward'):
        t = phase_ms[ph] * 1e-3
        entry[ph] = {
            'hbm_frac': (phase_bytes(ph, FIELDS, form, name) / t / 1e9 / peaks['hbm_gbs']
                         if peaks.get('hbm_gbs') else None),
            'pipe_frac': mult * folded / t / 1e12 / peak if peak else None}
      out.setdefault(name, {})[form] = entry
      del plan, y
    del x
    torch.cuda.empty_cache()
  return out


def run_ours(args):
  import torch
  import torch.distributed as dist
  from dinosaur_b200 import _lib
  from dinosaur_b200 import spherical_harmonic as sh

  world = int(os.environ.get('WORLD_SIZE', '1'))
  rank = int(os.environ.get('RANK', '0'))
  local = int(os.environ.get('LOCAL_RANK', '0'))
  torch.cuda.set_device(local)
  if world > 1:
    import datetime
    dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))

  def barrier():
    if world > 1:
      dist.barrier()

  fields = FIELDS
  make_grid = lambda precision: sh.Grid.TL255(
      spherical_harmonics_impl=functools.partial(sh.CudaSphericalHarmonics,
                                                 precision=precision))
  grid = make_grid(args.precision)
  plan = grid.plan
  with on_gpu_numa_node(torch.cuda.current_device()):
    x_host = torch.from_numpy(modal_input(fields, seed=replica_seed(rank))).pin_memory()
  x = x_host.cuda()
  stream = torch.cuda.current_stream()

  def step():
    nodal = plan.inverse(x)
    return plan.forward(nodal)

  lw, L, I, J, M, _ = workload_dims()
  phases = {'legendre_inverse': 0, 'fourier_inverse': 1, 'fourier_forward': 2,
            'legendre_forward': 3}
  if args.profile_phase:
    # One phase over all fields, the last launch inside an NVTX range named
    # "phase" (for an ncu capture with --nvtx --nvtx-include "phase/").
    shapes = [(fields, M, L), (fields, M, J), (fields, I, J), (fields, M, J)]
    code = phases[args.profile_phase]
    src = x if code == 0 else torch.randn(shapes[code], device='cuda')
    dst = torch.empty(shapes[(code + 1) % 4], device='cuda')
    for i in range(args.warmup + 1):
      if i == args.warmup:
        torch.cuda.nvtx.range_push('phase')
      _lib.check(_lib.lib().dino_sht_phase(plan.handle, code, sh.ptr(src), sh.ptr(dst),
                                           fields, sh.stream_handle()))
      if i == args.warmup:
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    if rank == 0:
      print(json.dumps({'profile_phase': args.profile_phase}), flush=True)
    return

  for _ in range(args.warmup):
    y = step()
  torch.cuda.synchronize()
  rt_err = float(torch.linalg.vector_norm(y - x) / torch.linalg.vector_norm(x))

  # Device-resident timed region (working set ~0.3 GB > 126 MB L2).
  sampler = ClockSampler(local)
  barrier()
  torch.cuda.synchronize()
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record(stream)
  for _ in range(args.steps):
    y = step()
  e1.record(stream)
  torch.cuda.synchronize()
  barrier()
  clocks = sampler.stop()
  ms = e0.elapsed_time(e1) / args.steps
  if args.profile:
    if rank == 0:
      print(json.dumps({'profile_ms_per_step': ms}), flush=True)
    if world > 1:
      dist.destroy_process_group()
    return
  ms_max = max_over_ranks(ms, device='cuda')
  value = aggregate_tflops(sht_flops(fields), world, ms_max)

  # End to end through the public API with pinned host buffers: every step
  # copies its input batch in, runs Grid.to_nodal / Grid.to_modal and copies
  # the result out.  Consecutive steps are pipelined on three streams
  # (copy-in, transforms, copy-out) with double-buffered device arrays, so
  # the full-duplex host link carries one step's input while the previous
  # step's output drains.
  with on_gpu_numa_node(torch.cuda.current_device()):
    out_host = torch.empty_like(x_host).pin_memory()
  s_in = torch.cuda.Stream()
  s_out = torch.cuda.Stream()
  xs = [torch.empty_like(x) for _ in range(2)]
  ys = [torch.empty_like(x) for _ in range(2)]
  ev_in = [torch.cuda.Event() for _ in range(2)]
  ev_done = [torch.cuda.Event() for _ in range(2)]
  ev_out = [torch.cuda.Event() for _ in range(2)]
  for e in ev_out:
    e.record(s_out)

  def e2e_steps(n):
    s_in.wait_stream(stream)
    for i in range(n):
      b = i % 2
      with torch.cuda.stream(s_in):
        s_in.wait_event(ev_done[b])  # the transforms finished reading xs[b]
        xs[b].copy_(x_host, non_blocking=True)
        ev_in[b].record(s_in)
      stream.wait_event(ev_in[b])
      stream.wait_event(ev_out[b])   # ys[b] has been copied out
      yd = grid.to_modal(grid.to_nodal(xs[b]))
      ys[b].copy_(yd)
      ev_done[b].record(stream)
      with torch.cuda.stream(s_out):
        s_out.wait_event(ev_done[b])
        out_host.copy_(ys[b], non_blocking=True)
        ev_out[b].record(s_out)
    stream.wait_stream(s_out)

  # Untimed warm-up of the pipelined loop (allocator, streams), then the
  # timed steps.
  e2e_steps(args.warmup)
  barrier()
  torch.cuda.synchronize()
  e2 = torch.cuda.Event(enable_timing=True)
  e3 = torch.cuda.Event(enable_timing=True)
  e2.record(stream)
  e2e_steps(args.steps)
  e3.record(stream)
  torch.cuda.synchronize()
  barrier()
  ms_e2e = max_over_ranks(e2.elapsed_time(e3) / args.steps, device='cuda')
  e2e_value = aggregate_tflops(sht_flops(fields), world, ms_e2e)
  e2e_err = float(torch.linalg.vector_norm(out_host.cuda() - y) /
                  torch.linalg.vector_norm(y))
  link = host_link(torch, x_host, xs[0], ys[1], out_host, s_in, s_out, stream)
  link['bound_tflops'] = aggregate_tflops(sht_flops(fields), world, link['step_ms'])
  link['frac'] = e2e_value / link['bound_tflops']

  # Per-phase kernel timing (live CUDA events on the launching stream).
  phase_ms = time_phases(torch, plan, x, GRID['name'], max(5, args.steps))
  dominant = max(phase_ms, key=phase_ms.get)
  peaks = {}
  try:
    with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
      peaks = json.load(fh)
  except OSError:
    pass
  hbm_peak = peaks.get('hbm_gbs', 6650.0)
  peak_src = 'measured' if 'hbm_gbs' in peaks else 'fallback'
  achieved = phase_bytes(dominant, fields, args.precision) / (phase_ms[dominant] * 1e-3) / 1e9
  per_field = M * J * 4
  cap = max(1, (48 << 20) // per_field)
  chunks = -(-fields // min(cap, plan.max_fields))
  # Per chunk: inverse Legendre, inverse FFT, forward FFT, forward Legendre
  # (the split forms' operand split and fold run inside the Legendre kernels).
  launches_per_step = chunks * 4

  extra = {}
  if not args.no_extra and world == 1:
    # Every Legendre form at TL255 and T85 with its rooflines; the other
    # forms' TL255 pairs are also listed as sht_<form>.
    extra['peaks'] = compute_peaks(torch, peaks, clocks.get('sm_mhz'))
    extra['legendre_forms'] = legendre_forms(torch, args, extra['peaks'])
    for other in [f for f in FORMS if f != args.precision]:
      e = extra['legendre_forms']['TL255'][other]
      extra['sht_' + other] = {'value': e['tflops'], 'unit': 'TFLOP/s',
                               'ms_per_step': e['ms_per_pair'],
                               'round_trip_rel_l2': e['round_trip_rel_l2']}
    extra.update(pe_extras(torch))

  if rank == 0:
    line = {
        'metric': 'SHT TFLOP/s (TL255 fwd+inv pair, 128 fields)',
        'value': value, 'unit': 'TFLOP/s', 'n_gpus': world,
        'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': ms_max,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32' if args.precision == 'fp32' else args.precision + '->f32',
        'data': 'synthetic',
        'config': {'workload': 'SHT pair TL255 x 128 fields', 'grid': 'TL255',
                   'fields': fields, 'precision': args.precision,
                   'plan': plan.describe(),
                   'parallelism': f'replicas x{world}',
                   'l2': 'working set ~0.3 GB per step > 126 MB L2 (no flush)'},
        'e2e': {'value': e2e_value, 'unit': 'TFLOP/s',
                'h2d_bytes_per_step': int(x_host.numel() * 4),
                'd2h_bytes_per_step': int(out_host.numel() * 4),
                'pipelined': 'copy-in / transforms / copy-out streams',
                'host_buffers': ('pinned, on the GPU NUMA node'
                                 if gpu_local_cpus(torch, torch.cuda.current_device())
                                 else 'pinned'),
                'result_matches_device_run': e2e_err == 0.0,
                'link': link},
        'roofline': {'bound': 'hbm', 'kernel': dominant, 'achieved': achieved,
                     'peak': hbm_peak, 'unit': 'GB/s',
                     'frac': achieved / hbm_peak, 'peak_source': peak_src,
                     'traffic': PHASE_TRAFFIC.get((args.precision, dominant)),
                     'traffic_unit': 'bytes per launch (ncu, one capture)',
                     'phase_ms': phase_ms},
        'clocks': clocks,
        'gpu_launches': launches_per_step * args.steps,
        'round_trip_rel_l2': rt_err,
    }
    if world == 1 and not args.no_cpu_baseline:
      line['cpu_baseline'] = cpu_baseline_entry()
      if extra:
        extra['cpu_pe'] = cpu_pe_baseline()
    if extra:
      line['extra'] = extra
    print(json.dumps(line), flush=True)
  if world > 1:
    dist.destroy_process_group()


def pe_step_bytes(eng, grid_name):
  """Algorithmic HBM bytes of one filtered SIL3 step of the unfused phase
  sequence: every phase reads its inputs and writes its outputs once.

  Per explicit evaluation (3 per step): the modal pre-pass (state in,
  auxiliary planes out), the inverse transform (n_inv modal in, n_inv nodal
  out, Legendre table), the nodal column kernel (n_inv in, n_fwd out), the
  forward transform (n_fwd nodal in, n_fwd modal out, table) and the modal
  post-pass (n_fwd modal and the state in, a tendency out).  The Fourier
  intermediates are not counted (chunks are sized to stay in L2).  Implicit
  part: the four operator products read their n_impl implicit planes and
  write n_impl (2 n_impl for the stage that also forms G Y2); the three
  combines read y0 and 1, 2, 3 explicit tendencies plus 1, 1, 2 implicit
  ones and write a state."""
  import ctypes
  from dinosaur_b200 import _lib
  counts = (ctypes.c_int32 * 5)()
  _lib.check(_lib.lib().dino_pe_counts(eng.handle, counts), 'dino_pe_counts')
  n_state, n_aux, n_inv, n_fwd, n_impl = list(counts)
  lw, L, I, J, M, _ = workload_dims_any(grid_name)
  ml, ij = M * L * 4, I * J * 4
  table = 4 * ((J + 1) // 2) * sum(L - m for m in range(lw))
  explicit = ((n_state + n_aux) + n_inv + 2 * n_fwd + n_state) * ml + \
      (2 * n_inv + 2 * n_fwd) * ij + 2 * table
  implicit = 9 * n_impl * ml + (3 * n_state + 4 * n_state + 5 * n_state) * ml + \
      (1 + 1 + 2) * n_impl * ml
  return 3 * explicit + implicit


def workload_dims_any(name):
  """(lw, L, I, J, M, N_tri) of a standard Grid by name (T / TL)."""
  if name in GRIDS:
    return workload_dims(name)
  linear = name.startswith('TL')
  tmax = int(name[2:] if linear else name[1:])
  gaussian = {21: 16, 31: 24, 42: 32, 85: 64, 63: 32, 127: 64, 255: 128}[tmax]
  lw, L, I, J = tmax + 1, tmax + 2, 4 * gaussian, 2 * gaussian
  M = 2 * lw - 1
  return lw, L, I, J, M, L + 2 * sum(L - m for m in range(1, lw))


def pe_extras(torch):
  """Primitive-equation steps/s on the benchmark grids (CUDA-graph replay).

  Synthetic states near rest (seeded small modal noise); the moist case adds
  specific humidity (5 g/kg mean) and two passive tracers.  Each case runs
  with the plain FP32 and the split-BF16 Legendre contraction where both are
  listed (the dry TL255 case also with split-TF32, and on 32 analytic hybrid
  sigma-pressure levels with split-BF16)."""
  from dinosaur_b200 import coordinate_systems, held_suarez, primitive_equations as pe
  from dinosaur_b200 import hybrid_coordinates
  from dinosaur_b200 import sigma_coordinates, spherical_harmonic as sh
  from dinosaur_b200 import time_integration as ti, units
  out = {}
  cases = [
      # name, grid, layers, members, held_suarez, moist, dt [min], precision
      ('T42_L24_x16_held_suarez', 'T42', 24, 16, True, False, 15, 'fp32'),
      ('T42_L24_x16_held_suarez_bf16x3', 'T42', 24, 16, True, False, 15, 'bf16x3'),
      ('TL255_L32_dry', 'TL255', 32, 1, False, False, 6, 'fp32'),
      ('TL255_L32_dry_bf16x3', 'TL255', 32, 1, False, False, 6, 'bf16x3'),
      ('TL255_L32_dry_tf32x3', 'TL255', 32, 1, False, False, 6, 'tf32x3'),
      ('TL255_L32_hybrid_dry_bf16x3', 'TL255', 32, 1, False, False, 6, 'bf16x3'),
      ('TL255_L32_moist3_x4', 'TL255', 32, 4, False, True, 6, 'fp32'),
      ('TL255_L32_moist3_x4_bf16x3', 'TL255', 32, 4, False, True, 6, 'bf16x3'),
  ]
  for name, grid_name, layers, members, hs, moist, dt_min, precision in cases:
    impl = functools.partial(sh.CudaSphericalHarmonics, precision=precision)
    g = getattr(sh.Grid, grid_name)(spherical_harmonics_impl=impl)
    hybrid = 'hybrid' in name
    vert = (hybrid_coordinates.HybridCoordinates.analytic_levels(layers) if hybrid
            else sigma_coordinates.SigmaCoordinates.equidistant(layers))
    coords = coordinate_systems.CoordinateSystem(g, vert)
    ps = units.SimUnits()
    tref = np.full(layers, 285.0) if hs else np.linspace(220.0, 288.0, layers)
    eq_cls = pe.PrimitiveEquationsHybrid if hybrid else pe.PrimitiveEquationsSigma
    eq = eq_cls(tref, np.zeros(g.modal_shape, np.float32), coords, ps,
                humidity_key='specific_humidity' if moist else None)
    if hs:
      eq = ti.compose_equations([eq, held_suarez.HeldSuarezForcingSigma(coords, ps, tref)])
    dt = units.nondim_time(dt_min * 60.0)
    if hs:
      flt = ti.exponential_step_filter(g, dt, tau=0.0087504, order=1.5, cutoff=0.8)
    else:
      flt = ti.exponential_step_filter(g, dt)
    step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt), [flt])
    rng = np.random.default_rng(0)
    lead = (members, layers) if members > 1 else (layers,)
    shape = lead + g.modal_shape
    lshape = ((members, 1) if members > 1 else (1,)) + g.modal_shape
    _, l = g.modal_mesh
    scale = g.mask / (l + 1.0) ** 2
    noise = lambda s, a=1e-4: (a * rng.standard_normal(s) * scale).astype(np.float32)
    t = lambda a: torch.as_tensor(a, device='cuda')
    tracers = {}
    if moist:
      const = np.zeros(shape, np.float32)
      const[..., 0, 0] = 2.0 * np.sqrt(np.pi)  # the constant field 1
      tracers = {'specific_humidity': t(5e-3 * const + noise(shape, 1e-6)),
                 'tracer_a': t(const + noise(shape)),
                 'tracer_b': t(const + noise(shape))}
    lnps = noise(lshape)
    if hybrid:
      # Hybrid levels need a physical surface pressure: 1e5 Pa as the l = 0
      # term (the constant field 1 has the coefficient 2 sqrt(pi)).
      lnps[..., 0, 0] += np.log(units.nondim_pressure(1e5)) * 2.0 * np.sqrt(np.pi)
    state = pe.State(t(noise(shape)), t(noise(shape)), t(noise(shape)),
                     t(lnps), tracers=tracers)
    eng = eq.engine(state)
    buf = eng.pack(state)
    eng.step_(buf, dt, step.filter_scaling, 3, graph=True)
    torch.cuda.synchronize()
    n = 10 if 'moist' in name else (20 if grid_name == 'TL255' else 60)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record()
    eng.step_(buf, dt, step.filter_scaling, n, graph=True)
    a1.record()
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / n
    nbytes = pe_step_bytes(eng, grid_name)
    hbm = _measured_peaks().get('hbm_gbs', 6650.0)
    out[name] = {'ms_per_step': ms, 'steps_per_s': 1e3 / ms,
                 'member_steps_per_s': members * 1e3 / ms,
                 'precision': precision, 'plan': g.plan.describe(),
                 'algorithmic_bytes_per_step': nbytes,
                 'hbm_frac': nbytes / (ms * 1e-3) / 1e9 / hbm,
                 'finite': bool(torch.isfinite(buf).all())}
    del eng, buf, state, eq
    torch.cuda.empty_cache()
  out.update(small_and_gradient_cases(torch))
  out.update(large_gradient_case(torch))
  return out


def large_gradient_case(torch):
  """The reverse pass of the large configuration: 12 filtered SIL3 steps of
  TL255 / 32 levels, moist with two passive tracers, 4 members, split-BF16
  Legendre -- forward with per-step checkpoints, then the step VJPs."""
  from dinosaur_b200 import coordinate_systems, primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates, spherical_harmonic as sh
  from dinosaur_b200 import time_integration as ti, units
  layers, members, steps = 32, 4, 12
  impl = functools.partial(sh.CudaSphericalHarmonics, precision='bf16x3')
  g = sh.Grid.TL255(spherical_harmonics_impl=impl)
  coords = coordinate_systems.CoordinateSystem(
      g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
  eq = pe.PrimitiveEquationsSigma(np.linspace(220.0, 288.0, layers),
                                  np.zeros(g.modal_shape, np.float32), coords,
                                  units.SimUnits(), humidity_key='specific_humidity')
  dt = units.nondim_time(6 * 60.0)
  step = ti.repeated(ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                                          [ti.exponential_step_filter(g, dt)]), steps)
  rng = np.random.default_rng(2)
  _, l = g.modal_mesh
  scale = g.mask / (l + 1.0) ** 2
  shape = (members, layers) + g.modal_shape
  noise = lambda s, a=1e-4: torch.as_tensor((a * rng.standard_normal(s) * scale)
                                            .astype(np.float32), device='cuda')
  const = np.zeros(shape, np.float32)
  const[..., 0, 0] = 2.0 * np.sqrt(np.pi)
  const = torch.as_tensor(const, device='cuda')

  # Inputs are generated once, outside the timed region.
  base = [noise(shape), noise(shape), noise(shape), noise((members, 1) + g.modal_shape)]
  tracers = {'specific_humidity': 5e-3 * const + noise(shape, 1e-6),
             'tracer_a': const + noise(shape), 'tracer_b': const + noise(shape)}

  def run():
    leaves = [b.clone().requires_grad_(True) for b in base]
    x = pe.State(*leaves, tracers=tracers)
    y = step(x)
    loss = (y.temperature_variation ** 2).mean() + (y.vorticity ** 2).mean()
    loss.backward()
    return bool(all(torch.isfinite(t.grad).all() for t in leaves))

  run()
  torch.cuda.synchronize()
  a0 = torch.cuda.Event(enable_timing=True)
  a1 = torch.cuda.Event(enable_timing=True)
  a0.record()
  finite = run()
  a1.record()
  torch.cuda.synchronize()
  ms = a0.elapsed_time(a1)
  return {'TL255_L32_moist3_x4_bf16x3_grad_12_steps': {
      'ms_per_rollout': ms, 'steps': steps, 'members': members,
      'precision': 'bf16x3', 'what': 'forward (checkpointed) + reverse sweep',
      'finite': finite}}


def small_and_gradient_cases(torch):
  """T21 / 12 levels, 72 filtered steps (one day at dt = 20 min) from a
  near-rest state; and the gradient of a tracking loss through 24 steps of
  T42 / 20 levels (forward with per-step checkpoints + reverse sweep)."""
  from dinosaur_b200 import coordinate_systems, primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates, spherical_harmonic as sh
  from dinosaur_b200 import time_integration as ti, units
  out = {}
  for name, grid_name, layers, steps, grad in [('T21_L12_72_steps', 'T21', 12, 72, False),
                                                ('T42_L20_grad_24_steps', 'T42', 20, 24, True)]:
    g = getattr(sh.Grid, grid_name)()
    coords = coordinate_systems.CoordinateSystem(
        g, sigma_coordinates.SigmaCoordinates.equidistant(layers))
    tref = np.linspace(220.0, 288.0, layers)
    eq = pe.PrimitiveEquationsSigma(tref, np.zeros(g.modal_shape, np.float32), coords,
                                    units.SimUnits())
    dt = units.nondim_time(20 * 60.0)
    step = ti.repeated(ti.step_with_filters(ti.imex_rk_sil3(eq, dt),
                                            [ti.exponential_step_filter(g, dt)]), steps)
    rng = np.random.default_rng(1)
    _, l = g.modal_mesh
    scale = g.mask / (l + 1.0) ** 2
    shape = (layers,) + g.modal_shape
    t = lambda s: torch.as_tensor((1e-4 * rng.standard_normal(s) * scale).astype(np.float32),
                                  device='cuda')
    leaves = [t(shape), t(shape), t(shape), t((1,) + g.modal_shape)]
    target = [t(shape) for _ in range(2)]

    def run():
      x = pe.State(*[v.clone().requires_grad_(grad) for v in leaves])
      y = step(x)
      if grad:
        loss = (((y.temperature_variation - target[0]) ** 2).mean() +
                ((y.vorticity - target[1]) ** 2).mean())
        loss.backward()
      return y

    for _ in range(2):
      run()
    torch.cuda.synchronize()
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    reps = 3
    a0.record()
    for _ in range(reps):
      y = run()
    a1.record()
    torch.cuda.synchronize()
    ms = a0.elapsed_time(a1) / reps
    entry = {'ms_per_rollout': ms, 'steps': steps, 'precision': 'fp32',
             'finite': bool(torch.isfinite(y.vorticity).all())}
    if grad:
      entry['what'] = 'forward (checkpointed) + reverse sweep'
    else:
      entry['steps_per_s'] = steps * 1e3 / ms
    out[name] = entry
  return out


def run_pe_profile(args):
  """Eager (no CUDA graph) filtered SIL3 steps of the primitive equations, so
  that a kernel profiler sees every launch: seeded small random states on
  the chosen grid, levels and members.  Prints the mean step time."""
  import torch
  from dinosaur_b200 import coordinate_systems, held_suarez, hybrid_coordinates
  from dinosaur_b200 import primitive_equations as pe
  from dinosaur_b200 import sigma_coordinates, spherical_harmonic as sh
  from dinosaur_b200 import time_integration as ti, units
  impl = functools.partial(sh.CudaSphericalHarmonics, precision=args.precision)
  g = getattr(sh.Grid, args.pe_grid)(spherical_harmonics_impl=impl)
  layers, members = args.pe_layers, args.pe_members
  vert = (hybrid_coordinates.HybridCoordinates.analytic_levels(layers) if args.pe_hybrid
          else sigma_coordinates.SigmaCoordinates.equidistant(layers))
  coords = coordinate_systems.CoordinateSystem(g, vert)
  ps = units.SimUnits()
  hs = args.pe_held_suarez
  tref = np.full(layers, 285.0) if hs else np.linspace(220.0, 288.0, layers)
  eq_cls = pe.PrimitiveEquationsHybrid if args.pe_hybrid else pe.PrimitiveEquationsSigma
  eq = eq_cls(tref, np.zeros(g.modal_shape, np.float32), coords, ps,
              humidity_key='specific_humidity' if args.pe_moist else None)
  if hs:
    eq = ti.compose_equations([eq, held_suarez.HeldSuarezForcingSigma(coords, ps, tref)])
  dt = units.nondim_time(args.pe_dt_minutes * 60.0)
  flt = (ti.exponential_step_filter(g, dt, tau=0.0087504, order=1.5, cutoff=0.8) if hs
         else ti.exponential_step_filter(g, dt))
  step = ti.step_with_filters(ti.imex_rk_sil3(eq, dt), [flt])
  rng = np.random.default_rng(0)
  lead = (members,) if members > 1 else ()
  _, l = g.modal_mesh
  scale = g.mask / (l + 1.0) ** 2
  dev = lambda a: torch.as_tensor(np.asarray(a, np.float32), device='cuda')
  noise = lambda shp, a=1e-4: dev(a * rng.standard_normal(shp) * scale)
  shape = lead + (layers,) + g.modal_shape
  tracers = {}
  if args.pe_moist:
    const = np.zeros(shape, np.float32)
    const[..., 0, 0] = 2.0 * np.sqrt(np.pi)  # the constant field 1
    tracers = {'specific_humidity': dev(5e-3 * const) + noise(shape, 1e-6),
               'tracer_a': dev(const) + noise(shape), 'tracer_b': dev(const) + noise(shape)}
  lnps = noise(lead + (1,) + g.modal_shape)
  if args.pe_hybrid:
    # A physical surface pressure (1e5 Pa) as the l = 0 term.
    lnps[..., 0, 0] += float(np.log(units.nondim_pressure(1e5)) * 2.0 * np.sqrt(np.pi))
  state = pe.State(noise(shape), noise(shape), noise(shape), lnps, tracers=tracers)
  eng = eq.engine(state)
  buf = eng.pack(state)
  eng.step_(buf, dt, step.filter_scaling, max(1, args.warmup), graph=False)
  torch.cuda.synchronize()
  e0 = torch.cuda.Event(enable_timing=True)
  e1 = torch.cuda.Event(enable_timing=True)
  e0.record()
  eng.step_(buf, dt, step.filter_scaling, args.steps, graph=False)
  e1.record()
  torch.cuda.synchronize()
  print(json.dumps({'pe_profile': {
      'grid': args.pe_grid, 'layers': layers, 'members': members, 'held_suarez': hs,
      'moist': args.pe_moist, 'hybrid': args.pe_hybrid, 'precision': args.precision,
      'us_per_step_eager': e0.elapsed_time(e1) / args.steps * 1e3,
      'finite': bool(torch.isfinite(buf).all())}}), flush=True)


def main():
  ap = argparse.ArgumentParser()
  ap.add_argument('--gpus', type=int, default=1)
  ap.add_argument('--steps', type=int, default=20)
  ap.add_argument('--warmup', type=int, default=5)
  ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
  ap.add_argument('--precision', default=os.environ.get('DINO_BENCH_PRECISION', 'bf16x3'),
                  choices=['fp32', 'bf16x3', 'tf32x3'])
  ap.add_argument('--no-extra', action='store_true')
  ap.add_argument('--no-cpu-baseline', action='store_true')
  ap.add_argument('--profile', action='store_true',
                  help='only the device-resident timed loop (for ncu captures)')
  ap.add_argument('--profile-phase', default=None,
                  choices=['legendre_inverse', 'fourier_inverse', 'fourier_forward',
                           'legendre_forward'],
                  help='only one transform phase over all fields (for ncu captures)')
  pe_grp = ap.add_argument_group(
      'primitive-equation step profiling (eager launches, for a kernel profiler)')
  pe_grp.add_argument('--pe-grid', default=None, help='e.g. T42 or TL255')
  pe_grp.add_argument('--pe-layers', type=int, default=24)
  pe_grp.add_argument('--pe-members', type=int, default=1)
  pe_grp.add_argument('--pe-held-suarez', action='store_true')
  pe_grp.add_argument('--pe-moist', action='store_true',
                      help='specific humidity and two passive tracers')
  pe_grp.add_argument('--pe-hybrid', action='store_true',
                      help='analytic hybrid sigma-pressure levels')
  pe_grp.add_argument('--pe-dt-minutes', type=float, default=15.0)
  args = ap.parse_args()
  if args.pe_grid:
    run_pe_profile(args)
    return
  if args.warmup < 3:
    args.warmup = 3
  if args.impl == 'reference':
    run_reference(args)
  else:
    run_ours(args)


if __name__ == '__main__':
  main()
