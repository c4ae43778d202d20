#!/usr/bin/env python3
"""
bench.py -- windows/s of framecor's Correlator.correlate on B200s.

Workload (the 720p configuration): a seeded synthetic 300-frame 720 x 1280 uint8 video (smoothed
texture, 0.5 px random-walk camera, a 0 -> 40 px fault step over frames 100-130), the reference
frame 0, the window grid of window_grid(720, 1280, 64, 48, 16) (35 x 70 = 2450 windows of 64 px,
search +-48 px), per-frame gross offsets = the rounded camera motion. One step = one correlate
call on a batch of 16 frames (39,200 windows); steps walk through the video.

  value       device-timed (CUDA events, max over ranks): frames already in HBM, the device entry
              point of the C ABI, in the form chosen by --form (default: the tensor-core form with
              its exact peak refinement, the library's default at this geometry)
  e2e         the host entry point with pageable numpy frames (as the reference's callers pass
              them) -> outputs in numpy arrays, host->device and device->host copies inside the
              timed region; e2e_pinned the same from page-locked frames
  roofline    the correlation kernel's achieved rate over its own CUDA-event time, by the unit of
              work of the form: useful DFT-GEMM FLOPs per window for the tensor-core form (against
              the measured bf16 tensor peak), useful FFT FLOPs for the FP32 form, 2 W^2 M^2 integer
              ops for the exact form; traffic from one ncu capture of the same launch
  accuracy    the timed step's outputs against the exact integer form on the whole step and against
              the FP64 oracle on a sub-grid
  other_forms the same step in the other forms
  cpu_baseline the reference's CPU backend (its own sources, FFT by the oracle's shim) on 2 frames

--impl reference: the reference's CPU backend alone (rank 0), one frame per step.
--gpus N: each rank correlates its own batches (no collective in the data path); run without a
launcher, bench.py starts its N ranks itself through torch.distributed.run.
--workload: the other configurations (mixed grids, 1080p streaming, the differentiable path,
stabilize, auto_slip's scans), one JSON line each.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'windows/s at 720p 64px ±48: TC split-precision vs FP32 FFT, ≤0.01 px err'
H, W_, WIN, SEARCH, SKIP, BATCH, NFRAMES = 720, 1280, 64, 48, 16, 16, 300
PUBLISHED_WPS = 2450 / 0.022   # framecor CUDA (cuFFT), RTX 4060 laptop, 22 ms per 720p frame


def fft_flops(n):
    """useful FP32 work of one window: forward + inverse 2-D real FFT of n x n, conj product"""
    return 2 * 2.5 * n * n * np.log2(n * n) + 6 * n * (n // 2 + 1)


def tc_flops(n, m):
    """executed tensor-core FLOPs of one window in the DFT-GEMM form (FFT size n, m shifts per
    axis): the five GEMM stages with their 128-row tiles and 16-column padding"""
    kp = (n // 2 + 1 + 15) // 16 * 16
    no = (m + 15) // 16 * 16
    t1 = (n + 127) // 128
    return 4 * 128 * t1 * kp * n + 8 * 128 * n * n + 8 * 128 * no * n + 4 * 128 * no * kp


class Clocks:
    """nvidia-smi samples of one GPU while running."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')
    NAMES = ('hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap')

    def __init__(self, device):
        self.device, self.lines, self.proc = device, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--query-gpu={self.FIELDS}', '--format=csv,noheader,nounits',
                                          '-lms', '200', '-i', str(self.device)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=lambda: self.lines.extend(self.proc.stdout), daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        for line in self.lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, f[5:9]):
                if flag.lower().startswith('active'):
                    reasons.add(name)
        if not sm:
            return None
        return {'sm_mhz': statistics.median(sm), 'sm_max_mhz': max(mx), 'reasons': sorted(reasons),
                'samples': len(sm)}


# dram bytes per 16-frame launch of the correlation kernel (dram__bytes_read.sum + dram__bytes_write.sum
# of one ncu capture of this workload's launch, per form)
TRAFFIC_PER_LAUNCH = {("fft32", 160): 328990464, ("tc", 160): 380023808}


def dft_gemm_flops(n, m):
    """useful DFT-GEMM work of one window (FFT size n, m shifts per axis), one pass at the GEMM form's
    operand sizes: forward row real DFT 4 n^2 (n/2+1) + column complex DFT 8 n^2 (n/2+1); inverse pruned to the m
    output rows and columns, column 8 m n (n/2+1) + row 4 m^2 (n/2+1) (38.0 MFLOP at n = 160, m = 97)"""
    nh = n // 2 + 1
    return 4 * n * n * nh + 8 * n * n * nh + 8 * m * n * nh + 4 * m * m * nh


def direct_ops(w, m):
    """useful integer work of one window in the exact form: w^2 multiply-adds for each of m^2 shifts"""
    return 2 * w * w * m * m


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            return json.load(f)
    except OSError:
        return {}


def reference_cpu(frames, gross, down, across, nframes):
    """windows/s of the reference CPU backend on nframes frames; (value, seconds, cores)."""
    from oracle import oracle
    mod = oracle.reference_module()
    kind = 'reference'
    if mod is None:
        kind = 'port'
    cores = os.cpu_count()
    if mod is not None:
        cor = mod.Correlator(H, W_, list(down), list(across), window=WIN, search=SEARCH, backend='cpu')
        cor.set_reference(frames[0])
        t = time.perf_counter()
        cor.correlate(frames[1:1 + nframes], gross=gross[1:1 + nframes])
        dt = time.perf_counter() - t
    else:
        t = time.perf_counter()
        oracle.correlate(H, W_, down, across, frames[0], frames[1:1 + nframes], gross[1:1 + nframes],
                         window=WIN, search=SEARCH, mode='ref32')
        dt = time.perf_counter() - t
    return nframes * len(down) * len(across) / dt, dt, cores, kind


def reference_cuda(workload='hd'):
    """The reference's own CUDA backend (cuFFT) on this GPU, on the same workload through its own API
    (host arrays, 64 frames): oracle/ref_cuda_bench.py in a process of its own."""
    import subprocess
    try:
        r = subprocess.run([sys.executable, os.path.join(os.path.dirname(os.path.abspath(__file__)), 'oracle',
                                                         'ref_cuda_bench.py'), '--workload', workload],
                           capture_output=True, text=True, timeout=300)
        return json.loads(r.stdout.strip().splitlines()[-1])
    except Exception as e:   # a baseline only: its absence does not stop the line
        return {'unavailable': f'{type(e).__name__}: {e}'[:200]}


def run_reference(args):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    from slipcam_b200 import synth
    from slipcam_b200.framecor import window_grid
    down, across = window_grid(H, W_, WIN, SEARCH, SKIP)
    nwin = len(down) * len(across)
    need = args.warmup + args.steps + 1
    frames, motion, step, gross = synth.hd(n=NFRAMES, count=min(NFRAMES, need))
    from oracle import oracle
    mod = oracle.reference_module()
    if mod is None:
        print(json.dumps({'impl': 'reference', 'unavailable': 'the reference CPU module (oracle/_ref) is not built'}))
        return
    cor = mod.Correlator(H, W_, list(down), list(across), window=WIN, search=SEARCH, backend='cpu')
    cor.set_reference(frames[0])
    k = 1
    for _ in range(args.warmup):
        cor.correlate(frames[k:k + 1], gross=gross[k:k + 1])
        k = 1 + k % (len(frames) - 1)
    t = time.perf_counter()
    for _ in range(args.steps):
        cor.correlate(frames[k:k + 1], gross=gross[k:k + 1])
        k = 1 + k % (len(frames) - 1)
    dt = time.perf_counter() - t
    value = args.steps * nwin / dt
    out = {'impl': 'reference', 'metric': METRIC, 'value': value, 'unit': 'windows/s', 'n_gpus': args.gpus,
           'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': dt / args.steps * 1e3,
           'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': value / PUBLISHED_WPS, 'dtype': 'f32',
           'data': 'synthetic',
           'config': {'workload': '720p video, window 64, search 48, skip 16 (2450 windows/frame), per-frame gross',
                      'frames_per_step': 1, 'windows_per_step': nwin, 'backend': 'reference cpu (FFTW-API shim)'},
           'cpu_baseline': {'value': value, 'unit': 'windows/s', 'cores': os.cpu_count(), 'kind': 'reference',
                            'sample': f'{args.steps} frames, one per step, OpenMP on all cores'},
           'e2e': {'value': value, 'unit': 'windows/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(out))


def shard_starts(rank, world, nframes, batch, count):
    """The first frames of the `count` batches that rank takes from a video of nframes frames (frame 0
    the reference): batch b (frames 1 + b batch ...) goes to rank b % world, so the ranks' batches
    are disjoint until the video is used up, then they wrap around. No data crosses ranks."""
    nb = (nframes - 1) // batch
    if nb < 1:
        raise ValueError('the video holds no full batch')
    return [1 + ((rank + world * i) % nb) * batch for i in range(count)]


def max_over_ranks(x, dist, device):
    """x's maximum over the ranks (the slowest rank's time); x itself with one rank"""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def accuracy(cor, frames, gross, gross_d, down, across, step_start, form, batch):
    """The chosen form's offsets on the timed workload: every pair of one whole 16-frame step against
    the exact integer form (whose offsets are the FP64 oracle's within 1e-4 px on every golden case)
    and the FP32 form, and over 2,000 pairs against the FP64 direct-correlation oracle (frames 100, 110,
    120 and 130, where the fault step ramps through 0 .. 40 px, and the step's first frame, on a
    sub-grid of every second row and third column of windows), with the windows whose search region
    straddles the fault line reported apart."""
    import math

    import torch

    from oracle import oracle

    def stats(d, snr_rel):
        d = np.asarray(d, float)
        return {'pairs': int(d.size), 'max_px': float(d.max()), 'p99_px': float(np.quantile(d, 0.99)),
                'median_px': float(np.median(d)), 'frac_above_0.01px': float((d > 0.01).mean()),
                'snr_rel_max': float(np.max(snr_rel)), 'snr_rel_p99': float(np.quantile(snr_rel, 0.99))}

    out = {}
    s = step_start
    f, g = frames[s:s + batch], gross_d[s:s + batch]

    def versus(a, b):   # a against b on every pair of the step that b finds valid
        ao, bo = a['offsets'].cpu().numpy(), b['offsets'].cpu().numpy()
        valid = np.isfinite(bo[..., 0])
        d = np.abs(ao - bo).max(-1)[valid]
        snr = np.abs(a['snr'].cpu().numpy()[valid] / b['snr'].cpu().numpy()[valid] - 1)
        ok = d <= 0.5
        return dict(stats(d[ok], snr[ok]), integer_peak_mismatches=int((d > 0.5).sum()), frames=f'{s}..{s + batch - 1}')

    a = cor.correlate(f, gross=g)
    for ref_form in ('int8', 'fft32'):   # the exact integer form (the FP64 oracle's results to 1e-4 px), FP32
        if ref_form != form:
            cor.set_form(ref_form)
            out[f'vs_{ref_form}_whole_step'] = versus(a, cor.correlate(f, gross=g))
    cor.set_form(form)
    pick = [100, 110, 120, 130, s]
    fr = frames[pick].cpu().numpy()
    gr = gross[pick]
    ref0 = frames[0].cpu().numpy()
    dsub, asub = down[::2], across[::3]
    o = oracle.correlate(H, W_, dsub, asub, ref0, fr, gr, window=WIN, search=SEARCH, mode='f64')
    r = cor.correlate(fr, gross=gr)
    ro = r['offsets'][:, ::2, ::3]
    valid = np.isfinite(o['offsets64'][..., 0])
    d = np.abs(o['offsets64'] - ro).max(-1)
    snr = np.abs(r['snr'][:, ::2, ::3] / np.where(valid, o['snr'], 1) - 1)
    ok = valid & (d <= 0.5)
    # the fault line of the synthetic video: 30 degrees through the frame centre
    an = math.radians(30.0)
    yc = np.asarray(dsub)[:, None] + WIN / 2.0 - H / 2.0
    xc = np.asarray(asub)[None, :] + WIN / 2.0 - W_ / 2.0
    straddle = np.abs(-xc * math.sin(an) + yc * math.cos(an)) <= (WIN + 2 * SEARCH) / 2.0
    st = ok & straddle[None]
    out['vs_fp64_oracle'] = dict(stats(d[ok], snr[ok]), integer_peak_mismatches=int((valid & (d > 0.5)).sum()),
                                 frames=pick, windows='rows ::2, columns ::3 of the grid')
    out['vs_fp64_oracle_fault_straddling'] = stats(d[st], snr[st]) if st.any() else None
    return out


def run_b200(args):
    import torch
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))

    from slipcam_b200 import framecor, synth
    down, across = framecor.window_grid(H, W_, WIN, SEARCH, SKIP)
    nwin = len(down) * len(across)
    frames, motion, step, gross = synth.hd(n=NFRAMES, device='cuda', count=args.video)
    gross_d = torch.as_tensor(gross).cuda()
    cor = framecor.Correlator(H, W_, down, across, window=WIN, search=SEARCH, backend='b200', device=local)
    cor.set_form(args.form)
    cor.set_reference(frames[0])
    fft_n = cor.info()[2]
    BATCH = args.batch
    starts = shard_starts(rank, world, len(frames), BATCH, args.warmup + args.steps + 8)

    def step_dev(i):
        s = starts[i]
        return cor.correlate(frames[s:s + BATCH], gross=gross_d[s:s + BATCH])

    def device_rate(form):   # windows/s of a form on the timed steps (device time, this rank)
        cor.set_form(form)
        for i in range(2):
            step_dev(i)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(args.steps):
            step_dev(args.warmup + i)
        e1.record()
        torch.cuda.synchronize()
        return world * args.steps * BATCH * nwin / (e0.elapsed_time(e1) / 1e3)

    for i in range(args.warmup):
        step_dev(i)
    torch.cuda.synchronize()
    cor.profile(True)
    cor.profile_read()
    launches0 = cor.info()[3]
    clocks = Clocks(local)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step_dev(args.warmup + i)
    e1.record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    kernel_ms, kernel_launches, pairs = cor.profile_read()
    cor.profile(False)
    launches = cor.info()[3] - launches0
    ms = max_over_ranks(ms, dist, 'cuda')
    value = world * args.steps * BATCH * nwin / (ms / 1e3)

    # the other forms on the same steps (device time), for comparison
    others = {}
    for form in ('fft32', 'tc', 'int8'):
        if form != args.form and not args.no_others:
            others[form] = device_rate(form)
    cor.set_form(args.form)

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({'value': value, 'form': args.form, 'kernel_ms': kernel_ms, 'kernel_launches': kernel_launches,
                              'other_forms': others, 'clocks': clk}))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    # end to end through the host entry point, the way the reference's caller passes frames: a plain
    # (pageable) numpy array; then the same from page-locked memory
    host = torch.empty(frames.shape, dtype=torch.uint8, pin_memory=True)
    host.copy_(frames)
    pinned_np = host.numpy()
    pageable_np = np.array(pinned_np)   # an ordinary copy in pageable memory

    def e2e_rate(src):
        for i in range(2):
            s = starts[i]
            cor.correlate(src[s:s + BATCH], gross=gross[s:s + BATCH])
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for i in range(args.steps):
            s = starts[args.warmup + i]
            cor.correlate(src[s:s + BATCH], gross=gross[s:s + BATCH])
        dt = max_over_ranks(time.perf_counter() - t, dist, 'cuda')
        return world * args.steps * BATCH * nwin / dt

    e2e = e2e_rate(pageable_np)
    e2e_pinned = e2e_rate(pinned_np)

    acc = None
    cpu = None
    if rank == 0:
        acc = accuracy(cor, frames, gross, gross_d, down, across, starts[args.warmup], args.form, BATCH)
        if world == 1 and not args.no_cpu:
            cpu = reference_cpu(pinned_np[:1 + args.cpu_frames], gross, down, across, args.cpu_frames)

    if rank == 0:
        pk = peaks()
        m = 2 * SEARCH + 1
        if args.form == 'tc':
            bound, unit, peak_v = 'tensor', 'TFLOP/s', pk.get('bf16_tflops', 1590.0)
            peak_src = ('measured cuBLAS bf16 burst (MEASURED_PEAKS.json)' if 'bf16_tflops' in pk
                        else 'fallback 1.59 PFLOP/s')
            work = dft_gemm_flops(fft_n, m)
            kname = f'corr_tc_kernel<{fft_n}>'
            executed = tc_flops(fft_n, m)
        elif args.form == 'int8':
            bound, unit = 'tensor', 'TOP/s'
            peak_v = 2 * pk.get('bf16_tflops', 1590.0)
            peak_src = ('twice the measured cuBLAS bf16 burst (MEASURED_PEAKS.json): the B200 int8 tensor rate is '
                        'twice its bf16 rate')
            work = direct_ops(WIN, m)
            kname = 'corr_i8_kernel'
            executed = 2 * 128 * ((m + 15) // 16 * 16) * ((WIN + 2 * SEARCH + 31) // 32 * 32) * WIN
        else:
            sm_max = (clk or {}).get('sm_max_mhz') or pk.get('sm_max_mhz', 1965.0)
            bound, unit, peak_v = 'fp32', 'TFLOP/s', 148 * 128 * 2 * sm_max * 1e6 / 1e12
            peak_src = 'nominal FP32 CUDA-core peak: 148 SMs x 128 lanes x 2 x max SM clock'
            work = fft_flops(fft_n)
            kname = f'corr_kernel<{fft_n}>'
            executed = work
        achieved = work * pairs / (kernel_ms / 1e3) / 1e12 if kernel_ms > 0 else None
        traffic = TRAFFIC_PER_LAUNCH.get((args.form, fft_n)) if BATCH == 16 else None
        out = {
            'metric': METRIC, 'value': value, 'unit': 'windows/s', 'n_gpus': world, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': ms / args.steps, 'higher_is_better': True, 'scaling': 'weak',
            'vs_baseline': value / PUBLISHED_WPS,
            'dtype': {'tc': 'f16 operands, f32 accumulation; each peak\'s 3 x 3 recomputed in u8 x u8 -> s32',
                      'int8': 'u8 operands, s32 accumulation',
                      'fft32': 'f32'}[args.form],
            'data': 'synthetic',
            'config': {'workload': '720p video (300 frames), window 64, search 48, skip 16 (2450 windows/frame), '
                                   'per-frame gross = rounded camera motion',
                       'frames_per_step': BATCH, 'windows_per_step': BATCH * nwin, 'fft_size': fft_n,
                       'form': args.form, 'parallelism': f'frames sharded over {world} GPU(s)',
                       'l2': 'per step: 254 MB of resident reference spectra + 14.7 MB of frames read '
                             '(> 126 MB L2); the batches walk through a 276 MB video'},
            'e2e': {'value': e2e, 'unit': 'windows/s', 'h2d_bytes_per_step': BATCH * H * W_ + BATCH * 2 * 4,
                    'd2h_bytes_per_step': BATCH * nwin * 7 * 4,
                    'input': 'pageable numpy frames (as track_offsets passes them), outputs in numpy arrays'},
            'e2e_pinned': {'value': e2e_pinned, 'unit': 'windows/s', 'input': 'frames in page-locked host memory'},
            'gpu_launches': launches,
            'roofline': {'bound': bound, 'achieved': achieved, 'peak': peak_v, 'unit': unit,
                         'frac': (achieved / peak_v) if achieved else None,
                         'traffic': traffic,
                         'traffic_source': f'ncu dram bytes of one 16-frame launch of {kname}'
                                           f' (profiles/corr_{args.form}_720p_w64_s48.md)' if traffic else None,
                         'kernel': kname, 'kernel_ms_per_launch': kernel_ms / max(kernel_launches, 1),
                         'peak_source': peak_src, 'work_per_window': work, 'executed_per_window': executed,
                         'work_source': {'tc': 'useful DFT-GEMM FLOPs, one pass (forward 4n^2 nh + 8n^2 nh, '
                                                'inverse 8 m n nh + 4 m^2 nh)',
                                         'int8': 'useful integer ops of the direct correlation, 2 W^2 M^2',
                                         'fft32': 'useful FFT FLOPs 2 x 2.5 n^2 log2 n^2 + 6 n nh'}[args.form],
                         'useful_fft_flop_per_window': fft_flops(fft_n)},
            'other_forms': {k: {'value': v, 'unit': 'windows/s'} for k, v in others.items()},
            'accuracy': acc,
            'clocks': clk,
        }
        if cpu is not None:
            out['cpu_baseline'] = {'value': cpu[0], 'unit': 'windows/s', 'cores': cpu[2], 'kind': cpu[3],
                                   'sample': f'{args.cpu_frames} frames of the same workload ({cpu[1]:.1f} s)'}
        if world == 1 and not args.no_cpu:
            out['reference_cuda'] = reference_cuda()
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_mixed(args):
    """
    The mixed-grid workload: 720p frames with flat (100 DN), saturated and striped regions, three
    grids (window/search 32/16, 64/48, 128/64, skip 16: 3116 + 2450 + 1856 = 7422 windows per
    frame, FFT sizes 64, 160, 256), per-window gross U[-20, 20]. One step = 16 frames through all
    three grids: the group's persistent launch (tuned, CUDA graph) against the three grids as
    separate Correlators on the same frames. Device time, CUDA events; one GPU.
    """
    import torch
    from slipcam_b200 import framecor, synth
    H, W_, n = 720, 1280, 16
    specs = [(32, 16), (64, 48), (128, 64)]
    nvideo = n * 4
    video, _ = synth.mixed(n=nvideo + 1, h=H, w=W_)
    frames = torch.as_tensor(video[1:]).cuda()
    rng = np.random.default_rng(9)
    grids, gross = [], []
    for w, r in specs:
        down, across = framecor.window_grid(H, W_, w, r, 16)
        grids.append(dict(down=down, across=across, window=w, search=r))
        gross.append(torch.as_tensor(rng.integers(-20, 21, (nvideo, len(down), len(across), 2)).astype(np.int32)).cuda())
    nwin = sum(len(g['down']) * len(g['across']) for g in grids)
    mc = framecor.MultiCorrelator(H, W_, grids)
    mc.set_reference(video[0])
    buf = torch.empty((n, H, W_), dtype=torch.uint8, device='cuda')
    gbuf = [torch.empty((n,) + tuple(g.shape[1:]), dtype=torch.int32, device='cuda') for g in gross]

    def load(i):
        s = (i * n) % nvideo
        buf.copy_(frames[s:s + n])
        for gb, g in zip(gbuf, gross):
            gb.copy_(g[s:s + n])

    load(0)
    tuned_ms, cfg = mc.tune(buf, gross=gbuf)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(step):
        for i in range(args.warmup):
            load(i)
            step()
        torch.cuda.synchronize()
        total = 0.0
        for i in range(args.steps):
            load(args.warmup + i)
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            total += e0.elapsed_time(e1)
        return total

    ms = timed(lambda: mc.correlate(buf, gross=gbuf))
    singles = mc.grids
    ms_sep = timed(lambda: [c.correlate(buf, gross=gb) for c, gb in zip(singles, gbuf)])
    persistent = {}
    for th, ch in ((256, 1), (512, 2)):   # the single persistent launch, whatever the tuner chose
        mc.set_config(threads=th, chunk=ch, costly_first=True, per_grid=False, graph=True)
        t_ms = timed(lambda: mc.correlate(buf, gross=gbuf))
        persistent[f'threads{th}_chunk{ch}'] = {'value': args.steps * n * nwin / (t_ms / 1e3), 'ms_per_step': t_ms / args.steps}
    mc.set_config(**{k: v for k, v in cfg.items() if k != 'graph'}, graph=cfg['graph'])
    value = args.steps * n * nwin / (ms / 1e3)
    print(json.dumps({
        'metric': 'windows/s, three grids of one video in one group step (mixed workload)',
        'value': value, 'unit': 'windows/s', 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms / args.steps, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None,
        'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': '720p, 16 frames per step, grids 32/16 + 64/48 + 128/64 (skip 16, 7422 windows/frame), '
                               'flat/saturated/striped regions, per-window gross U[-20, 20]',
                   'group': cfg, 'tuned_kernel_ms': tuned_ms, 'frames_in_l2': 'frames 14.7 MB, tables reused per step'},
        'separate_launches': {'value': args.steps * n * nwin / (ms_sep / 1e3), 'unit': 'windows/s',
                              'ms_per_step': ms_sep / args.steps},
        'persistent_launch': persistent,
    }))


def run_stream(args):
    """
    The streaming workload: 1080p video (a 5 Hz 4 px shake plus a random walk, a 60 px fault step,
    noise 3 DN), window 64, search 64, skip 8: 23,976 windows per frame, FFT size 192 (the FP32
    form). value: device-resident batches of 32 frames (CUDA events); e2e: the streaming driver
    (slipcam_b200.track) from a host array of the whole video in chunks of 32 frames, disk-like reads
    into page-locked buffers overlapped with the correlation. One GPU.
    """
    import torch
    from slipcam_b200 import framecor, synth, track
    H, W_, n, batch = 1080, 1920, args.video if args.video != NFRAMES else 256, 32
    frames, _, _, _ = synth.stream(n=n + 1, device='cuda')
    host = frames.cpu().numpy()
    down, across = framecor.window_grid(H, W_, 64, 64, 8)
    nwin = len(down) * len(across)
    cor = framecor.Correlator(H, W_, down, across, window=64, search=64, backend='b200')
    cor.set_reference(frames[0])
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i in range(args.warmup):
        cor.correlate(frames[1 + (i * batch) % n:1 + (i * batch) % n + batch])
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, n // batch))
    e0.record()
    for i in range(steps):
        cor.correlate(frames[1 + i * batch:1 + (i + 1) * batch])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = steps * batch * nwin / (ms / 1e3)

    # the tensor-core form at this FFT size: the exact integer form (tcgen05 kind::i8, two 128-lane
    # tiles for the 129 shifts a side) on the same batches; the FP16 DFT-GEMM form does not hold a
    # 192-point transform beside its operands in shared memory
    cor.set_form('int8')
    for i in range(2):
        cor.correlate(frames[1 + i * batch:1 + (i + 1) * batch])
    torch.cuda.synchronize()
    e0.record()
    for i in range(steps):
        cor.correlate(frames[1 + i * batch:1 + (i + 1) * batch])
    e1.record()
    torch.cuda.synchronize()
    value_i8 = steps * batch * nwin / (e0.elapsed_time(e1) / 1e3)
    # both forms against the FP64 oracle on a sample: 2 frames, every 12th row and 16th column of windows
    from oracle import oracle
    pick = [1, n // 2]
    dsub, asub = down[::12], across[::16]
    o = oracle.correlate(H, W_, dsub, asub, host[0], host[pick], None, window=64, search=64, mode='f64')
    valid = np.isfinite(o['offsets64'][..., 0])
    acc = {}
    for form in ('int8', 'fft32'):
        cor.set_form(form)
        rr = cor.correlate(frames[pick])
        ro = rr['offsets'].cpu().numpy()[:, ::12, ::16]
        d = np.abs(o['offsets64'] - ro).max(-1)
        ok = valid & (d <= 0.5)
        snr = np.abs(rr['snr'].cpu().numpy()[:, ::12, ::16][ok] / o['snr'][ok] - 1)
        acc[form] = {'pairs': int(valid.sum()), 'max_px': float(d[ok].max()), 'median_px': float(np.median(d[ok])),
                     'frac_above_0.01px': float((d[ok] > 0.01).mean()), 'integer_peak_mismatches': int((valid & (d > 0.5)).sum()),
                     'snr_rel_max': float(snr.max())}
    cor.set_form('fft32')
    t = time.perf_counter()   # the whole job as a user runs it: Correlator, reference spectra, stream
    r = track.track(host, 0, np.arange(1, n + 1), window=64, skip=8, search=64, chunk=batch)
    job_s = time.perf_counter() - t
    t = time.perf_counter()   # the stream alone, on a prepared Correlator
    r = track.track(host, 0, np.arange(1, n + 1), window=64, skip=8, search=64, chunk=batch, correlator=cor)
    e2e_s = time.perf_counter() - t
    e2e = n * nwin / e2e_s
    print(json.dumps({
        'metric': 'windows/s, streaming 1080p video (window 64, search 64, skip 8)',
        'value': value, 'unit': 'windows/s', 'n_gpus': 1, 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': ms / steps, 'ms_per_frame': ms / steps / batch, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32', 'data': 'synthetic',
        'config': {'workload': f'1080p stream, {n} frames, window 64, search 64, skip 8 ({nwin} windows/frame), '
                               f'batches of {batch} frames', 'fft_size': cor.info()[2], 'form': 'fft32'},
        'e2e': {'value': e2e, 'unit': 'windows/s', 'ms_per_frame': e2e_s * 1e3 / n,
                'h2d_bytes_per_step': batch * H * W_, 'd2h_bytes_per_step': batch * nwin * 28,
                'path': 'slipcam_b200.track over a host array, chunks of 32 frames, prepared Correlator'},
        'whole_job': {'value': n * nwin / job_s, 'unit': 'windows/s', 's': job_s,
                      'includes': 'Correlator creation, reference spectra (3.6 GB), the stream'},
        'valid_fraction': float(np.isfinite(r['offsets'][..., 0]).mean()),
        'other_forms': {'int8': {'value': value_i8, 'unit': 'windows/s',
                                 'note': 'exact tensor-core form (u8 x u8 -> s32 on tcgen05), the same device batches'}},
        'accuracy_vs_fp64_oracle': dict(acc, sample=f'frames {pick}, windows rows ::12, columns ::16'),
        'reference_cuda': reference_cuda('stream'),
    }))


def run_diff(args):
    """
    The differentiable path: 256 x 256 float frames moved by continuous shifts U[-3, 3] (41 moved
    frames x 25 windows = 1025 windows), window 64, search 8, skip 32. value: the continuous
    refinement (slipcam_b200.diff.DiffCorrelator.refine, 8 Newton steps, each a forward pass and an
    adjoint) in windows/s; also one forward + backward of the surfaces (autograd, frames and shift)
    and the refinement's error against the true shifts. One GPU, CUDA events.
    """
    import torch
    from slipcam_b200 import diff, framecor, synth
    frames, shifts = synth.shifts_f32(n=42)
    down, across = framecor.window_grid(256, 256, 64, 8, 32)
    dc = diff.DiffCorrelator(256, 256, down, across, window=64, search=8)
    dc.set_reference(torch.as_tensor(frames[0]))
    f = torch.as_tensor(frames[1:]).cuda()
    nwin = len(down) * len(across) * f.shape[0]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        r = dc.refine(f, iters=8)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        r = dc.refine(f, iters=8)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    err = np.abs(r['offsets'].cpu().numpy() - shifts[1:, None, None, :]).max(-1)
    fr = f.clone().requires_grad_(True)
    sh = torch.full((f.shape[0], len(down), len(across), 2), 0.25, device='cuda', requires_grad=True)
    for _ in range(args.warmup):
        (dc.surface(fr, sh) ** 2).sum().backward()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        (dc.surface(fr, sh) ** 2).sum().backward()
    e1.record()
    torch.cuda.synchronize()
    fb_ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({
        'metric': 'windows/s, continuous sub-pixel refinement (8 Newton steps: forward + adjoint)',
        'value': nwin / (ms / 1e3), 'unit': 'windows/s', 'n_gpus': 1, 'steps': args.steps, 'warmup': args.warmup,
        'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
        'data': 'synthetic',
        'config': {'workload': '41 float 256 x 256 frames moved by U[-3, 3] px, window 64, search 8, skip 32 '
                               f'({nwin} windows)', 'iterations': 8},
        'refine_error_px': {'max': float(err.max()), 'median': float(np.median(err))},
        'surface_forward_backward': {'ms': fb_ms, 'windows': nwin, 'grads': 'frames and shift'},
    }))


def run_stabilize(args):
    """
    Coarse similarity tracking (stabilize.coarse_track, the reference's defaults: 96-px templates 96
    px apart, +-32 px search, min_peak 0.5): a 720p camera video (a random walk of 2 px, 1e-3 rad and
    1e-3 scale per frame, two burned-in text boxes) tracked from frame 0. A step tracks the whole
    video; the frames are sequential (each is searched around the previous one's prediction), so a
    frame is a latency-bound chain of three launches. value: device-resident frames on prepared
    templates (CUDA events); e2e: coarse_track from a host array, templates included; cpu_baseline:
    the oracle's restatement of the reference (numpy FFT, one thread) on a few frames. One GPU.
    """
    import torch
    from oracle import oracle
    from slipcam_b200 import stabilize, synth
    n = args.video if args.video != NFRAMES else 200
    text_boxes = ((900, 24, 1240, 68), (40, 650, 630, 700))
    frames, truth, text = synth.camera(n, 720, 1280, ref=0, seed=11, walk=(2.0, 2.0, 0.001, 0.001), text=text_boxes,
                                       device='cuda')
    host = frames.cpu().numpy()
    tr = stabilize.CoarseTracker(frames[0], text)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        p, u, c = tr.run(frames, 0)
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 10))
    launches0 = tr._cor.info()[3]
    e0.record()
    for _ in range(steps):
        p, u, c = tr.run(frames, 0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    launches = (tr._cor.info()[3] - launches0) // steps
    def e2e_time(call):   # after a warm-up call, the median of three timed calls
        call()
        times = []
        for _ in range(3):
            t = time.perf_counter()
            r = call()
            times.append(time.perf_counter() - t)
        return statistics.median(times), r

    e2e_s, (pe, ue, _) = e2e_time(lambda: stabilize.coarse_track(host, 0, text))
    cpu_frames = 4
    t = time.perf_counter()
    po, uo, _ = oracle.coarse_track(host[:cpu_frames + 1], 0, text)
    cpu_s = time.perf_counter() - t
    err = np.abs(p - truth)
    # the resampling half (stabilize.stabilize): the frames warped onto the reference with the
    # tracked transforms, the text blanked
    st = stabilize.Stabilizer(text)
    for _ in range(args.warmup):
        st.run(frames, p)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        warped, union = st.run(frames, p)
    e1.record()
    torch.cuda.synchronize()
    ms_w = e0.elapsed_time(e1) / steps
    e2e_w, _ = e2e_time(lambda: stabilize.stabilize(host, p, text))
    t = time.perf_counter()
    ow, _ = oracle.stabilize(host[:2], p[:2], text)
    cpu_w = time.perf_counter() - t
    print(json.dumps({
        'metric': 'frames/s, coarse similarity tracking of a 720p video (stabilize.coarse_track defaults)',
        'value': (n - 1) / (ms / 1e3), 'unit': 'frames/s', 'n_gpus': 1, 'steps': steps, 'warmup': args.warmup,
        'ms_per_step': ms, 'us_per_frame': ms * 1e3 / (n - 1), 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f32 correlation, f64 fit', 'data': 'synthetic',
        'config': {'workload': f'720p camera video, {n} frames, window 96, step 96, search 32 ({tr.nwin} templates, '
                               f'{c} in use)', 'form': 'fft32'},
        'e2e': {'value': (n - 1) / e2e_s, 'unit': 'frames/s', 'h2d_bytes_per_step': (n - 1) * 720 * 1280,
                'd2h_bytes_per_step': (n - 1) * 36,
                'path': 'stabilize.coarse_track over a host array (templates built per call), median of 3 calls'},
        'gpu_launches': launches,
        'cpu_baseline': {'value': cpu_frames / cpu_s, 'unit': 'frames/s', 'cores': 1, 'kind': 'port',
                         'sample': f'{cpu_frames} frames of the same video ({cpu_s:.1f} s)'},
        'agreement': {'vs_oracle_max_px': float(np.abs(po[1:] - p[1:cpu_frames + 1])[:, :2].max()),
                      'used_equal': bool(np.array_equal(uo[1:], u[1:cpu_frames + 1])),
                      'host_equals_device': bool(np.array_equal(pe, p))},
        'error_vs_truth': {'shift_px': float(err[:, :2].max()), 'rotation_scale': float(err[:, 2:].max())},
        'resample': {'what': 'stabilize.stabilize: text blanked (31 px box means), frames warped (bilinear), text union',
                     'value': n / (ms_w / 1e3), 'unit': 'frames/s', 'ms_per_step': ms_w,
                     'e2e': {'value': n / e2e_w, 'unit': 'frames/s',
                             'path': 'stabilize.stabilize over a host array, median of 3 calls'},
                     'cpu_baseline': {'value': 2 / cpu_w, 'unit': 'frames/s', 'cores': 1, 'kind': 'port',
                                      'sample': f'2 frames ({cpu_w:.2f} s)'},
                     'equals_oracle': bool(np.array_equal(warped[:2].cpu().numpy(), ow))},
    }))


def run_scans(args):
    """
    auto_slip's scans around the path on the b200 backend (one GPU): frame_differences over a 720p
    video (300 frames), the burned-in text mask from 150 of its frames (chunks of 10), and
    periodicity of the reference frame's 720p grid (window 64, search 48, skip 16: 2450 windows).
    The frame-difference kernel is timed by CUDA events through the C ABI on device-resident frames
    (its roofline: HBM, two frames read per pair); the rest through the public calls. CPU: the
    oracle's restatements of the reference functions on bounded samples, one thread.
    """
    import ctypes

    import torch
    from oracle import oracle
    from slipcam_b200 import _lib, framecor, scans, synth
    n, h, w = (args.video if args.video != NFRAMES else 300), 720, 1280
    boxes = ((900, 24, 1240, 68), (40, 650, 630, 700))
    frames, _, _ = synth.camera(n, h, w, ref=0, seed=15, walk=(1.0, 1.0, 0.0005, 0.0005), text=boxes, device='cuda')
    host = frames.cpu().numpy()
    lib, stream = _lib.lib(), torch.cuda.current_stream().cuda_stream
    out = torch.empty(n - 1, dtype=torch.float32, device='cuda')
    sums = torch.empty(n - 1, dtype=torch.int64, device='cuda')
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def diff_launch():
        rc = lib.b200_frame_diff_device(frames.data_ptr(), n, h, w, w, out.data_ptr(), sums.data_ptr(), stream)
        assert rc == _lib.OK
    for _ in range(args.warmup):
        diff_launch()
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 20))
    e0.record()
    for _ in range(steps):
        diff_launch()
    e1.record()
    torch.cuda.synchronize()
    diff_ms = e0.elapsed_time(e1) / steps
    diff_bytes = float(n) * h * w   # the algorithmic minimum: every frame read once
    pk = peaks()
    hbm = pk.get('hbm_gbs', 6650.0)
    d_gpu = scans.frame_differences(host)   # from host memory, the public call
    t = time.perf_counter()
    scans.frame_differences(host)
    diff_e2e_s = time.perf_counter() - t
    cpu_n = 60
    t = time.perf_counter()
    d_cpu = oracle.frame_differences(host[:cpu_n])
    diff_cpu_s = time.perf_counter() - t

    def timed(call, reps=3):
        call()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t = time.perf_counter()
            r = call()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t)
        return statistics.median(ts), r
    tm_s, mask = timed(lambda: scans.text_mask(frames, 0, nframes=150, chunk=10))
    tm_e2e_s, mask_h = timed(lambda: scans.text_mask(host, 0, nframes=150, chunk=10))
    t = time.perf_counter()
    mask_cpu = oracle.text_mask(host, 0, nframes=150, chunk=10)
    tm_cpu_s = time.perf_counter() - t
    down, across = framecor.window_grid(h, w, 64, 48, 16)
    per_s, per = timed(lambda: framecor.periodicity(frames[0], down, across, 64, 48))
    sub_d, sub_a = down[::9][:3], across[::14][:5]
    t = time.perf_counter()
    per_cpu = oracle.periodicity(host[0], sub_d, sub_a, 64, 48)
    per_cpu_s = time.perf_counter() - t
    print(json.dumps({
        'metric': 'frames/s, auto_slip frame differences of a 720p video', 'value': (n - 1) / (diff_ms / 1e3),
        'unit': 'frames/s', 'n_gpus': 1, 'steps': steps, 'warmup': args.warmup, 'ms_per_step': diff_ms,
        'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'u8 -> int64 sums',
        'data': 'synthetic',
        'config': {'workload': f'720p camera video, {n} frames, two burned-in text boxes; text mask from 150 frames '
                               '(chunks of 10); periodicity of the reference frame, window 64, search 48, skip 16 '
                               f'({len(down) * len(across)} windows)', 'l2': f'{n} frames = {n * h * w / 1e6:.0f} MB > L2'},
        'roofline': {'bound': 'hbm', 'achieved': diff_bytes / (diff_ms / 1e3) / 1e9, 'peak': hbm, 'unit': 'GB/s',
                     'frac': diff_bytes / (diff_ms / 1e3) / 1e9 / hbm, 'kernel': 'frame_diff_kernel',
                     'algorithmic_bytes': 'every frame read once (n x 720 x 1280 bytes)', 'traffic': None,
                     'peak_source': 'MEASURED_PEAKS.json hbm_gbs' if 'hbm_gbs' in pk else 'fallback 6.65 TB/s'},
        'e2e': {'value': (n - 1) / diff_e2e_s, 'unit': 'frames/s', 'h2d_bytes_per_step': n * h * w,
                'd2h_bytes_per_step': (n - 1) * 4, 'path': 'scans.frame_differences over a host array'},
        'gpu_launches': 1,
        'cpu_baseline': {'value': (cpu_n - 1) / diff_cpu_s, 'unit': 'frames/s', 'cores': 1, 'kind': 'port',
                         'sample': f'{cpu_n} frames ({diff_cpu_s:.2f} s)'},
        'agreement': {'frame_differences_equal': bool(np.array_equal(d_gpu[:cpu_n - 1], d_cpu)),
                      'text_mask_equal': bool(np.array_equal(mask, mask_cpu) and np.array_equal(mask_h, mask_cpu)),
                      'periodicity_max_abs': float(np.abs(per[::9][:3, ::14][:, :5] - per_cpu).max())},
        'text_mask': {'ms': tm_s * 1e3, 'ms_from_host': tm_e2e_s * 1e3, 'cpu_ms': tm_cpu_s * 1e3,
                      'cpu_kind': 'port, 1 thread', 'pixels': int(mask.sum())},
        'periodicity': {'windows_per_s': len(down) * len(across) / per_s, 'ms': per_s * 1e3,
                        'cpu_windows_per_s': per_cpu.size / per_cpu_s,
                        'cpu_sample': f'{per_cpu.size} windows, FP64 direct restatement ({per_cpu_s:.1f} s)'},
    }))


def launch_ranks(n):
    """--gpus N without a launcher: start N ranks of this same command through torch.distributed.run
    (one process per GPU, rendezvous on 127.0.0.1) and return its exit code. N above the visible
    device count is refused with a message."""
    import socket

    try:
        import torch
        if torch.cuda.is_available() and n > torch.cuda.device_count():
            print(f'bench.py: --gpus {n} but {torch.cuda.device_count()} CUDA device(s) are visible', file=sys.stderr)
            return 2
    except ImportError:
        pass
    with socket.socket() as sk:   # a free port for the rendezvous
        sk.bind(('127.0.0.1', 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, '-m', 'torch.distributed.run', '--nnodes=1', f'--nproc-per-node={n}', '--master-addr',
           '127.0.0.1', '--master-port', str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def run_launch_check(args):
    """The multi-rank plumbing alone (no GPU needed): every rank joins the process group (gloo without
    CUDA), takes its batches with shard_starts, times a small host computation, and rank 0 prints the
    line with the max over ranks, as the correlation workload does."""
    import datetime

    import torch
    import torch.distributed as dist
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    if world > 1:
        dist.init_process_group('nccl' if torch.cuda.is_available() else 'gloo', timeout=datetime.timedelta(seconds=60))
    starts = shard_starts(rank, world, NFRAMES, BATCH, args.steps)
    t = time.perf_counter()
    a = np.random.default_rng(rank).random((256, 256))
    for _ in range(args.steps):
        a = a @ a.T / 256.0
    dt = time.perf_counter() - t
    dev = 'cuda' if torch.cuda.is_available() else 'cpu'
    slowest = max_over_ranks(dt, dist if world > 1 else None, dev)
    seen = [None] * world
    if world > 1:
        dist.all_gather_object(seen, {'rank': rank, 'first_batch': starts[0]})
    else:
        seen = [{'rank': 0, 'first_batch': starts[0]}]
    if rank == 0:
        print(json.dumps({'metric': 'launch check', 'n_gpus': world, 'ranks': seen, 'value': world * args.steps / slowest,
                          'unit': 'steps/s', 'steps': args.steps}))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=30)
    p.add_argument('--warmup', type=int, default=5)
    p.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    p.add_argument('--cpu-frames', type=int, default=2)
    p.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline')
    p.add_argument('--no-e2e', action='store_true', help='device timing only (profiling runs)')
    p.add_argument('--no-others', action='store_true', help='skip the other forms on the same steps (profiling runs)')
    p.add_argument('--video', type=int, default=NFRAMES, help='frames of the synthetic video to render')
    p.add_argument('--batch', type=int, default=BATCH, help='frames per step')
    p.add_argument('--form', default='tc', choices=['fft32', 'tc', 'int8'], help='the arithmetic of the transforms')
    p.add_argument('--workload', default='hd', choices=['hd', 'mixed', 'stream', 'diff', 'stabilize', 'scans',
                                                       'launch-check'],
                   help='hd: the 720p headline; mixed: three grids in one group step; stream: 1080p streaming; '
                        'diff: the differentiable path; stabilize: coarse similarity tracking; '
                        'scans: frame differences, text mask, periodicity')
    args = p.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and 'WORLD_SIZE' not in os.environ:
        sys.exit(launch_ranks(args.gpus))
    if args.workload == 'launch-check':
        return run_launch_check(args)
    if args.workload == 'mixed' and args.impl != 'reference':
        run_mixed(args)
    elif args.workload == 'stream' and args.impl != 'reference':
        run_stream(args)
    elif args.workload == 'diff' and args.impl != 'reference':
        run_diff(args)
    elif args.workload == 'stabilize' and args.impl != 'reference':
        run_stabilize(args)
    elif args.workload == 'scans' and args.impl != 'reference':
        run_scans(args)
    elif args.impl == 'reference':
        run_reference(args)
    else:
        run_b200(args)


if __name__ == '__main__':
    main()
