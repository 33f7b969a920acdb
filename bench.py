# -*- coding: utf-8 -*-
"""Benchmark of the synchrosqueezing hot path on one B200 per rank.

Headline (the JSON line's `value`): ssq_cwt forward, float32, one N=160,000
signal per GPU per step (linear chirp 0.01->0.2 cycles/sample + AM tone at
0.3 + N(0, 0.1^2) noise), GMW gamma=3 beta=60, nv=32, log-piecewise scales
(293 rows), reflect padding (Npad = 262,144), inputs resident in HBM and
outputs preallocated (the C-ABI calls of one ssq_cwt: fused CWT + squeeze).
`e2e` is the same metric through the public `ssq_cwt` call from pinned host
memory, with the host->device copy of x and the device->host copy of Tx.

Further legs, each a key of the same line:
  batched  256 signals of uneven length in [4096, 65536], Morlet mu=6, one
           SsqCwtBatch plan (CUDA graph) vs one ssq_cwt call per signal;
  long     8 x N=1,048,576, GMW, 'log:maximal' (613 rows): plain forward,
           batched forward, forward + backward, peak memory;
  fwd_bwd  64 x N=16,384 Morlet: loss MSE(|Tx(x)|,|Tx(y)|) + MSE(icwt(Wx), y),
           forward vs forward + backward through the adjoint kernels;
  stft     ssq_stft of the headline signal, Hann 512, n_fft 512, hop 1.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Each rank processes its own signals (weak scaling, no collective on the
data path). `--impl reference` times the CPU restatement of ssqueezepy's
algorithm (oracle/ssq_oracle.py, float64, all host threads) on the headline
workload.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("ssq_cwt signal-samples/s fwd & fwd+bwd, batched vs plain, "
          "% of HBM roofline")
UNIT = "signal-samples/s"
N_SIG = 160000
WAVELET = ('gmw', {'gamma': 3., 'beta': 60., 'dtype': 'float32'})
L2_BYTES = 126 * 2**20
# DRAM bytes the fused CWT call moves per (row, sample), from the ncu capture
# summarised in profiles/traffic_ssq_cwt_N40000_gmw.md
CWT_TRAFFIC_PER_ROW_SAMPLE = 15.73


def chirp_signal(N, seed=0):
    t = np.arange(N, dtype=np.float64)
    rng = np.random.default_rng(seed)
    return (np.cos(2 * np.pi * (0.01 * t + 0.19 * t**2 / (2 * N)))
            + (0.5 + 0.5 * np.cos(2 * np.pi * 0.001 * t))
            * np.cos(2 * np.pi * 0.3 * t)
            + 0.1 * rng.standard_normal(N))


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def fp64_peak_tflops(torch, dev):
    """Measured float64 throughput of this GPU: cuBLAS DGEMM 4096^3 (2 N^3
    flops), best of 5 after a warm-up, CUDA events. The denominator of the
    CWT kernel's compute roofline (its float64 FFTs), measured here because
    the peak file holds HBM and bf16 figures only."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = float('inf')
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
         'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
         'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu_index):
        self.rows, self.proc = [], None
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', '--query-gpu=' + self.Q, '--format=csv,noheader,nounits',
                 '-lms', '200', '-i', str(gpu_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) stalls kernel launches
        # for milliseconds: let it finish before any timed step
        t0 = time.time()
        while not self.rows and time.time() - t0 < 10 and self.proc.poll() is None:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(',')])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown',
                 'sw_power_cap']
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == 'active':
                        reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def max_over_ranks(values, device):
    """Element-wise max of per-rank timings over all ranks (every rank takes
    the same collective; one rank returns its own values)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def oracle_step(x, scales, f_asc, const):
    from oracle import ssq_oracle as O
    return O.ssq_cwt(x, 'gmw_l1', (3., 60.), scales, f_asc, const)


def host_params(N=N_SIG):
    from ssqueezepy_b200 import _params as P
    w = P.Wavelet(WAVELET)
    sc, st, na, nv = P.process_scales('log-piecewise', N, w, nv=32,
                                      get_params=True)
    f = P.compute_associated_frequencies(sc, N, w, st, 'peak', True, 1., 'cwt')
    _, st_a, _, nv_a = P.process_scales(sc, N, get_params=True)  # per-row nv
    const = P.squeeze_weights(sc, st_a, nv_a, 'cwt')
    return w, sc.ravel(), f, const, na


def cpu_path(N=N_SIG):
    """The reference's CPU execution of the headline ssq_cwt (float32,
    SSQ_PARALLEL=1, cached wavelet), restated in oracle/ssq_cpu_path.py."""
    from oracle.ssq_cpu_path import SsqCwtCpu
    from ssqueezepy_b200 import _params as P
    w, sc, f, const, na = host_params(N)
    mode, bp = P.bin_params(f, True)
    return SsqCwtCpu(N, 'gmw_l1', (3., 60.), sc, mode, bp, const), na


CPU_SAMPLE = ("one full N=%d ssq_cwt per step, float32, as the reference's CPU path "
              "runs it (SSQ_PARALLEL=1, cache_wavelet=True): scipy.fft over %d threads, "
              "cached float32 wavelet bank, OpenMP column-parallel squeeze "
              "(oracle/ssq_cpu_path.py)")


def run_reference(args):
    rank = int(os.environ.get('RANK', 0))
    if rank != 0:
        return 0
    port, na = cpu_path()
    x = chirp_signal(N_SIG, seed=0).astype(np.float32)
    for _ in range(max(args.warmup, 3)):
        port(x)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        port(x)
        ts.append(time.perf_counter() - t0)
    dt = float(np.median(ts))
    v = N_SIG / dt
    cores = os.cpu_count()
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "ssq_cwt N=160000 GMW(3,60) nv=32 log-piecewise "
                                   "(293 rows) float32 reflect, one signal per GPU",
                       "N": N_SIG, "na": na, "parallelism": "rank0 CPU",
                       "timing": "median of the timed steps"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": CPU_SAMPLE % (N_SIG, cores)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _lib as L
    from ssqueezepy_b200 import _params as P

    world = int(os.environ.get('WORLD_SIZE', 1))
    rank = int(os.environ.get('RANK', 0))
    local = int(os.environ.get('LOCAL_RANK', 0))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    lib = L.load()
    N = args.n
    w, sc, f, const, na = host_params(N)
    Npad, n1, _ = P.p2up(N)
    x_np = chirp_signal(N, seed=rank).astype(np.float32)
    x = torch.as_tensor(x_np, device=dev)
    Wx = torch.empty((1, na, N), dtype=torch.complex64, device=dev)
    Tx = torch.empty_like(Wx)
    ipitch = L.idx_pitch(N)
    idx = torch.empty((1, na, ipitch), dtype=torch.uint16, device=dev)
    wsb = lib.ssqb_cwt_workspace_bytes(1, N, Npad, na, L.F32)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    sc_d = torch.as_tensor(sc, dtype=torch.float64, device=dev)
    cst_d = torch.as_tensor(const, dtype=torch.float64, device=dev)
    cw = L.wavelet_struct(w)
    mode, bp = P.bin_params(f, True)
    cb = L.make_bins(mode, bp, na, True)
    gamma = 10 * P.EPS32
    st = torch.cuda.current_stream()
    sp = L.stream_ptr(st)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)
    # float32 data, float64 arithmetic (the default of the public API)
    prec = L.F32X if args.arith == 'float64' else L.F32
    wsb = max(wsb, lib.ssqb_cwt_workspace_bytes(1, N, Npad, na, prec))
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    sc_h = np.ascontiguousarray(sc, np.float64)  # host scales: per-row plan
    launches = lib.ssqb_cwt_ex_launches(1, Npad, na, prec, wsb, sc_h.ctypes.data, cw) + 1

    def step(ev=None, prec=prec):
        if ev:
            ev[0].record(st)
        L.check(lib.ssqb_cwt_ex(L.ptr(x), 1, N, Npad, n1, 1, 0, L.ptr(sc_d),
                                sc_h.ctypes.data, na, cw, 1.0, cb, gamma, prec, L.ptr(Wx),
                                None, None, L.ptr(idx), ipitch, L.ptr(ws), wsb, sp), 'cwt')
        if ev:
            ev[1].record(st)
        L.check(lib.ssqb_squeeze(L.ptr(Wx), L.ptr(idx), ipitch, L.ptr(cst_d), 1, na, N,
                                 na, L.F32, L.ptr(Tx), sp), 'squeeze')
        if ev:
            ev[2].record(st)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    fp64_tf = fp64_peak_tflops(torch, dev) if rank == 0 else None
    clk = Clocks(local) if rank == 0 else None  # samples through every timed leg
    for _ in range(max(args.warmup, 3)):
        step()
    assert L.device_status() == 0
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)]
           for _ in range(args.steps)]
    barrier()
    for k in range(args.steps):
        flush.zero_()  # write 252 MB > L2 between timed steps (outside events)
        step(evs[k])
    barrier()
    cwt_ms = [e[0].elapsed_time(e[1]) for e in evs]
    sq_ms = [e[1].elapsed_time(e[2]) for e in evs]
    step_ms = float(np.sum(cwt_ms) + np.sum(sq_ms)) / args.steps
    step_ms_max, = max_over_ranks([step_ms], dev)
    value = world * N / (step_ms_max * 1e-3)

    # end to end through the public API from pinned host memory
    e2e_value = None
    if args.no_e2e:
        pass
    else:
        e2e_value = run_e2e(sb, torch, dist, x_np, na, N, st, world, dev, barrier,
                            args)
    Tx_keep = Tx[0].cpu().numpy() if rank == 0 else None
    Wx_keep = Wx[0].cpu().numpy() if rank == 0 else None
    idx_keep = idx[0, :, :N].cpu().numpy() if rank == 0 else None
    batched = None
    if not args.no_batch:
        del Wx, Tx, idx, ws
        batched = run_batched(args, torch, dev, world, barrier, flush)
    stft_ = None
    if not args.no_stft:
        stft_ = run_stft(args, torch, dev, world, barrier, flush)
    long_ = None
    if not args.no_long:
        torch.cuda.empty_cache()
        long_ = run_long(args, torch, dev, world, barrier)
    train = None
    if not args.no_train:
        torch.cuda.empty_cache()
        train = run_train(args, torch, dev, world, barrier, flush)
    next_ = None
    if not args.no_next:
        torch.cuda.empty_cache()
        next_ = run_next(args, torch, dev, world, barrier, flush)
    clocks = clk.stop() if clk else None
    if rank == 0:
        emit(args, world, N, na, Npad, step_ms_max, value, cwt_ms, sq_ms, e2e_value,
             launches, clocks, sc, f, const, Tx_keep, Wx_keep, batched, train, long_,
             stft_, next_, fp64_tf, idx_keep)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_e2e(sb, torch, dist, x_np, na, N, st, world, dev, barrier, args):
    """The headline metric through the public API from host buffers: every
    step copies its signal from pinned host memory to the device, runs
    ssq_cwt and copies Tx (na x N complex64) back to pinned host memory. Steps
    alternate between two streams, as a streaming caller would, so one step's
    copy back overlaps the next step's transform; the region ends when every
    step's copy back has finished."""
    x_pin = torch.from_numpy(x_np).pin_memory()
    Tx_pin = [torch.empty((na, N), dtype=torch.complex64).pin_memory() for _ in range(2)]
    streams = [torch.cuda.Stream(dev), torch.cuda.Stream(dev)]

    def step(k):
        s = streams[k % 2]
        with torch.cuda.stream(s):
            Tp, *_ = sb.ssq_cwt(x_pin, WAVELET, scales='log-piecewise', nv=32)
            Tx_pin[k % 2].copy_(Tp, non_blocking=True)

    for k in range(2):
        step(k)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(4, min(args.steps, 10))
    e0.record(st)
    for s in streams:
        s.wait_event(e0)
    for k in range(e2e_steps):
        step(k)
    for s in streams:
        st.wait_stream(s)
    e1.record(st)
    barrier()
    e2e_ms, = max_over_ranks([e0.elapsed_time(e1) / e2e_steps], dev)
    return world * N / (e2e_ms * 1e-3)


def run_batched(args, torch, dev, world, barrier, flush):
    """256 float32 signals of lengths uniform in [4096, 65536] (seeded chirp
    mixtures), Morlet mu=6, nv=32 log-piecewise: one autotuned SsqCwtBatch
    plan (a CUDA graph per step) against one public ssq_cwt call per signal,
    both with inputs resident on the device."""
    import torch.distributed as dist
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200._batch import SsqCwtBatch
    from ssqueezepy_b200 import _signals as S
    rank = int(os.environ.get('RANK', 0))
    xs = [x.astype(np.float32) for x in
          S.uneven_batch(args.batch, 4096, 65536, seed=1234 + rank)]
    lengths = [len(x) for x in xs]
    wav = ('morlet', {'mu': 6., 'dtype': 'float32'})
    plan = SsqCwtBatch(lengths, wavelet=wav, graph=True, device=dev, autotune=True)
    plan.load(xs)
    st = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 3)):
        plan.run()
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for e in evs:
        flush.zero_()
        e[0].record(st)
        plan.run()
        e[1].record(st)
    barrier()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    # the same signals, one public ssq_cwt call each (inputs on the device)
    xd = [torch.as_tensor(x, device=dev) for x in xs]
    for x in xd:  # host parameter plans for every length, kernels warm
        sb.ssq_cwt(x, wav, scales='log-piecewise', nv=32)
    barrier()
    psteps = max(1, min(args.steps, 3))
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    flush.zero_()
    p0.record(st)
    for _ in range(psteps):
        for x in xd:
            sb.ssq_cwt(x, wav, scales='log-piecewise', nv=32)
    p1.record(st)
    barrier()
    plain_ms = p0.elapsed_time(p1) / psteps
    ms, plain_ms = max_over_ranks([ms, plain_ms], dev)
    nas = plan.sig_np['na'].astype(np.int64)
    Ns = plan.sig_np['N'].astype(np.int64)
    tot = int(Ns.sum())
    alg = int(((4 + 16 * nas) * Ns).sum())
    hbm, src = peaks()
    tx_err = None
    if rank == 0 and not args.no_cpu:
        from oracle import ssq_oracle as O
        outs = plan.outputs()
        errs = []
        for i in (int(np.argmin(Ns)), int(np.argmax(Ns))):
            To, _, _ = O.ssq_cwt(xs[i].astype(np.float64), 'morlet', (6.,),
                                 plan.scales64[i], plan.ssq_freqs[i][::-1].copy(),
                                 plan.weights64[i])
            Tg = outs[i][0].cpu().numpy()
            errs.append(float(np.linalg.norm(Tg - To) / np.linalg.norm(To)))
        tx_err = max(errs)
    return {
        "workload": "ssq_cwt batch of %d float32 signals, N uniform in [4096, 65536] "
                    "(sum N = %d), Morlet mu=6 nv=32 log-piecewise (%d-%d rows), "
                    "reflect; one SsqCwtBatch plan replayed as a CUDA graph"
                    % (len(xs), tot, nas.min(), nas.max()),
        "value": world * tot / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
        "plain_value": world * tot / (plain_ms * 1e-3), "plain_ms_per_step": plain_ms,
        "speedup_vs_plain": plain_ms / ms,
        "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": hbm,
                     "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / hbm,
                     "peak_source": src,
                     "bytes": "sum_i N_i (4 + 16 na_i): read x, write Wx and Tx"},
        "gpu_launches": plan.launches * args.steps,
        "l2": "252 MB buffer written between timed steps; outputs %.1f GB"
              % (plan.n_out * 16 / 1e9),
        "Tx_rel_l2_vs_oracle_shortest_longest": tx_err,
        "autotune": plan.tuning,
    }


def run_train(args, torch, dev, world, barrier, flush):
    """Differentiable ssq_cwt + icwt on a batch of 64 float32 signals of
    N = 16,384 (chirp mixtures), Morlet mu=6, nv=32 log-piecewise: loss =
    MSE(|Tx(x)|, |Tx(y)|) + MSE(icwt(Wx(x)), y). Times the forward (loss)
    and forward + backward (gradient of x through the adjoint kernels)."""
    import torch.distributed as dist
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _signals as S
    rank = int(os.environ.get('RANK', 0))
    B, N = args.train_batch, 16384
    wav = ('morlet', {'mu': 6., 'dtype': 'float32'})
    xs = torch.tensor(S.same_length_batch(B, N, 5678 + rank), dtype=torch.float32,
                      device=dev)
    y = torch.tensor(S.same_length_batch(B, N, 9012 + rank), dtype=torch.float32,
                     device=dev)
    with torch.no_grad():
        Ty = sb.ssq_cwt(y, wav)[0].abs()

    def fwd(x):
        Tx, Wx, _, _ = sb.ssq_cwt(x, wav)
        xr = sb.icwt(Wx, wav, x_len=N)
        return ((Tx.abs() - Ty) ** 2).mean() + ((xr - y) ** 2).mean()

    x = xs.clone().requires_grad_(True)
    st = torch.cuda.current_stream()
    for _ in range(max(args.warmup, 3)):
        fwd(x).backward()
    barrier()
    steps = max(1, min(args.steps, 5))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    flush.zero_()
    ev[0].record(st)
    for _ in range(steps):
        with torch.no_grad():
            fwd(xs)
    ev[1].record(st)
    barrier()
    flush.zero_()
    ev[2].record(st)
    for _ in range(steps):
        x.grad = None
        fwd(x).backward()
    ev[3].record(st)
    barrier()
    f_ms, fb_ms = max_over_ranks([ev[0].elapsed_time(ev[1]) / steps,
                                  ev[2].elapsed_time(ev[3]) / steps], dev)
    peak = torch.cuda.max_memory_allocated(dev)
    return {
        "workload": "ssq_cwt + icwt loss, batch %d x N=%d float32 chirp mixtures, "
                    "Morlet mu=6 nv=32 log-piecewise; backward through the adjoint "
                    "kernels (bins held fixed)" % (B, N),
        "fwd_value": world * B * N / (f_ms * 1e-3), "fwd_ms": f_ms,
        "fwd_bwd_value": world * B * N / (fb_ms * 1e-3), "fwd_bwd_ms": fb_ms,
        "fwd_bwd_over_fwd": fb_ms / f_ms, "unit": UNIT,
        "peak_memory_gb": peak / 1e9,
    }


def run_stft(args, torch, dev, world, barrier, flush):
    """ssq_stft of the headline signal (N = 160,000) through the public API with
    x resident on the device, float32 data, float64 arithmetic: Hann window of
    512, n_fft = 512, hop 1 (257 x N); and the reference's own benchmark
    length, n_fft = 598 (300 x N; README.md:40-54), which is not a power of
    two and goes through the chirp-z kernel."""
    import ssqueezepy_b200 as sb
    rank = int(os.environ.get('RANK', 0))
    N = args.n
    x = torch.as_tensor(chirp_signal(N, seed=rank).astype(np.float32), device=dev)
    st = torch.cuda.current_stream()
    hbm, src = peaks()

    def leg(n_fft):
        for _ in range(max(args.warmup, 3)):
            sb.ssq_stft(x, 'hann', n_fft=n_fft)
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        for e in evs:
            flush.zero_()
            e[0].record(st)
            sb.ssq_stft(x, 'hann', n_fft=n_fft)
            e[1].record(st)
        barrier()
        ms, = max_over_ranks([float(np.mean([a.elapsed_time(b) for a, b in evs]))], dev)
        nrow = n_fft // 2 + 1
        alg = (4 + 16 * nrow) * N
        return {"workload": "ssq_stft N=%d, Hann %d, n_fft %d, hop 1 (%d rows), float32, "
                            "reflect" % (N, n_fft, n_fft, nrow),
                "value": world * N / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9,
                             "peak": hbm, "unit": "GB/s",
                             "frac": alg / (ms * 1e-3) / 1e9 / hbm, "peak_source": src,
                             "bytes": "N (4 + 16 * %d): read x, write Sx and Tx" % nrow}}
    out = leg(512)
    out["n_fft_598"] = leg(598)
    return out


def run_next(args, torch, dev, world, barrier, flush):
    """The rows beside the path, on the headline signal (N = 160,000, GMW(3,60),
    293 rows, float32 data) through the public API with inputs resident on the
    device: ssq_cwt with higher-order GMWs averaged over orders (0, 1), the
    phase transform by unwrapped angle (difftype='phase', get_w=True), the
    full inverse issq_cwt of Tx, extract_ridges of Tx (one ridge, bw 15), and
    istft of the Hann-512 hop-1 STFT (257 x N). Each entry: mean device time
    of `steps` calls after warm-up, L2 flushed between calls."""
    import ssqueezepy_b200 as sb
    rank = int(os.environ.get('RANK', 0))
    N = args.n
    x = torch.as_tensor(chirp_signal(N, seed=rank).astype(np.float32), device=dev)
    st = torch.cuda.current_stream()
    wav = ('gmw', {'gamma': 3., 'beta': 60.})
    Tx, Wx, f, sc = sb.ssq_cwt(x, wav)
    na = int(Tx.shape[0])
    del Wx
    Sx = sb.stft(x, 'hann', n_fft=512)

    def timed(fn, steps):
        for _ in range(max(args.warmup, 3)):
            fn()
        barrier()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        for e in evs:
            flush.zero_()
            e[0].record(st)
            fn()
            e[1].record(st)
        barrier()
        return float(np.mean([a.elapsed_time(b) for a, b in evs]))

    ridge_steps = max(1, min(args.steps, 3))
    ms = [timed(lambda: sb.ssq_cwt(x, wav), args.steps),
          timed(lambda: sb.ssq_cwt(x, wav, order=(0, 1)), args.steps),
          timed(lambda: sb.ssq_cwt(x, wav, difftype='phase', get_w=True), args.steps),
          timed(lambda: sb.issq_cwt(Tx, wav), args.steps),
          timed(lambda: sb.extract_ridges(Tx, sc, penalty=2., n_ridges=1, bw=15),
                ridge_steps),
          timed(lambda: sb.istft(Sx, 'hann', n_fft=512, N=N), args.steps)]
    ms = max_over_ranks(ms, dev)
    hbm, src = peaks()

    def entry(name, t, nbytes, what):
        gbs = nbytes / (t * 1e-3) / 1e9
        return {"workload": name, "ms": t, "value": world * N / (t * 1e-3), "unit": UNIT,
                "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s",
                             "frac": gbs / hbm, "bytes": what}}
    ssq_bytes = (4 + 16 * na) * N
    return {
        "ssq_cwt_api": entry("ssq_cwt through the public API (reference point)", ms[0],
                             ssq_bytes, "N (4 + 16 na): read x, write Wx and Tx"),
        "higher_order_avg01": entry("ssq_cwt order=(0, 1): one transform with the mean "
                                    "wavelet", ms[1], ssq_bytes,
                                    "N (4 + 16 na): read x, write Wx and Tx"),
        "difftype_phase": entry("ssq_cwt difftype='phase', get_w=True", ms[2],
                                (4 + 16 * na + 16 * na + 4 * na) * N,
                                "N (4 + 8 na + 16 na + 4 na + 8 na): x; Wx written and "
                                "read; w; Tx"),
        "issq_cwt": entry("issq_cwt of Tx (full inversion)", ms[3], (8 * na + 8) * N,
                          "N (8 na + 8): read Tx, write x (float64)"),
        "extract_ridges": dict(entry("extract_ridges of Tx, 1 ridge, bw 15", ms[4],
                                     (8 * na + 8) * N, "N (8 na + 8): read Tx, write the "
                                     "ridge"), note="forward sweep is sequential in "
                                     "time: latency-bound, not HBM-bound"),
        "istft": entry("istft of stft(x, hann, n_fft=512, hop 1) (257 x N)", ms[5],
                       (8 * 257 + 4) * N, "N (8 * 257 + 4): read Sx, write x"),
        "peak_source": src,
    }


def run_long(args, torch, dev, world, barrier):
    """Long signals: 8 float32 chirp mixtures of N = 1,048,576 (Npad 2,097,152),
    GMW(3,60), scales='log:maximal' (613 rows). Plain forward (one signal per
    call), batched forward (all 8 in one call) and forward + backward of
    MSE(|Tx(x)|, |Tx(y)|) + MSE(icwt(Wx(x)), y) one signal at a time. The
    backward keeps only the uint16 bin index of the forward (not Wx) and
    needs no recomputation of Wx."""
    import torch.distributed as dist
    import ssqueezepy_b200 as sb
    from ssqueezepy_b200 import _signals as S
    rank = int(os.environ.get('RANK', 0))
    B, N = 8, 1 << 20
    wav = ('gmw', {'gamma': 3., 'beta': 60., 'dtype': 'float32'})
    kw = dict(scales='log:maximal')
    xs = torch.tensor(S.same_length_batch(B, N, 4321 + rank), dtype=torch.float32,
                      device=dev)
    ys = torch.tensor(S.same_length_batch(B, N, 8765 + rank), dtype=torch.float32,
                      device=dev)
    st = torch.cuda.current_stream()
    steps = max(1, min(args.steps, 2))

    def timed(fn, n):
        fn()
        barrier()
        torch.cuda.reset_peak_memory_stats(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n):
            fn()
        e1.record(st)
        barrier()
        return e0.elapsed_time(e1) / n, torch.cuda.max_memory_allocated(dev) / 1e9

    na = int(sb.ssq_cwt(xs[0], wav, **kw)[1].shape[0])

    def plain():
        for i in range(B):
            sb.ssq_cwt(xs[i], wav, **kw)

    def batched():
        sb.ssq_cwt(xs, wav, **kw)

    with torch.no_grad():
        Ty = [sb.ssq_cwt(ys[i], wav, **kw)[0].abs() for i in range(B)]

    def fwd_bwd():
        for i in range(B):
            x = xs[i].clone().requires_grad_(True)
            Tx, Wx, _, _ = sb.ssq_cwt(x, wav, **kw)
            xr = sb.icwt(Wx, wav, x_len=N, **kw)
            del Wx
            loss = ((Tx.abs() - Ty[i]) ** 2).mean() + ((xr - ys[i]) ** 2).mean()
            del Tx, xr
            loss.backward()

    with torch.no_grad():
        p_ms, p_mem = timed(plain, steps)
        torch.cuda.empty_cache()
        b_ms, b_mem = timed(batched, steps)
    torch.cuda.empty_cache()
    fb_ms, fb_mem = timed(fwd_bwd, steps)
    del Ty
    torch.cuda.empty_cache()
    p_ms, b_ms, fb_ms = max_over_ranks([p_ms, b_ms, fb_ms], dev)
    hbm, src = peaks()
    fwd_bytes = B * N * (4 + 16 * na)
    bwd_bytes = B * N * (8 * na + 4 + 4)
    frac = lambda by, ms: by / (ms * 1e-3) / 1e9 / hbm
    return {
        "workload": "ssq_cwt, %d float32 chirp mixtures of N = %d, GMW(3,60), "
                    "scales='log:maximal' (%d rows), reflect" % (B, N, na),
        "plain_fwd": {"value": world * B * N / (p_ms * 1e-3), "ms": p_ms,
                      "hbm_frac": frac(fwd_bytes, p_ms), "peak_memory_gb": p_mem},
        "batched_fwd": {"value": world * B * N / (b_ms * 1e-3), "ms": b_ms,
                        "hbm_frac": frac(fwd_bytes, b_ms), "peak_memory_gb": b_mem},
        "fwd_bwd": {"value": world * B * N / (fb_ms * 1e-3), "ms": fb_ms,
                    "hbm_frac": frac(fwd_bytes + bwd_bytes, fb_ms),
                    "peak_memory_gb": fb_mem,
                    "note": "one signal per forward + backward; the backward keeps the "
                            "bin index, not Wx"},
        "unit": UNIT, "peak_source": src,
    }


def emit(args, world, N, na, Npad, step_ms_max, value, cwt_ms, sq_ms, e2e_value,
         launches, clocks, sc, f, const, Tg, Wg, batched=None, train=None, long_=None,
         stft_=None, next_=None, fp64_tf=None, idx_g=None):
    hbm, src = peaks()
    if True:
        alg_cwt = (4 + 8 * na) * N          # read x, write Wx
        alg_total = (4 + 16 * na) * N       # read x, write Wx and Tx
        cwt_avg = float(np.mean(cwt_ms))
        sq_avg = float(np.mean(sq_ms))
        dom, dom_ms, dom_bytes = (('cwt', cwt_avg, alg_cwt) if cwt_avg >= sq_avg else
                                  ('squeeze', sq_avg, 8 * na * N))
        achieved = dom_bytes / (dom_ms * 1e-3) / 1e9
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": step_ms_max,
            # the other workloads' headline figures (details in their own keys)
            "batched_samples_per_s": batched and batched["value"],
            "batched_vs_plain": batched and batched["speedup_vs_plain"],
            "batched_hbm_frac": batched and batched["roofline"]["frac"],
            "train_fwd_bwd_samples_per_s": train and train["fwd_bwd_value"],
            "train_fwd_bwd_over_fwd": train and train["fwd_bwd_over_fwd"],
            "long_fwd_samples_per_s": long_ and long_["plain_fwd"]["value"],
            "long_fwd_bwd_samples_per_s": long_ and long_["fwd_bwd"]["value"],
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "ssq_cwt N=%d GMW(3,60) nv=32 log-piecewise "
                                   "(%d rows) float32 reflect, one signal per GPU"
                                   % (N, na),
                       "arithmetic": args.arith,
                       "N": N, "na": na, "Npad": Npad, "batch_per_gpu": 1,
                       "l2": "252 MB buffer written between timed steps",
                       "parallelism": "dp%d" % world},
            "stages_ms": {"cwt": cwt_avg, "squeeze": sq_avg},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved,
                         "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None,
                         "traffic_source": "not re-captured: the last ncu dram__bytes "
                                           "read+write of the fused CWT (N=40,000, "
                                           "%.2f B per (row, sample)) was taken with the "
                                           "64 MB two-pass intermediate; this length now "
                                           "uses 512 MB, part of which lives in DRAM"
                                           % CWT_TRAFFIC_PER_ROW_SAMPLE,
                         "peak_source": src,
                         "path_frac": alg_total / (step_ms_max * 1e-3) / 1e9 / hbm},
            "compute_roofline": None if fp64_tf is None else {
                "kernel": "cwt", "bound": "fp64",
                "flops_per_call": 10.0 * Npad * np.log2(Npad) * na,
                "flop_count": "2 complex inverse FFTs of Npad per row, 5 Npad log2 Npad "
                              "each (radix-2 count); wavelet, twiddle and phase-transform "
                              "arithmetic not counted",
                "achieved": 10.0 * Npad * np.log2(Npad) * na / (cwt_avg * 1e-3) / 1e12,
                "peak": fp64_tf, "unit": "TFLOP/s",
                "frac": 10.0 * Npad * np.log2(Npad) * na / (cwt_avg * 1e-3) / 1e12 / fp64_tf,
                "peak_source": "measured here: cuBLAS float64 GEMM 4096^3"},
            "e2e": (None if e2e_value is None else
                    {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 4 * N,
                     "d2h_bytes_per_step": 8 * na * N,
                     "schedule": "public API from pinned host memory, steps alternating "
                                 "over two streams (a step's copy back overlaps the next "
                                 "step's transform)"}),
            "gpu_launches": launches * args.steps,
            "clocks": clocks,
        }
        if batched is not None:
            line["batched"] = batched
        if train is not None:
            line["fwd_bwd"] = train
        if long_ is not None:
            line["long"] = long_
        if stft_ is not None:
            line["stft"] = stft_
        if next_ is not None:
            line["next_rows"] = next_
        if world == 1 and not args.no_cpu:
            port, _ = cpu_path(N)
            x32 = chirp_signal(N, seed=0).astype(np.float32)
            ts = []
            for k in range(6):  # 3 warm-up calls, then the median of 3
                t0 = time.perf_counter()
                port(x32)
                ts.append(time.perf_counter() - t0)
            del port
            tc = float(np.median(ts[3:]))
            line["cpu_baseline"] = {
                "value": N / tc, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                "sample": CPU_SAMPLE % (N, os.cpu_count())}
            # parity on the float32 input the GPU saw (rounding of x not counted)
            from oracle import ssq_oracle as O
            x64 = x32.astype(np.float64)
            Wo, dWo = O.cwt(x64, 'gmw_l1', (3., 60.), sc)
            g = 10 * O.EPS32
            wo = O.phase_cwt(Wo, dWo, g)
            use = np.abs(Wo) > g
            ko = O.bin_index(np.where(use, wo, 1.), f, True, True)
            To = O.squeeze(Wo, ko, use, const)
            line["parity"] = {
                "input": "the float32 signal, as float64 (float32 input rounding excluded)",
                "Wx_rel_l2": float(np.linalg.norm(Wg - Wo) / np.linalg.norm(Wo)),
                "Tx_rel_l2": float(np.linalg.norm(Tg - To) / np.linalg.norm(To)),
                "bins": (None if idx_g is None else
                         O.bin_parity(idx_g, Wo, dWo, f, True, True, g))}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--no-cpu', action='store_true',
                    help='skip the CPU baseline / parity leg')
    ap.add_argument('--no-e2e', action='store_true',
                    help='skip the end-to-end (host buffers) leg')
    ap.add_argument('--arith', default='float64', choices=['float64', 'float32'],
                    help='arithmetic inside the transforms (data stay float32)')
    ap.add_argument('--no-batch', action='store_true',
                    help='skip the batched uneven-length leg')
    ap.add_argument('--batch', type=int, default=256,
                    help='signals in the batched leg (default 256)')
    ap.add_argument('--no-stft', action='store_true',
                    help='skip the ssq_stft leg')
    ap.add_argument('--no-long', action='store_true',
                    help='skip the 8 x 1,048,576 long-signal leg')
    ap.add_argument('--no-train', action='store_true',
                    help='skip the forward + backward (training loss) leg')
    ap.add_argument('--no-next', action='store_true',
                    help='skip the legs of the rows beside the path (higher-order '
                         'GMW, difftype phase, issq, ridges, istft)')
    ap.add_argument('--train-batch', type=int, default=64,
                    help='signals of N=16384 in the forward + backward leg')
    ap.add_argument('--n', type=int, default=N_SIG,
                    help='signal length (default 160000; smaller for profiling)')
    args = ap.parse_args()
    if args.impl == 'reference':
        return run_reference(args)
    return run_ours(args)


if __name__ == '__main__':
    sys.exit(main())
