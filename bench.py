"""Benchmark: plain FP32 filtered backprojection of a slice stack on B200.

Workload (the slice-stack case of the north star): 256 float32 sinograms of
1800 projections over [0, 180 deg) x 2560 detector pixels, exact projections
of a seeded 30-ellipsoid phantom (attenuation U(0.05, 0.5)) with Poisson
noise at 1e4 photons per pixel before the log, Hann filter, FFT length 4096,
centre of rotation +3.5 px, 2560 x 2560 float32 slices.  Inputs are generated
on the device (seeded, synthetic); 4.7 GB of input per step is larger than the
126 MB L2, so no flush is needed between steps.

One step = one pass of the hot path (filter + backprojection) over the stack.
    value : slices/s with sinograms and slices resident in HBM (device C-ABI
            call, CUDA events on the launching stream, max over ranks)
    e2e   : slices/s through the host C-ABI call (ctas_fbp_reconstruct_stack)
            from pinned host memory, host<->device copies inside the timed
            region, filtered sinograms written back as CTrec::reconstruct does
Also reported: Gupdates/s (N*W^2 per slice), error against the FP64 oracle on
sampled rows, the same run with the FP16-stored filtered sinogram, the roofline
of the dominant kernel (backprojection: shared-memory gather bound) and of the
filter (HBM bound), and the reference's CPU path timed on the host cores.

Multi-GPU: every rank reconstructs its own 256-slice stack (slices are
independent; no data-path collective), value = all slices / max rank time.
`--impl reference` times the reference's own CPU path -- its CTrec (lct.cpp
built in place into oracle/_ref, -O2) on its InThread pool, one slice per
thread -- on rank 0, with the as-shipped build (no -O) timed beside it.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_ANGLES, WIDTH, SLICES, PAD, CENTER = 1800, 2560, 256, 4096, 3.5
N_ELLIPSOIDS, PHOTONS, SEED = 30, 1.0e4, 20261203
BATCH_N = 64   # sinograms of the uneven-batch workload
WORKLOAD = ("slice stack: 256 x (1800 x 2560) float32 sinograms -> 2560 x 2560 float32 "
            "slices, Hann, FFT length 4096, centre +3.5 px, 30-ellipsoid phantom, "
            "Poisson 1e4 photons")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ inputs
def make_sinograms(torch, slices: int, seed: int, noise: bool = True):
    """Seeded synthetic stack on the device: exact ellipsoid projections,
    Poisson noise at PHOTONS, -log with the deAbs clamp (noise=False: the
    exact line integrals)."""
    from ctas_b200 import phantom as ph
    ell = ph.random_ellipsoids(seed, N_ELLIPSOIDS, WIDTH, slices, rho=(0.05, 0.5))
    # attenuation U(0.05, 0.5) per quarter field width: line integrals of
    # order 1, so the transmitted counts stay well above zero
    ell[:, 7] *= 4.0 / WIDTH
    per_slice = np.stack([ph.ellipsoid_sections(ell, z + 0.5) for z in range(slices)])
    out = torch.empty((slices, N_ANGLES, WIDTH), device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    for s0 in range(0, slices, 32):
        s1 = min(slices, s0 + 32)
        p = ph.sinogram_dev(per_slice[s0:s1], N_ANGLES, WIDTH, center=CENTER)
        if not noise:
            out[s0:s1] = p
            del p
            continue
        counts = torch.poisson(PHOTONS * torch.exp(-p), generator=g)
        tr = counts / PHOTONS
        mx = tr.amax(dim=(1, 2), keepdim=True)
        out[s0:s1] = -torch.log(torch.maximum(tr, mx / 1e6))
        del p, counts, tr
    return out


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.proc or not self.path:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, parts[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU leg
def cpu_reference_lct(sino: np.ndarray, threads: int, target_s: float, variant: str = "o2",
                      n_sub: int | None = None):
    """Time the reference's own CPU path: its CTrec (src/common/lct.cpp, built in
    place into oracle/_ref; `variant` "o2" = -O2 -ffast-math, "shipped" = its own
    flags, -ffast-math and no -O) reconstructing one slice per thread on the
    reference's InThread pool, one CTrec clone per thread (the ct tool's slice
    loop, ct.cpp:156-236).  Bounded sample: every k-th projection of the
    sinogram (n_sub of N, still evenly spaced over 180 degrees); filter and
    backprojection both do work proportional to the projection count, so the
    time is extrapolated by N / n_sub.  A subsampled sinogram stays in the
    cores' caches, so subsampling overstates the speed (about 2x at every 8th
    projection of 1800 x 2560): the timed legs use n_sub = N where the time
    allows.  The reference pads to its own rule, 8192 for 2560 pixels.  Returns
    (slices/s, description, n_sub, seconds)."""
    import oracle as O
    N, W = sino.shape

    def run(n):
        k = max(1, N // n)
        sub_ = np.ascontiguousarray(sino[::k][:n], np.float32)
        stack = np.ascontiguousarray(np.broadcast_to(sub_, (threads,) + sub_.shape))
        _, sec = O.lct_reconstruct_stack(stack, O.PHS, 5, 0.0, 180.0, CENTER, threads=threads,
                                         keep=False, variant=variant)
        return sec

    if n_sub is None:
        probe = 18
        sec = run(probe)
        n_sub = int(min(N, max(probe, round(target_s * probe / max(sec, 1e-6)))))
        n_sub = N // max(1, N // n_sub)
    sec = run(n_sub)
    slices_per_s = threads / (sec * N / n_sub)
    flags = "-O2 -ffast-math" if variant == "o2" else "-ffast-math, no -O (as shipped)"
    desc = (f"{threads} slices, one per thread, by the reference's CTrec (lct.cpp built in "
            f"place, {flags}) on its InThread pool ({threads} threads), on every "
            f"{N // n_sub}-th projection ({n_sub} of {N}, {sec:.1f} s), extrapolated to {N} "
            f"projections; reference padding 8192; Hann, centre {CENTER}")
    return slices_per_s, desc, n_sub, sec


def cpu_reference_sample(sino: np.ndarray, target_s: float, threads: int,
                         rows_hint: int | None = None):
    """Time the reference's CPU path on a bounded sample of one slice.

    Backprojection: the reference's own kernel (ct.cl) compiled for the host,
    run over evenly spaced rows of the slice with `threads` threads.  Filter:
    the oracle's restatement of prepare_sino (FFTW is absent), one thread, on
    a sample of projection rows.  Returns (slices/s, description, rows)."""
    import oracle as O
    N, W = sino.shape
    tab = O.angle_table(180.0, N)
    G = O.filter_window(5, 0.0, PAD, W, O.PHS)
    # filter: 64 projections, extrapolated to N
    nf = min(64, N)
    t0 = time.perf_counter()
    q_part = O.prepare_sino(sino[:nf], PAD, O.PHS, G)
    t_filter_slice = (time.perf_counter() - t0) * N / nf
    q = np.ascontiguousarray(np.tile(q_part, (N // nf + 1, 1))[:N])
    # backprojection rows: calibrate on a few rows, then size to target_s
    out = np.zeros((W, W), np.float32)
    if rows_hint is None:
        rows = np.linspace(0, W - 1, 2 * threads).astype(np.int64)
        t0 = time.perf_counter()
        O.ref_fbp_rows(q, tab, CENTER, 1.0, rows, out, threads)
        per_row = (time.perf_counter() - t0) * threads / len(rows)   # one thread
        rows_hint = int(max(threads, min(W, target_s * threads / max(per_row, 1e-6))))
    rows = np.linspace(0, W - 1, rows_hint).astype(np.int64)
    t0 = time.perf_counter()
    O.ref_fbp_rows(q, tab, CENTER, 1.0, rows, out, threads)
    t_rows = time.perf_counter() - t0
    t_bp_slice = t_rows * W / len(rows)          # with `threads` threads
    # `threads` slices in flight, one per thread (RecInThread, ct.cpp:156-206)
    slices_per_s = 1.0 / (t_bp_slice + t_filter_slice / threads)
    desc = (f"{len(rows)} evenly spaced rows of one 1800x2560 slice backprojected by the "
            f"reference's ct.cl kernel (compiled for the host, -O2) on {threads} threads "
            f"({t_rows:.1f} s) + filter of {nf} projections by the oracle's FFTW "
            f"restatement (1 thread), extrapolated to whole slices")
    return slices_per_s, desc, rows_hint, t_rows + t_filter_slice * nf / N


# ------------------------------------------------------------------ roofline
def roofline(bp_ms_per_launch, slices_per_launch, filter_ms_per_launch, smem_peak_gbs,
             clocks, sms, l2_peak_gbs=None, tile=None):
    import oracle as O
    from ctas_b200 import ct
    mask = O.mask(WIDTH, CENTER)
    inmask = int(mask.sum())
    bp_bytes = 4.0 * N_ANGLES * inmask * slices_per_launch    # 4 B fetched per update
    achieved = bp_bytes / (bp_ms_per_launch * 1e-3) / 1e9
    # detector windows the staged kernel copies from L2 by TMA: one window of
    # `box` samples per projection for every tile that has a pixel in the disc
    l2 = None
    if tile is not None and tile >= 0 and l2_peak_gbs:
        ty, tx, box = ct.tile_shape(tile)
        active = sum(1 for j0 in range(0, WIDTH, ty) for i0 in range(0, WIDTH, tx)
                     if mask[j0:j0 + ty, i0:i0 + tx].any())
        wbytes = 4.0 * box * N_ANGLES * active * slices_per_launch
        l2_ach = wbytes / (bp_ms_per_launch * 1e-3) / 1e9
        l2 = {"window_bytes_per_launch": wbytes, "achieved": round(l2_ach, 1),
              "peak": round(l2_peak_gbs, 1), "frac": round(l2_ach / l2_peak_gbs, 4),
              "unit": "GB/s", "peak_source": "measured in this run by ctas_probe_l2_read "
                                            "(16-byte L2 reads of a 32 MiB buffer)"}
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f)
        if "bp_fast_per_slice_bytes" in tr:
            traffic = tr["bp_fast_per_slice_bytes"] * slices_per_launch
    filt_bytes = 4.0 * N_ANGLES * WIDTH * 2 * slices_per_launch   # read + write rows
    hbm_peak = 6541.8
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        with open(mp) as f:
            hbm_peak = float(json.load(f).get("hbm_gbs", hbm_peak))
    f_ach = filt_bytes / (filter_ms_per_launch * 1e-3) / 1e9 if filter_ms_per_launch else None
    # the filter's binding term: a row pair's FFT of length PAD in radix-8/4/2
    # stages makes 4 ns - 4 passes over PAD complex floats in shared memory
    # (first stage from global memory, last stage to it, the middle stage and
    # every other stage read and written once)
    ns = int(np.ceil(np.log2(PAD) / 3))
    smem_b = ((N_ANGLES + 1) // 2) * (4 * ns - 4) * PAD * 8.0 * slices_per_launch
    nominal_smem = 128.0 * sms * (clocks.get("sm_mhz") or 1965.0) * 1e6 / 1e9
    f_smem = None
    if filter_ms_per_launch:
        a_smem = smem_b / (filter_ms_per_launch * 1e-3) / 1e9
        f_smem = {"bytes_per_launch": smem_b, "achieved": round(a_smem, 1),
                  "peak": round(nominal_smem, 1), "frac": round(a_smem / nominal_smem, 4),
                  "unit": "GB/s", "note": "shared-memory traffic of the FFT stages against "
                  "the nominal 128 B/clk/SM; this term, not HBM, bounds the filter"}
    nominal = 128.0 * sms * (clocks.get("sm_mhz") or 1965.0) * 1e6 / 1e9
    return {
        "bound": "smem", "kernel": "bp_fast (backprojection)", "unit": "GB/s",
        "achieved": round(achieved, 1), "peak": round(nominal, 1),
        "frac": round(achieved / nominal, 4),
        "peak_source": "nominal shared-memory load bandwidth: 128 B/clk/SM x SMs x the median "
                       "SM clock under load (no shared-memory figure in MEASURED_PEAKS.json)",
        "probe": {"peak": round(smem_peak_gbs, 1), "frac": round(achieved / smem_peak_gbs, 4),
                  "probe_frac_of_nominal": round(smem_peak_gbs / nominal, 4),
                  "source": "measured in this run by ctas_probe_smem_gather (conflict-free "
                            "32-bit shared loads and adds)"},
        "l2_windows": l2,
        "traffic": traffic,
        "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of "
                          "this kernel (profiles/ncu_traffic.json, per slice, scaled to the "
                          "launch): a committed measurement, not taken in this run",
        "algorithmic_bytes_per_launch": bp_bytes,
        "unit_note": "4 B per in-mask update (N x in-mask pixels per slice)",
        "filter": {"bound": "hbm", "unit": "GB/s",
                   "achieved": round(f_ach, 1) if f_ach else None, "peak": hbm_peak,
                   "frac": round(f_ach / hbm_peak, 4) if f_ach else None,
                   "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                   "smem_passes": f_smem},
    }


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slices", type=int, default=SLICES)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--train-steps", type=int, default=1500,
                    help="learned workload: Adam steps on 256 x 256 crops")
    ap.add_argument("--train-phantoms", type=int, default=96,
                    help="learned workload: training phantoms, generated on the GPU while "
                         "training (a pool of 128 is refreshed 16 at a time); the full case "
                         "uses 20000")
    ap.add_argument("--eval-phantoms", type=int, default=8,
                    help="learned workload: held-out phantoms (the full case uses 200)")
    ap.add_argument("--vol-full", type=int, default=0,
                    help="volume workload: also stream this many slices (2048 = the full "
                         "case) through the volume call, the sample's sinograms repeating")
    ap.add_argument("--quick", action="store_true",
                    help="only the timed device-resident stack (for profiler runs)")
    ap.add_argument("--workload", default="stack",
                    choices=["stack", "axis", "ts", "volume", "learned", "batch"],
                    help="stack: the slice-stack reconstruction (default); axis: the "
                         "rotation-axis search on one sinogram of the same data; ts: "
                         "tomosynthesis (ts_add) of a projection series; volume: the "
                         "large streamed volume (3600 x 4096 sinograms from host memory); "
                         "learned: sparse-angle FBP + U-Net against full-angle FBP; batch: "
                         "an uneven batch of 64 sinograms as one CUDA graph vs a launch loop")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "axis":
        return run_axis(args, rank, world, local)
    if args.workload == "ts":
        return run_ts(args, rank, world, local)
    if args.workload == "batch":
        return run_batch(args, rank, world, local)
    if args.workload == "volume":
        return run_volume(args, rank, world, local)
    if args.workload == "learned":
        return run_learned(args, rank, world, local)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from ctas_b200 import ct

    S = args.slices
    log(f"[rank {rank}] generating {S} sinograms on cuda:{local}")
    sinos = make_sinograms(torch, S, SEED + rank)
    slices = torch.empty((S, WIDTH, WIDTH), device="cuda")
    torch.cuda.synchronize()

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        from ctas_b200.replicas import max_over_ranks as mor
        return mor(x, device="cuda")

    rec = ct.CTrec((N_ANGLES, WIDTH), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), pad=PAD,
                   device=local)
    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        rec.reconstruct_stack_dev(sinos, slices, CENTER, stream.cuda_stream)
    barrier()
    rec.profile_read(0)
    rec.profile_read(1)
    rec.set_profiling(True)
    launches0 = rec.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            rec.reconstruct_stack_dev(sinos, slices, CENTER, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        barrier()
    rec.set_profiling(False)
    launches = rec.kernel_launches() - launches0
    ms = max_over_ranks(e0.elapsed_time(e1))
    f_ms, f_n = rec.profile_read(0)
    b_ms, b_n = rec.profile_read(1)
    clocks = clk.summary()
    total_slices = S * args.steps * world
    value = total_slices / (ms * 1e-3)
    gup = value * N_ANGLES * WIDTH * WIDTH / 1e9
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": "slices/s", "value": round(value, 3), "unit": "slices/s",
                              "quick": True, "slices": S, "steps": args.steps,
                              "kernel_ms": {"filter": f_ms / max(f_n, 1),
                                            "backprojection": b_ms / max(b_n, 1)}}), flush=True)
        if dist:
            dist.destroy_process_group()
        return

    # ---- error against the FP64 oracle on sampled rows of slice 0
    import oracle as O
    s0 = sinos[0].cpu().numpy()
    out0 = slices[0].cpu().numpy()
    qd = O.prepare_sino(s0, PAD, O.PHS, O.filter_window(5, 0.0, PAD, WIDTH, O.PHS, fp64=True),
                        fp64=True)
    tab = O.angle_table(180.0, N_ANGLES)
    rows = np.linspace(200, WIDTH - 200, 12).astype(int)
    ref64 = np.concatenate([O.bp_compat(qd, tab, CENTER, 1.0, rows=(int(r), int(r) + 1))
                            for r in rows])
    got = out0[rows]
    m = O.mask(WIDTH, CENTER)[rows]
    rel_rmse = float(np.sqrt(np.mean((got[m] - ref64[m]) ** 2)) / np.sqrt(np.mean(ref64[m] ** 2)))
    max_abs_rel = float(np.abs(got[m] - ref64[m]).max() / (ref64[m].max() - ref64[m].min()))

    # ---- FP16-stored filtered sinograms (FP32 accumulation)
    rec16 = ct.CTrec((N_ANGLES, WIDTH), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), pad=PAD,
                     store=1, device=local)
    for _ in range(2):
        rec16.reconstruct_stack_dev(sinos, slices, CENTER, stream.cuda_stream)
    barrier()
    rec16.profile_read(0)
    rec16.profile_read(1)
    rec16.set_profiling(True)
    e0.record(stream)
    for _ in range(max(1, args.steps // 2)):
        rec16.reconstruct_stack_dev(sinos, slices, CENTER, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    ms16 = max_over_ranks(e0.elapsed_time(e1))
    f16_ms, f16_n = rec16.profile_read(0)
    b16_ms, b16_n = rec16.profile_read(1)
    tile16 = rec16.last_tile()
    v16 = S * max(1, args.steps // 2) * world / (ms16 * 1e-3)
    got16 = slices[0].cpu().numpy()[rows]
    rel16 = float(np.sqrt(np.mean((got16[m] - ref64[m]) ** 2)) / np.sqrt(np.mean(ref64[m] ** 2)))
    rec16.close()

    # ---- roofline of the dominant kernel
    smem_peak = ct.probe_smem_gather(local) / 1e9
    l2_peak = ct.probe_l2_read(local) / 1e9
    props = torch.cuda.get_device_properties(local)
    per_launch = S / max(1, b_n // args.steps) if b_n else S
    roof = roofline(b_ms / max(b_n, 1), per_launch, f_ms / max(f_n, 1), smem_peak, clocks,
                    props.multi_processor_count, l2_peak, rec.last_tile())

    # ---- end to end through the host C ABI (pinned host buffers)
    # The call filters the host stack in place, so every step first restores it
    # from the device copy (outside the timed region): no second host copy, so
    # that 8 ranks on one node hold 8 x 11.4 GB of pinned host memory, no more.
    del slices
    torch.cuda.empty_cache()
    h_in = torch.empty((S, N_ANGLES, WIDTH), dtype=torch.float32, pin_memory=True)
    h_in.copy_(sinos)
    h_out = torch.empty((S, WIDTH, WIDTH), dtype=torch.float32, pin_memory=True)
    np_in, np_out = h_in.numpy(), h_out.numpy()
    rec_h = ct.CTrec((N_ANGLES, WIDTH), ct.Contrast.PHS, 180.0, ct.Filter("HANN"), pad=PAD,
                     device=local)
    rec_h.reconstruct_stack(np_in[:8], np_out[:8], CENTER)   # warm-up
    times = []
    for _ in range(args.e2e_steps):
        h_in.copy_(sinos)              # the call writes the filtered stack back
        barrier()
        t0 = time.perf_counter()
        rec_h.reconstruct_stack(np_in, np_out, CENTER)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(float(np.median(times)))
    e2e_val = S * world / e2e_s
    rec_h.close()

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            import oracle as O2
            if O2.lct_available("o2"):
                threads = os.cpu_count() or 1
                v, desc, _, _ = cpu_reference_lct(sinos[0].cpu().numpy(), threads, 15.0)
                cpu = {"value": round(v, 6), "unit": "slices/s", "cores": threads,
                       "kind": "reference", "sample": desc}
            else:
                cpu = {"value": None, "unit": "slices/s", "cores": 0, "kind": "reference",
                       "sample": "oracle/_ref not built on this machine"}
        except Exception as exc:  # the GPU numbers stand without it
            cpu = {"value": None, "unit": "slices/s", "cores": 0, "kind": "reference",
                   "sample": f"failed: {exc}"}

    if rank == 0:
        # the graded fraction of the whole step: t_bound / t_measured per slice,
        # t_bound = max(compulsory HBM bytes / HBM peak, dense updates x 4 B /
        # nominal shared-memory fetch peak at the maximum SM clock)
        hbm_b = 4.0 * N_ANGLES * WIDTH * 3 + 4.0 * WIDTH * WIDTH + 8.0 * N_ANGLES
        fetch_peak = 128.0 * props.multi_processor_count * (clocks.get("sm_max_mhz") or 1965.0) * 1e6
        t_bound = max(hbm_b / (roof["filter"]["peak"] * 1e9),
                      4.0 * N_ANGLES * WIDTH * WIDTH / fetch_peak)
        t_meas = (ms / args.steps) * 1e-3 / S
        roof["step_graded"] = {
            "t_bound_ms_per_slice": round(t_bound * 1e3, 4),
            "t_measured_ms_per_slice": round(t_meas * 1e3, 4),
            "frac": round(t_bound / t_meas, 4),
            "fetch_peak_gbs": round(fetch_peak / 1e9, 1),
            "convention": "dense N x W^2 updates at 4 B each against 128 B/clk/SM at the "
                          "maximum SM clock; HBM term: raw read, filtered write and read, "
                          "slice write"}
        line = {
            "metric": "slices/s", "value": round(value, 3), "unit": "slices/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded ellipsoid phantom, exact projections, Poisson noise)",
            "config": {"workload": WORKLOAD, "slices_per_gpu": S, "n_angles": N_ANGLES,
                       "width": WIDTH, "pad": PAD, "filter": "HANN", "center": CENTER,
                       "contrast": "PHS", "l2": "inputs 4.7 GB per step > 126 MB L2; no flush",
                       "parallelism": f"replicas x{world} (independent slices)"},
            "gupdates_per_s": round(gup, 1),
            "gupdates_per_s_in_mask": round(gup * float(O.mask(WIDTH, CENTER).mean()), 1),
            "error_vs_fp64": {"rel_rmse": rel_rmse, "max_abs_over_range": max_abs_rel,
                              "rows": len(rows)},
            "fp16_store": {"value": round(v16, 3), "unit": "slices/s", "rel_rmse_vs_fp64": rel16,
                           "filter_ms_avg": f16_ms / max(f16_n, 1),
                           "backprojection_ms_avg": b16_ms / max(b16_n, 1), "bp_tile": tile16},
            "e2e": {"value": round(e2e_val, 3), "unit": "slices/s",
                    "h2d_bytes_per_step": 4 * S * N_ANGLES * WIDTH,
                    "d2h_bytes_per_step": 4 * S * (WIDTH * WIDTH + N_ANGLES * WIDTH),
                    "call": "ctas_fbp_reconstruct_stack (host buffers, pinned)"},
            "gpu_launches": int(launches),
            "bp_tile": rec.last_tile(),
            "kernel_ms": {"filter_avg": f_ms / max(f_n, 1), "filter_launches": f_n,
                          "backprojection_avg": b_ms / max(b_n, 1), "backprojection_launches": b_n},
            "roofline": roof,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


AXIS_MAX_DEV = 0.05


def run_axis(args, rank, world, local):
    """Rotation-axis search (raxis algorithm 1: average-gradient grid of 33
    centres at max_dev 0.05, then bisection) on one absorption sinogram of the
    benchmark data (1800 x 2560, true axis 0.5 (W-1) + 3.5).  Rank 0 only (one
    sinogram; replicas would search their own).
        value : average-gradient trials/s of the grid phase through
                AverageGradient.apply (33 centres: multi-centre
                backprojection + smoothing/Sobel/mean kernel; synchronous call)
        e2e   : whole searches through ctas_raxis from the host sinogram
                (upload, filter, every trial), searches/s
    cpu_baseline: the reference's per-trial cost on the host -- one slice
    backprojected by its ct.cl kernel per thread, all threads busy as
    AGinThread runs the grid (the FFT smoothing is not counted: FFTW absent)."""
    if rank != 0:
        return
    import torch
    from ctas_b200 import axis, ct
    torch.cuda.set_device(local)
    # exact projections: with Poisson noise the reference's metric is minimal at
    # centre 0 whatever the axis (its noise-dominated sum is divided by a region
    # that shrinks with |centre|), so noise-free data show where it finds the axis
    sino = make_sinograms(torch, 1, SEED, noise=False)[0]
    T = torch.exp(-sino).cpu().numpy()            # transmission for the ABS contrast
    cent = 0.5 * (WIDTH - 1)
    true_axis = cent + CENTER
    steps = int(1 + 2 * (AXIS_MAX_DEV * WIDTH / 8))
    grid = (np.float32(cent) + np.float32(8) * (np.arange(steps) - (steps - 1) // 2)).astype(np.float32)
    # grid phase through the public AverageGradient
    with axis.AverageGradient(T, 180.0, device=local) as ag:
        for _ in range(max(1, args.warmup)):
            ag.apply(grid)
        times = []
        with ClockSampler(local) as clk:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                ag.apply(grid)
                times.append(time.perf_counter() - t0)
        clocks = clk.summary()
        sigma, taps = ag.sigma, ag.taps
    grid_s = float(np.median(times))
    value = steps / grid_s
    # the backprojection alone, device-timed (CUDA events, same centres)
    rec = ct.CTrec((N_ANGLES, WIDTH), ct.Contrast.ABS, 180.0, ct.Filter("RAMP"),
                   no_writeback=True, device=local)
    rec.sino(T.copy())
    out = torch.empty((steps, WIDTH, WIDTH), device="cuda")
    cs = grid - np.float32(cent)
    stream = torch.cuda.current_stream()
    for _ in range(2):
        rec.repeat_multi_dev(cs, out, stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        rec.repeat_multi_dev(cs, out, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    bp_ms = e0.elapsed_time(e1) / args.steps
    rec.close()
    del out
    # whole searches through the C ABI from host memory
    found, trials = axis.raxis(T, 180.0, AXIS_MAX_DEV, 1, device=local, return_trials=True)
    st = []
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        axis.raxis(T, 180.0, AXIS_MAX_DEV, 1, device=local)
        st.append(time.perf_counter() - t0)
    search_s = float(np.median(st))
    cpu = None
    if not args.no_cpu:
        try:
            import oracle as O
            if O.ref_available():
                threads = os.cpu_count() or 1
                v, desc, _, _ = cpu_reference_sample(-np.log(T), 10.0, threads)
                cpu = {"value": round(v, 6), "unit": "trials/s", "cores": threads,
                       "kind": "reference",
                       "sample": desc + "; one trial = one slice backprojection per thread"}
        except Exception as exc:
            cpu = {"value": None, "unit": "trials/s", "cores": 0, "kind": "reference",
                   "sample": f"failed: {exc}"}
    line = {
        "metric": "axis-search trials/s", "value": round(value, 3), "unit": "trials/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * grid_s, 3), "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (slice 0 of the benchmark phantom, exact projections as transmission)",
        "config": {"workload": f"raxis algorithm 1 on one 1800 x 2560 absorption sinogram, "
                               f"max_dev {AXIS_MAX_DEV}: grid of {steps} centres + bisection",
                   "grid_centres": steps, "sigma_px": round(sigma, 4), "gauss_taps": taps},
        "bp_ms_per_grid_device": round(bp_ms, 3),
        "bp_ms_per_trial_device": round(bp_ms / steps, 4),
        "e2e": {"value": round(1.0 / search_s, 4), "unit": "searches/s",
                "ms_per_search": round(1e3 * search_s, 1), "trials": int(trials),
                "axis": round(float(found), 4), "true_axis": true_axis,
                "h2d_bytes_per_step": 4 * N_ANGLES * WIDTH, "d2h_bytes_per_step": 4,
                "call": "ctas_raxis (host sinogram)"},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


TS_ROWS, TS_PIXELS, TS_PROJ = 2048, 2560, 61


def ts_cpu_port(proj: np.ndarray, rows: int, angle: float, plane: int, center: float):
    """ts_add restated with numpy (real FFT of each row's own length, as FFTW's
    R2HC/HC2R pair; ABS -log; the float projection step) on one thread, for
    `rows` rows: the CPU reference path of the ts tool (single-threaded)."""
    import oracle as O
    n = proj.shape[1]
    fw = O.filter_fill_plain(1, 0.0, n).astype(np.float32)
    fr = fw[: n // 2 + 1]                      # even window: rfft bins 0 .. n/2
    p = -np.log(proj[:rows])
    f = np.fft.irfft(np.fft.rfft(p, axis=1) * fr[None, :], n=n, axis=1).astype(np.float32)
    cs, cc = np.float32(np.sin(np.float32(angle))), np.float32(np.cos(np.float32(angle)))
    pc = np.float32(np.float32(plane) - np.float32(center)) * cs
    rc = np.float32(n * 0.5 + center)
    di = ((np.arange(n, dtype=np.float32) - rc) * cc - pc + rc).astype(np.float32)
    idx = np.clip(di, 0, n - 1).astype(np.int64)
    return f[:, idx]


def run_batch(args, rank, world, local):
    """Uneven batch: BATCH_N float32 sinograms whose widths and projection
    counts are drawn by seed (widths {1024, 1536, 2048, 3072, 4096},
    projections {900, 1800, 2400, 3600} over 180 degrees, centre U(-8, 8) px),
    random-ellipse phantoms scaled to the width, Shepp-Logan window, the
    reference padding rule, W x W slices.  Rank 0 only.
        value : slices/s of one batch as one CUDA graph (a filter launch over
                every sinogram's row pairs + one persistent backprojection)
        loop  : the same batch as a per-sinogram launch loop
    Both device-resident, CUDA events on the launching stream."""
    if rank != 0:
        return
    import torch
    from ctas_b200 import ct
    from ctas_b200 import phantom as ph
    torch.cuda.set_device(local)
    rng = np.random.default_rng(SEED)
    widths = rng.choice([1024, 1536, 2048, 3072, 4096], BATCH_N)
    counts = rng.choice([900, 1800, 2400, 3600], BATCH_N)
    centres = rng.uniform(-8.0, 8.0, BATCH_N)
    jobs, dense = [], 0.0
    for k in range(BATCH_N):
        W, N = int(widths[k]), int(counts[k])
        el = ph.random_ellipses(SEED + k, 12, W, scale=W / 2048.0)
        sino = ph.sinogram_dev(el[None], N, W, center=float(centres[k]))[0].contiguous()
        jobs.append((sino, torch.zeros((W, W), device="cuda"), float(centres[k])))
        dense += float(N) * W * W
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    b = ct.Batch(jobs, ct.Contrast.PHS, 180.0,
                 ct.Filter("SHEPP-LOGAN"))
    create_s = time.perf_counter() - t0
    res = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        for form, run in (("graph", b.run), ("loop", b.run_loop)):
            for _ in range(max(1, args.warmup)):
                run(stream.cuda_stream)
            torch.cuda.synchronize()
            ms = []
            for _ in range(args.steps):
                e0.record(stream)
                run(stream.cuda_stream)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
            res[form] = float(np.median(ms))
    clocks = clk.summary()
    tile = b.tile()
    b.close()
    value = BATCH_N / (res["graph"] * 1e-3)
    print(json.dumps({
        "metric": "slices/s", "value": round(value, 2), "unit": "slices/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(res["graph"], 3),
        "higher_is_better": True, "scaling": "none", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random-ellipse phantoms, exact projections)",
        "config": {"workload": f"uneven batch: {BATCH_N} sinograms, widths 1024-4096, "
                               "900-3600 projections over 180 deg, Shepp-Logan, reference "
                               "padding, W x W slices",
                   "dense_updates": dense},
        "gupdates_per_s_dense": round(dense / (res["graph"] * 1e-3) / 1e9, 1),
        "loop": {"value": round(BATCH_N / (res["loop"] * 1e-3), 2), "unit": "slices/s",
                 "ms_per_batch": round(res["loop"], 3)},
        "tile": tile, "create_s": round(create_s, 2), "clocks": clocks}), flush=True)


def run_ts(args, rank, world, local):
    """Tomosynthesis (the ts tool): TS_PROJ absorption projections of
    TS_ROWS x TS_PIXELS over +-30 degrees, each filtered with the RAMP window
    of its own row length and added into one plane (ts_add, lct.cpp:731-787).
    Rank 0 only.
        value : projections/s, device-resident, one batched call per step
                (filter + ordered backprojection + write-back of the filtered
                projections, as ts_add leaves them)
        e2e   : projections/s through the host call, one projection per call
                as ts.cpp:209-217 does (host image in, result and filtered
                image out)
    cpu_baseline: a one-thread numpy port of ts_add (the ts tool is
    single-threaded; FFTW is absent) on a row sample, extrapolated."""
    if rank != 0:
        return
    import torch
    from ctas_b200 import ct, ts
    torch.cuda.set_device(local)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    x = torch.linspace(-1, 1, TS_PIXELS, device="cuda")
    yy = torch.linspace(-1, 1, TS_ROWS, device="cuda")[:, None]
    base = 0.55 + 0.35 * torch.exp(-((x[None, :] / 0.35) ** 2 + (yy / 0.5) ** 2))
    projs = torch.empty((TS_PROJ, TS_ROWS, TS_PIXELS), device="cuda")
    for i in range(TS_PROJ):
        projs[i] = base * (1 + 0.02 * torch.randn((TS_ROWS, TS_PIXELS), device="cuda",
                                                  generator=g)).clamp_(0.5, 1.5)
    keep = projs.clone()
    angles = np.deg2rad(np.linspace(-30, 30, TS_PROJ)).astype(np.float32)
    result = torch.zeros((TS_ROWS, TS_PIXELS), device="cuda")
    center, plane = 3.5, 40
    t = ts.TS((TS_ROWS, TS_PIXELS), ct.Filter("RAMP"), ct.Contrast.ABS, device=local)
    stream = torch.cuda.current_stream()
    for _ in range(max(1, args.warmup)):
        projs.copy_(keep)
        t.add_batch_dev(projs, angles, result, center, plane, stream=stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            projs.copy_(keep)              # ts_add filters its input in place
            result.zero_()
            e0.record(stream)
            t.add_batch_dev(projs, angles, result, center, plane, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    clocks = clk.summary()
    step_ms = float(np.median(ms))
    value = TS_PROJ / (step_ms * 1e-3)
    img = 4.0 * TS_ROWS * TS_PIXELS
    bytes_per_proj = 5 * img                  # filter r+w, backprojection read, write-back r+w
    achieved = bytes_per_proj * TS_PROJ / (step_ms * 1e-3) / 1e9
    hbm_peak = 6541.8
    mp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(mp):
        with open(mp) as f:
            hbm_peak = float(json.load(f).get("hbm_gbs", hbm_peak))
    # end to end from host memory, one projection per call
    h_keep = keep.cpu().numpy()
    h_res = np.zeros((TS_ROWS, TS_PIXELS), np.float32)
    h_img = h_keep[0].copy()
    t.add(h_img, h_res, center, float(angles[0]), plane)        # warm-up
    n_e2e = min(TS_PROJ, 16)
    imgs = [h_keep[i].copy() for i in range(n_e2e)]
    t0 = time.perf_counter()
    for i in range(n_e2e):
        t.add(imgs[i], h_res, center, float(angles[i]), plane)
    e2e_s = time.perf_counter() - t0
    t.close()
    cpu = None
    if not args.no_cpu:
        rows = 128
        t0 = time.perf_counter()
        ts_cpu_port(h_keep[1], rows, float(angles[1]), plane, center)
        dt = time.perf_counter() - t0
        cpu = {"value": round(rows / (dt * TS_ROWS), 4), "unit": "projections/s", "cores": 1,
               "kind": "port",
               "sample": f"{rows} of {TS_ROWS} rows of one projection through a numpy port of "
                         f"ts_add (row FFTs, -log, projection step) on one thread "
                         f"({dt:.2f} s), extrapolated"}
    line = {
        "metric": "tomosynthesis projections/s", "value": round(value, 2),
        "unit": "projections/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_ms, 3), "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (smooth absorption projections with 2 % seeded noise)",
        "config": {"workload": f"ts_add of {TS_PROJ} projections {TS_ROWS} x {TS_PIXELS} over "
                               f"+-30 deg into plane {plane}, centre {center}, RAMP, ABS",
                   "fft_length": 8192},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm_peak,
                     "unit": "GB/s", "frac": round(achieved / hbm_peak, 4), "traffic": None,
                     "algorithmic_bytes_per_projection": bytes_per_proj},
        "e2e": {"value": round(n_e2e / e2e_s, 2), "unit": "projections/s",
                "h2d_bytes_per_step": 2 * int(img), "d2h_bytes_per_step": 2 * int(img),
                "call": "ctas_ts_add (host images, one per call)"},
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


VOL_N, VOL_W, VOL_PAD, VOL_CENTER, VOL_PHOTONS = 3600, 4096, 8192, 12.25, 5.0e3


def _vol_texture(tex_seed, z):
    """The band-limited texture of section z: a Gaussian random field of
    standard deviation 0.05 in the attenuation units of the ellipsoids (their
    densities U(0.05, 0.5) scaled by 4/W), correlation length 8 px."""
    from ctas_b200 import phantom as ph
    return ph.grf_texture_dev(tex_seed + int(z), VOL_W, std=0.05 * 4.0 / VOL_W, corr_px=8.0,
                              center=VOL_CENTER)


def _vol_sinos_dev(ell, z_list, g, tex_seed):
    """Noisy -log sinograms (3600 x 4096, centre +12.25, Poisson 5e3) of the
    sections at heights z + 0.5 of an ellipsoid volume plus their texture
    (ray-marched), on the device."""
    import torch
    from ctas_b200 import phantom as ph
    per = np.stack([ph.ellipsoid_sections(ell, z + 0.5) for z in z_list])
    p = ph.sinogram_dev(per, VOL_N, VOL_W, center=VOL_CENTER)
    tex = torch.cat([_vol_texture(tex_seed, z) for z in z_list])
    ph.project_image_dev(tex, VOL_N, center=VOL_CENTER, out=p)
    tr = torch.poisson(VOL_PHOTONS * torch.exp(-p), generator=g) / VOL_PHOTONS
    mx = tr.amax(dim=(1, 2), keepdim=True)
    return -torch.log(torch.maximum(tr, mx / 1e6))


def _volume_learned(args, h_in, h_out, S, local, picks):
    """Learned every-4th-angle form of the streamed volume: a U-Net trained on
    pairs (FBP of every 4th of the 3600 projections -> full-angle FBP) from a
    separate 24-slice phantom volume of the same kind, then the S sinograms
    streamed from pinned host memory: H2D of the sinograms, every 4th
    projection taken on the device, 900-angle filter + backprojection, U-Net,
    D2H of the slices, on three streams with two device buffer sets.  Wall
    clock around the whole stream."""
    import torch
    from ctas_b200 import ct, learned
    from ctas_b200 import phantom as ph
    K, n_train, C = 4, 24, 4
    filt = ct.Filter("HAMMING")
    full_rec = ct.CTrec((VOL_N, VOL_W), ct.Contrast.PHS, 180.0, filt, pad=VOL_PAD,
                        no_writeback=True, device=local)
    sparse_rec = ct.CTrec((VOL_N // K, VOL_W), ct.Contrast.PHS, 180.0, filt, pad=VOL_PAD,
                          no_writeback=True, device=local)
    ell = ph.random_ellipsoids(SEED + 5, 40, VOL_W, n_train, rho=(0.05, 0.5))
    ell[:, 7] *= 4.0 / VOL_W
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED + 5)
    xs, ys = [], []
    for s0 in range(0, n_train, 4):
        sino = _vol_sinos_dev(ell, range(s0, s0 + 4), g, SEED + 60_000)
        full = torch.empty((4, VOL_W, VOL_W), device="cuda")
        sparse = torch.empty((4, VOL_W, VOL_W), device="cuda")
        full_rec.reconstruct_stack_dev(sino, full, VOL_CENTER)
        sparse_rec.reconstruct_stack_dev(sino[:, ::K].contiguous(), sparse, VOL_CENTER)
        xs.append(sparse)
        ys.append(full)
        del sino
    xtr, ytr = torch.cat(xs), torch.cat(ys)
    del xs, ys
    net = learned.UNet(seed=SEED, scale=float(1.0 / ytr.std()), device=local)
    gc = torch.Generator(device="cuda")
    gc.manual_seed(SEED)
    Bc, Cr = 8, 256
    ar = torch.arange(Cr, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = []
    for step in range(args.train_steps):
        idx = torch.randint(0, n_train, (Bc,), device="cuda", generator=gc)
        oy = torch.randint(0, VOL_W - Cr + 1, (Bc,), device="cuda", generator=gc)
        ox = torch.randint(0, VOL_W - Cr + 1, (Bc,), device="cuda", generator=gc)
        rows = (oy[:, None] + ar[None, :])[:, :, None]
        cols = (ox[:, None] + ar[None, :])[:, None, :]
        xb = xtr[idx[:, None, None], rows, cols].contiguous()
        yb = ytr[idx[:, None, None], rows, cols].contiguous()
        losses.append(net.train_step(xb, yb, 1e-3 if step < 0.8 * args.train_steps else 2e-4))
    t_train = time.perf_counter() - t0
    del xtr, ytr
    torch.cuda.empty_cache()
    log(f"[volume] learned form trained in {t_train:.1f} s (loss {losses[0]:.2e} -> "
        f"{float(np.mean(losses[-50:])):.2e})")
    # streamed: two device buffer sets, three streams
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    s_cmp = torch.cuda.current_stream()
    d_sino = [torch.empty((C, VOL_N, VOL_W), device="cuda") for _ in range(2)]
    d_sparse = [torch.empty((C, VOL_W, VOL_W), device="cuda") for _ in range(2)]
    d_out = [torch.empty((C, VOL_W, VOL_W), device="cuda") for _ in range(2)]
    d_sparse_keep = {}

    def stream_all(keep=()):
        ev_out = [None, None]
        for k, s0 in enumerate(range(0, S, C)):
            s1, b = min(S, s0 + C), k & 1
            n = s1 - s0
            with torch.cuda.stream(s_in):
                if ev_out[b] is not None:
                    s_in.wait_event(ev_out[b])
                d_sino[b][:n].copy_(h_in[s0:s1], non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(s_in)
            s_cmp.wait_event(ev_in)
            sino_k = d_sino[b][:n, ::K].contiguous()
            sparse_rec.reconstruct_stack_dev(sino_k, d_sparse[b][:n], VOL_CENTER, s_cmp.cuda_stream)
            for i in range(n):
                net.forward(d_sparse[b][i:i + 1], d_out[b][i:i + 1], s_cmp.cuda_stream)
                if s0 + i in keep:
                    d_sparse_keep[s0 + i] = d_sparse[b][i].clone()
            ev_done = torch.cuda.Event()
            ev_done.record(s_cmp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_done)
                h_out[s0:s1].copy_(d_out[b][:n], non_blocking=True)
                ev_out[b] = torch.cuda.Event()
                ev_out[b].record(s_out)
        torch.cuda.synchronize()

    stream_all()   # warm-up
    times = []
    for _ in range(max(1, args.e2e_steps)):
        t0 = time.perf_counter()
        stream_all()
        times.append(time.perf_counter() - t0)
    log(f"[volume] learned form: e2e call times {[round(t, 3) for t in times]} s")
    stream_all(keep={int(k) for k in picks})   # untimed: keep the 900-angle FBPs of the picks
    full_rec.close()
    sparse_rec.close()
    net.close()
    return S / float(np.median(times)), d_sparse_keep, t_train


def _volume_files(np_in, S, local, steps, check_slices):
    """The ct tool's loop over raw volume files (ctas_vol_raw_reconstruct):
    the S sinograms written to a raw float32 file in /dev/shm (or the temp
    directory), reconstructed file to file as float32 and as 16-bit samples
    (the tool's -i 16, per-slice range).  Wall clock around each call: file
    reads, both copies, the kernels and file writes.  The outputs are checked
    against the stack call's slices (float32, bit for bit) and the oracle's
    limit<T> of them (16-bit)."""
    import shutil
    from ctas_b200 import ct, volume
    import oracle as O
    need = np_in.nbytes + S * VOL_W * VOL_W * 6 + (1 << 30)
    base = None
    for d in ("/dev/shm", tempfile.gettempdir()):
        try:
            if shutil.disk_usage(d).free > need:
                base = d
                break
        except OSError:
            pass
    if base is None:
        return {"skipped": f"no directory with {need >> 30} GiB free"}
    work = tempfile.mkdtemp(prefix="ctas_vol_", dir=base)
    try:
        fin = os.path.join(work, "sinos.f32")
        np_in.tofile(fin)
        res = {"dir": base, "unit": "slices/s"}
        outs = {}
        for bpp in (0, 16):
            fout = os.path.join(work, f"rec_{bpp}.raw")
            rec = ct.CTrec((VOL_N, VOL_W), ct.Contrast.PHS, 180.0, ct.Filter("HAMMING"),
                           pad=VOL_PAD, no_writeback=True, device=local)
            volume.reconstruct_raw(rec, fin, S, fout, VOL_CENTER, bpp)   # warm-up
            times = []
            for _ in range(max(1, steps)):
                t0 = time.perf_counter()
                volume.reconstruct_raw(rec, fin, S, fout, VOL_CENTER, bpp)
                times.append(time.perf_counter() - t0)
            rec.close()
            log(f"[volume] file to file, bpp {bpp}: call times {[round(t, 3) for t in times]} s")
            res["float32" if bpp == 0 else "int16_samples"] = round(S / float(np.median(times)), 3)
            outs[bpp] = fout
        f32 = np.memmap(outs[0], np.float32, "r", shape=(S, VOL_W, VOL_W))
        u16 = np.memmap(outs[16], np.uint16, "r", shape=(S, VOL_W, VOL_W))
        ok = True
        for k, sl in check_slices.items():
            ok &= bool(np.array_equal(np.asarray(f32[k]).view(np.uint32), sl.view(np.uint32)))
            ok &= bool(np.array_equal(np.asarray(u16[k]), O.limit(sl, 16)))
        res["checked_slices"] = len(check_slices)
        res["identical_to_stack_and_oracle_limit"] = ok
        del f32, u16
        return res
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _volume_full_length(n, np_in, S, local, sampled32):
    """n slices (2048 = the full case, ~120 GB in, ~137 GB out) streamed through
    ctas_fbp_reconstruct_volume: the reader callback copies sinogram k % S of
    the pinned sample into the library's pinned ring, the writer callback keeps
    eight sampled slices; host memory cannot hold the whole volume in and out.
    The kept slices must equal those of the sample run bit for bit."""
    from ctas_b200 import ct, volume
    # eight slices spread over the whole run, each a repeat of a slice sampled
    # in the sample run
    reps = np.linspace(0, max(0, n // S - 1), len(sampled32)).astype(int)
    picks = {int(p) + S * int(m) for p, m in zip(sorted(sampled32), reps) if int(p) + S * int(m) < n}
    kept = {}

    def read(first, count, buf):
        for i in range(count):
            np.copyto(buf[i], np_in[(first + i) % S])

    def write(first, count, buf):
        for i in range(count):
            if first + i in picks:
                kept[first + i] = buf[i].copy()

    rec = ct.CTrec((VOL_N, VOL_W), ct.Contrast.PHS, 180.0, ct.Filter("HAMMING"), pad=VOL_PAD,
                   no_writeback=True, device=local)
    volume.reconstruct_volume(rec, min(n, 2 * S), VOL_CENTER, read, write)  # warm-up
    kept.clear()
    t0 = time.perf_counter()
    volume.reconstruct_volume(rec, n, VOL_CENTER, read, write)
    dt = time.perf_counter() - t0
    rec.close()
    same = all(np.array_equal(v.view(np.uint32), sampled32[k % S].view(np.uint32))
               for k, v in kept.items() if k % S in sampled32)
    checked = sum(1 for k in kept if k % S in sampled32)
    return {"slices": n, "value": round(n / dt, 3), "unit": "slices/s", "seconds": round(dt, 2),
            "input_gb": round(4 * n * VOL_N * VOL_W / 1e9, 1),
            "output_gb": round(4 * n * VOL_W * VOL_W / 1e9, 1),
            "call": "ctas_fbp_reconstruct_volume (reader/writer callbacks, pinned rings)",
            "sampled_slices_bit_identical_to_sample_run": bool(same), "checked": checked}


def run_volume(args, rank, world, local):
    """Large streamed volume, a bounded sample of it: S sinograms of 3600 x 4096
    (default 32 = 1.9 GB in, 2.1 GB out; the full case is 2048 of them) in
    pinned host memory, reconstructed through the host C-ABI stack call, which
    streams chunks through HBM with copy/compute overlap on three streams.
    Hamming, FFT 8192, centre +12.25, 40-ellipsoid phantom, Poisson 5e3.  Rank
    0 only (replicas would stream their own slices).
        value : slices/s end to end (host in, host out; the filtered sinograms
                are not copied back, as the ct tool discards them)
        fp16  : the same with FP16-stored filtered sinograms
        device: slices/s with a chunk resident in HBM (context)
        error : vs the FP64 oracle on sampled rows of 8 sampled slices
        file_to_file: raw volume files through ctas_vol_raw_reconstruct
        learned_every_4th_angle: 900-angle FBP + U-Net, streamed end to end"""
    if rank != 0:
        return
    import torch
    from ctas_b200 import ct
    from ctas_b200 import phantom as ph
    import oracle as O
    torch.cuda.set_device(local)
    S = args.slices if args.slices != SLICES else 32
    log(f"[volume] generating {S} sinograms of {VOL_N} x {VOL_W}")
    ell = ph.random_ellipsoids(SEED + 4, 40, VOL_W, S, rho=(0.05, 0.5))
    ell[:, 7] *= 4.0 / VOL_W
    h_in = torch.empty((S, VOL_N, VOL_W), dtype=torch.float32, pin_memory=True)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED + 4)
    for s0 in range(0, S, 4):
        s1 = min(S, s0 + 4)
        h_in[s0:s1] = _vol_sinos_dev(ell, range(s0, s1), g, SEED + 70_000).cpu()
    torch.cuda.synchronize()
    h_out = torch.empty((S, VOL_W, VOL_W), dtype=torch.float32, pin_memory=True)
    np_in, np_out = h_in.numpy(), h_out.numpy()

    def e2e(store):
        rec = ct.CTrec((VOL_N, VOL_W), ct.Contrast.PHS, 180.0, ct.Filter("HAMMING"),
                       pad=VOL_PAD, store=store, no_writeback=True, device=local)
        rec.reconstruct_stack(np_in, np_out, VOL_CENTER)   # warm-up: tile search, work sets
        times = []
        for _ in range(max(1, args.e2e_steps)):
            t0 = time.perf_counter()
            rec.reconstruct_stack(np_in, np_out, VOL_CENTER)
            times.append(time.perf_counter() - t0)
        rec.close()
        log(f"[volume] store {store}: e2e call times {[round(t, 3) for t in times]} s")
        return S / float(np.median(times))

    with ClockSampler(local) as clk:
        v32 = e2e(0)
    clocks = clk.summary()
    picks = np.linspace(0, S - 1, min(8, S)).astype(int)
    sampled32 = {int(k): np_out[k].copy() for k in picks}
    v16 = e2e(1)
    sampled16 = {int(k): np_out[k].copy() for k in picks}
    # device-resident chunk for context
    C = min(S, 16)
    d_in = h_in[:C].cuda()
    d_out = torch.empty((C, VOL_W, VOL_W), device="cuda")
    rec = ct.CTrec((VOL_N, VOL_W), ct.Contrast.PHS, 180.0, ct.Filter("HAMMING"), pad=VOL_PAD,
                   no_writeback=True, device=local)
    stream = torch.cuda.current_stream()
    rec.reconstruct_stack_dev(d_in, d_out, VOL_CENTER, stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(max(1, args.steps)):
        rec.reconstruct_stack_dev(d_in, d_out, VOL_CENTER, stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    vdev = C * max(1, args.steps) / (e0.elapsed_time(e1) * 1e-3)
    tile = rec.last_tile()
    rec.close()
    del d_in, d_out
    full_len = None
    if args.vol_full:
        full_len = _volume_full_length(args.vol_full, np_in, S, local, sampled32)
    files = _volume_files(np_in, S, local, args.e2e_steps,
                          {int(k): sampled32[int(k)] for k in picks[:2]})
    vlrn, sparse_keep, t_train = _volume_learned(args, h_in, h_out, S, local, picks)
    sampled_l = {int(k): np_out[k].copy() for k in picks}
    sampled_s = {k: v.cpu().numpy() for k, v in sparse_keep.items()}
    # error vs the FP64 oracle (full-angle) on 8 sampled slices x 6 sampled rows
    G64 = O.filter_window(6, 0.0, VOL_PAD, VOL_W, O.PHS, fp64=True)
    tab = O.angle_table(180.0, VOL_N)
    rows = np.linspace(400, VOL_W - 400, 6).astype(int)
    m = O.mask(VOL_W, VOL_CENTER)[rows]
    err = {"fp32": [], "fp16": [], "learned": [], "sparse": []}
    for k in picks:
        qd = O.prepare_sino(np_in[k], VOL_PAD, O.PHS, G64, fp64=True)
        ref = np.concatenate([O.bp_compat(qd, tab, VOL_CENTER, 1.0, rows=(int(r), int(r) + 1))
                              for r in rows])
        for name, got in (("fp32", sampled32[int(k)][rows]), ("fp16", sampled16[int(k)][rows]),
                          ("learned", sampled_l[int(k)][rows]),
                          ("sparse", sampled_s[int(k)][rows])):
            err[name].append(float(np.sqrt(np.mean((got[m] - ref[m]) ** 2)) /
                                   np.sqrt(np.mean(ref[m] ** 2))))
    # quality against the phantom (the FBP without physics is density / pi),
    # whole slices inside the reconstructed region
    msk = torch.from_numpy(O.mask(VOL_W, VOL_CENTER)).cuda()
    psnr = {"full_angle_fp32": [], "sparse_900_angles": [], "learned": []}
    for k in picks:
        truth = ((ph.image_dev(ph.ellipsoid_sections(ell, int(k) + 0.5), VOL_W, VOL_CENTER)
                  + _vol_texture(SEED + 70_000, int(k))[0])[msk] / np.pi).double()
        rng2 = float(truth.max() - truth.min()) ** 2
        for name, arr in (("full_angle_fp32", sampled32[int(k)]),
                          ("sparse_900_angles", sampled_s[int(k)]),
                          ("learned", sampled_l[int(k)])):
            d = torch.from_numpy(arr).cuda()[msk].double() - truth
            psnr[name].append(10 * np.log10(rng2 / float((d * d).mean())))
    psnr = {k: round(float(np.mean(v)), 2) for k, v in psnr.items()}
    line = {
        "metric": "slices/s", "value": round(v32, 3), "unit": "slices/s", "n_gpus": 1,
        "steps": args.e2e_steps, "warmup": 1, "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded 40-ellipsoid phantom, exact projections, plus a band-limited "
                "Gaussian-random-field texture per section (std 0.05 of the density scale, "
                "correlation 8 px, ray-marched projections); Poisson 5e3)",
        "config": {"workload": f"streamed volume sample: {S} x (3600 x 4096) float32 sinograms "
                               f"in pinned host memory -> 4096 x 4096 slices, Hamming, FFT "
                               f"8192, centre +12.25 (full case: 2048 sinograms, ~120 GB)",
                   "slices": S, "transfer": "H2D sinograms + D2H slices inside the timed "
                                            "region; filtered sinograms not copied back"},
        "e2e": {"value": round(v32, 3), "unit": "slices/s",
                "h2d_bytes_per_step": 4 * S * VOL_N * VOL_W,
                "d2h_bytes_per_step": 4 * S * VOL_W * VOL_W,
                "call": "ctas_fbp_reconstruct_stack (pinned host buffers)"},
        "fp16_store": {"value": round(v16, 3), "unit": "slices/s",
                       "rel_rmse_vs_fp64_max": max(err["fp16"])},
        "device_resident": {"value": round(vdev, 3), "unit": "slices/s", "chunk": C,
                            "bp_tile": tile},
        "error_vs_fp64": {"rel_rmse_max": max(err["fp32"]), "slices": len(picks),
                          "rows_per_slice": len(rows)},
        "file_to_file": files,
        "full_length_stream": full_len,
        "learned_every_4th_angle": {
            "value": round(vlrn, 3), "unit": "slices/s",
            "rel_rmse_vs_fp64_full_angle_max": max(err["learned"]),
            "rel_rmse_vs_fp64_full_angle_mean": float(np.mean(err["learned"])),
            "sparse_fbp_rel_rmse_vs_fp64_full_angle_mean": float(np.mean(err["sparse"])),
            "psnr_vs_phantom_db_mean": psnr,
            "training_s": round(t_train, 1), "train_steps": args.train_steps,
            "pipeline": "H2D sinograms, every 4th projection taken on the device, 900-angle "
                        "FBP, 4-level BF16 U-Net (tcgen05), D2H slices; three streams"},
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


LRN_W, LRN_N, LRN_K = 2048, 1800, 4
LRN_TEX_STD, LRN_TEX_CORR = 0.05, 8.0


def _ssim(a, b, rng):
    """Mean SSIM (11 x 11 Gaussian window, sigma 1.5, data range rng) of two
    (B, H, W) torch tensors."""
    import torch
    import torch.nn.functional as F
    g = torch.exp(-(torch.arange(11, device=a.device, dtype=torch.float32) - 5) ** 2 / 4.5)
    g = g / g.sum()
    k = (g[:, None] * g[None, :])[None, None]
    f = lambda t: F.conv2d(t[:, None], k)[:, 0]
    mu_a, mu_b = f(a), f(b)
    saa = f(a * a) - mu_a ** 2
    sbb = f(b * b) - mu_b ** 2
    sab = f(a * b) - mu_a * mu_b
    c1, c2 = (0.01 * rng) ** 2, (0.03 * rng) ** 2
    s = ((2 * mu_a * mu_b + c1) * (2 * sab + c2)) / ((mu_a ** 2 + mu_b ** 2 + c1) * (saa + sbb + c2))
    return float(s.mean())


def run_learned(args, rank, world, local):
    """Learned sparse-angle reconstruction (extension), the 2048 x 2048 case:
    phantoms of random ellipses (axes 20-480 px, density U(0.1, 1)) with exact
    projections plus a band-limited texture, 1800 x 2048, centre 0, RAMP;
    input = plain FBP of every 4th projection (450 angles), target = plain
    full-angle FBP.  The 4-level BF16 U-Net (32 base channels) is trained with
    Adam (lr 1e-3) on random 256 x 256 crops for --train-steps steps; the
    --train-phantoms training pairs are generated on the GPU while it trains
    (a pool of 128 pairs, 16 replaced at a time, so every phantom is used),
    then it is evaluated on --eval-phantoms held-out phantoms at 2048 x 2048.
    Rank 0 only.
        value: learned slices/s (450-angle FBP + U-Net inference, device-resident)
        plain: full-angle slices/s
        quality: PSNR / SSIM / RMSE of the sparse FBP and of the learned output
                 against the full-angle FBP (and against the phantom)"""
    if rank != 0:
        return
    import torch
    from ctas_b200 import ct, learned
    from ctas_b200 import phantom as ph
    torch.cuda.set_device(local)
    W, N, K = LRN_W, LRN_N, LRN_K
    n_train, n_eval = max(16, args.train_phantoms), max(1, args.eval_phantoms)
    if args.quick:  # U-Net forward passes on one 2048 x 2048 slice only (profiler runs)
        net = learned.UNet(seed=SEED, scale=1.0, device=local)
        x = torch.rand((1, W, W), device="cuda")
        y = torch.empty_like(x)
        stream = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        net.forward(x, y, stream.cuda_stream)
        e0.record(stream)
        for _ in range(max(1, args.steps)):
            net.forward(x, y, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / max(1, args.steps)
        flops = 2.0 * learned.UNet.macs_per_pixel() * W * W
        print(json.dumps({"quick": True, "unet_forward_ms": round(ms, 3),
                          "tflops": round(flops / (ms * 1e-3) / 1e12, 1)}), flush=True)
        net.close()
        return

    def phantoms(seed0, n):
        # (ellipses, texture seed): random ellipses plus a band-limited Gaussian
        # random field of standard deviation 0.05 (correlation length 8 px)
        return [(ph.random_ellipses(seed0 + i, 10, W, axes=(20.0, 480.0)), seed0 + 50_000 + i)
                for i in range(n)]

    def textures(items):
        return torch.cat([ph.grf_texture_dev(ts, W, std=LRN_TEX_STD, corr_px=LRN_TEX_CORR)
                          for _, ts in items])

    def pairs(items, chunk=16):
        full_rec = ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("RAMP"), device=local)
        sparse_rec = ct.CTrec((N // K, W), ct.Contrast.PHS, 180.0, ct.Filter("RAMP"),
                              device=local)
        xs, ys = [], []
        for c0 in range(0, len(items), chunk):
            e = np.stack([el for el, _ in items[c0:c0 + chunk]])
            sino = ph.sinogram_dev(e, N, W, center=0.0)
            ph.project_image_dev(textures(items[c0:c0 + chunk]), N, out=sino)
            S = sino.shape[0]
            full = torch.empty((S, W, W), device="cuda")
            sparse = torch.empty((S, W, W), device="cuda")
            full_rec.reconstruct_stack_dev(sino, full, 0.0)
            sparse_rec.reconstruct_stack_dev(sino[:, ::K].contiguous(), sparse, 0.0)
            xs.append(sparse)
            ys.append(full)
            del sino
        full_rec.close()
        sparse_rec.close()
        return torch.cat(xs), torch.cat(ys)

    pool = min(128, n_train)
    log(f"[learned] {n_train} training pairs at {W} x {W}, a pool of {pool} refreshed on the fly")
    t_gen = 0.0

    def gen(seed0, n):
        nonlocal t_gen
        torch.cuda.synchronize()
        t = time.perf_counter()
        x, y = pairs(phantoms(seed0, n))
        torch.cuda.synchronize()
        t_gen += time.perf_counter() - t
        return x, y

    xtr, ytr = gen(SEED + 100, pool)
    made = pool
    scale = float(1.0 / ytr.std())
    net = learned.UNet(seed=SEED, scale=scale, device=local)
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    Bc, C, R = 8, 256, 16
    # steps between pool refreshes of R pairs, so that all n_train are made
    nref = -(-(n_train - pool) // R) if n_train > pool else 0
    every = max(1, (args.train_steps - 1) // nref) if nref else 0
    losses = []
    t_train = 0.0
    slot = 0
    for step in range(args.train_steps):
        if every and step and step % every == 0 and made < n_train:
            r = min(R, n_train - made)
            xn, yn = gen(SEED + 100 + made, r)
            for k in range(r):
                xtr[(slot + k) % pool] = xn[k]
                ytr[(slot + k) % pool] = yn[k]
            slot = (slot + r) % pool
            made += r
            del xn, yn
        torch.cuda.synchronize()
        t = time.perf_counter()
        idx = torch.randint(0, pool, (Bc,), device="cuda", generator=g)
        oy = torch.randint(0, W - C + 1, (Bc,), device="cuda", generator=g)
        ox = torch.randint(0, W - C + 1, (Bc,), device="cuda", generator=g)
        ar = torch.arange(C, device="cuda")
        rows = (oy[:, None] + ar[None, :])[:, :, None]
        cols = (ox[:, None] + ar[None, :])[:, None, :]
        xb = xtr[idx[:, None, None], rows, cols].contiguous()
        yb = ytr[idx[:, None, None], rows, cols].contiguous()
        lr = 1e-3 if step < 0.8 * args.train_steps else 2e-4
        losses.append(net.train_step(xb, yb, lr))
        t_train += time.perf_counter() - t
    n_train = made
    del xtr, ytr
    torch.cuda.empty_cache()
    # held-out evaluation
    ev = phantoms(SEED + 10_000, n_eval)
    xev, yev = pairs(ev)
    outs = torch.empty_like(xev)
    for i in range(n_eval):
        net.forward(xev[i:i + 1], outs[i:i + 1])
    torch.cuda.synchronize()
    disc = torch.from_numpy(O_mask_disc(W)).cuda()
    # the reference's FBP without physics is density / pi (setPhysics multiplies
    # by pi / pixel size), so the phantom is compared in those units
    truth = (torch.stack([ph.image_dev(e, W) for e, _ in ev]) + textures(ev)) / np.float32(np.pi)
    fit = float((yev[:, disc] * truth[:, disc]).sum() / (truth[:, disc] ** 2).sum())

    def quality(a, ref):
        d = (a - ref)[:, disc]
        rng = float(ref[:, disc].max() - ref[:, disc].min())
        mse = float((d ** 2).mean())
        return {"psnr_db": round(10 * np.log10(rng ** 2 / mse), 3),
                "ssim": round(_ssim(a * disc, ref * disc, rng), 5),
                "rmse": float(np.sqrt(mse))}

    q = {"sparse_fbp_vs_full": quality(xev, yev), "learned_vs_full": quality(outs, yev),
         "full_vs_phantom": quality(yev, truth), "sparse_vs_phantom": quality(xev, truth),
         "learned_vs_phantom": quality(outs, truth),
         "phantom_units": "density / pi; least-squares scale of full FBP to it: %.4f" % fit}
    # throughput, device-resident, 8 slices per step
    S = 8
    e = np.stack([el for el, _ in ev[:S]])
    sino = ph.sinogram_dev(e, N, W, center=0.0)
    ph.project_image_dev(textures(ev[:S]), N, out=sino)
    sino_k = sino[:, ::K].contiguous()
    full_rec = ct.CTrec((N, W), ct.Contrast.PHS, 180.0, ct.Filter("RAMP"), device=local)
    sparse_rec = ct.CTrec((N // K, W), ct.Contrast.PHS, 180.0, ct.Filter("RAMP"), device=local)
    a = torch.empty((S, W, W), device="cuda")
    b = torch.empty((S, W, W), device="cuda")
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn, reps):
        for _ in range(2):
            fn()
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    ms_plain = timed(lambda: full_rec.reconstruct_stack_dev(sino, a, 0.0, stream.cuda_stream),
                     max(1, args.steps))

    def learned_step():
        sparse_rec.reconstruct_stack_dev(sino_k, a, 0.0, stream.cuda_stream)
        net.forward(a, b, stream.cuda_stream)   # the 8 slices as one batch

    ms_learned = timed(learned_step, max(1, args.steps))
    ms_net = timed(lambda: net.forward(a, b, stream.cuda_stream), max(1, args.steps))
    flops_net = 2.0 * learned.UNet.macs_per_pixel() * S * W * W
    full_rec.close()
    sparse_rec.close()
    net.close()
    line = {
        "metric": "slices/s", "value": round(S / (ms_learned * 1e-3), 3), "unit": "slices/s",
        "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "scaling": "none",
        "vs_baseline": None, "dtype": "bf16 network, f32 FBP",
        "data": "synthetic (seeded random-ellipse phantoms, exact projections, plus a band-limited "
                "Gaussian-random-field texture of std 0.05, correlation 8 px, projected by ray "
                "marching at 0.5 px with bilinear sampling)",
        "config": {"workload": f"learned sparse-angle FBP, {W} x {W}, every {K}th of {N} "
                               f"projections, 4-level U-Net 32 base channels",
                   "train_phantoms": n_train, "train_steps": args.train_steps,
                   "crop": C, "batch": Bc, "eval_phantoms": n_eval},
        "plain_full_angle": {"value": round(S / (ms_plain * 1e-3), 3), "unit": "slices/s"},
        "learned_vs_plain_speed": round(ms_plain / ms_learned, 3),
        "unet_forward": {"ms_per_slice": round(ms_net / S, 3),
                         "tflops": round(flops_net / (ms_net * 1e-3) / 1e12, 1)},
        "quality": q,
        "training": {"seconds": round(t_train, 1), "pair_generation_s": round(t_gen, 1),
                     "loss_first": losses[0], "loss_last_50": float(np.mean(losses[-50:]))},
    }
    print(json.dumps(line), flush=True)


def O_mask_disc(W):
    """Disc of radius W/2 - 2 about the centre: the reconstructed area of a
    centred scan, inside the reference's pixel mask."""
    hp = W // 2
    j, i = np.mgrid[0:W, 0:W]
    return ((j - hp) ** 2 + (i - hp) ** 2) < (hp - 2) ** 2


def run_reference(args, rank, world):
    """The reference's CPU path on this box's host cores, rank 0 only: its own
    CTrec (lct.cpp built in place, -O2 -ffast-math) through its InThread pool,
    one slice per thread, every projection of the slices (cpu_reference_lct;
    about 30 s a step on 16 cores); the as-shipped build (no -O, about ten
    times slower) is timed once beside it on a projection sample."""
    if rank != 0:
        return
    import oracle as O
    if not O.lct_available("o2"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref (the reference's lct.cpp built in place) "
                                         "was not built: reference sources absent"}))
        return
    from ctas_b200 import phantom as ph
    ell = ph.random_ellipsoids(SEED, N_ELLIPSOIDS, WIDTH, SLICES, rho=(0.05, 0.5))
    ell[:, 7] *= 4.0 / WIDTH
    p = ph.sinogram(ph.ellipsoid_sections(ell, SLICES / 2), N_ANGLES, WIDTH, center=CENTER,
                    dtype=np.float64)
    sino = ph.poisson_log(p, PHOTONS, SEED).astype(np.float32)
    threads = os.cpu_count() or 1
    # whole slices (every projection): a sample of every k-th projection keeps
    # each thread's sinogram in its caches and ran about 2x faster per
    # projection than the full 1800 x 2560 one, overstating the reference
    n_sub = N_ANGLES
    for _ in range(args.warmup):
        cpu_reference_lct(sino, threads, 3.0, n_sub=18)
    vals, secs, desc = [], [], ""
    for _ in range(args.steps):
        v, desc, _, sec = cpu_reference_lct(sino, threads, 3.0, n_sub=n_sub)
        vals.append(v)
        secs.append(sec)
    value = float(np.median(vals))
    shipped = None
    if O.lct_available("shipped"):
        vs, ds, _, _ = cpu_reference_lct(sino, threads, 6.0, variant="shipped")
        shipped = {"value": round(vs, 6), "unit": "slices/s", "sample": ds,
                   "note": "projection sample (whole slices would take minutes): the "
                           "sample's sinograms stay in cache, so this overstates the speed"}
    print(json.dumps({
        "impl": "reference", "metric": "slices/s", "value": round(value, 6), "unit": "slices/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * float(np.median(secs)), 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded ellipsoid phantom, exact projections, Poisson noise)",
        "config": {"workload": WORKLOAD, "slices_per_gpu": SLICES, "n_angles": N_ANGLES,
                   "width": WIDTH, "pad": PAD, "filter": "HANN", "center": CENTER,
                   "contrast": "PHS", "l2": "inputs 4.7 GB per step > 126 MB L2; no flush",
                   "parallelism": f"replicas x{world} (independent slices)"},
        "cpu_baseline": {"value": round(value, 6), "unit": "slices/s", "cores": threads,
                         "kind": "reference", "sample": desc},
        "shipped_build": shipped,
        "e2e": {"value": round(value, 6), "unit": "slices/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }), flush=True)


if __name__ == "__main__":
    main()
