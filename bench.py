"""Benchmark: 1080p SSIMULACRA2 pairs/s, batched vs plain, on B200.

Workload (the batched config of the reference's headline metric): 64 pairs of
1920x1080 NV12 (BT.709, limited range) frames, seeded synthetic content
(smooth luma gradient + band-limited noise; chroma noise; distorted by 8x8 DCT
quantisation with a step from {4, 8, 16, 32} per frame).  A step is one
submission of all 64 pairs (pyramid + fused tiles + finalize launches).

  value          pairs/s with the inputs resident in HBM (64 pairs x 6.2 MB of
                 NV12 = 398 MB per step, larger than the 126 MB L2, so no flush)
  plain          the drop-in path: one context, one compute + result read per
                 pair, pairs in sequence
  e2e            the public API with host buffers (s2_batch_submit_host):
                 every step uploads the 64 pairs from pinned host memory in
                 groups that overlap the compute of earlier groups, scores
                 them and reads the 64 results back; step k+1 is submitted
                 before step k's results are read (two submissions in flight)
  roofline       fused kernel: algorithmic bytes per launch (scale-0 NV12 of
                 both frames + the pyramid levels it reads) / its CUDA-event time
  cpu_baseline   the CPU SSIMULACRA2 path the reference validates against (the
                 oracle's restatement of examples/cpu.rs), all host cores,
                 bounded sample
  dssim          the sibling metric DSSIM (crates/dssim-cuda) on the same 64
                 pairs: both metrics from one prep pass, and DSSIM alone,
                 with the DSSIM passes' kernel time against their declared I/O

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
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
PKG = os.path.join(ROOT, "turbo-metrics_b200")
sys.path.insert(0, PKG)

N_PAIRS = 64
W, H = 1920, 1080
METRIC = "1080p SSIMULACRA2 pairs/s (batched, NV12 BT.709 limited, 64 pairs per step)"


def import_pkg():
    import importlib.util
    spec = importlib.util.spec_from_file_location("tmb", os.path.join(PKG, "__init__.py"),
                                                  submodule_search_locations=[PKG])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["tmb"] = mod
    spec.loader.exec_module(mod)
    return mod


def gen_pair(i):
    import synth
    (ry, ruv), (dy, duv) = synth.c1_pair(i, W, H)
    return ry, ruv, dy, duv


def replica_offset(rank, n_pairs):
    """First pair index of a replica: every rank scores its own n_pairs pairs."""
    return rank * n_pairs


def max_over_ranks(x, dist, device):
    """The slowest rank's time (the whole job ends with it); x itself on one rank."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, n_pairs, steps, ms):
    """Pairs per second of all replicas together over the max-over-ranks time."""
    return world * n_pairs * steps / (ms / 1e3)


def gen_pairs(n, offset=0):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        return pool.map(gen_pair, range(offset, offset + n))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 8:
                try:
                    rows.append((float(f[1]), float(f[2]), f[4:8]))
                except ValueError:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i in range(4) if r[i].lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def h2d_link_rate(nbytes, reps=5):
    """Host-to-device bandwidth of one plain copy of `nbytes` from pinned
    host memory (GB/s, CUDA events, best of `reps`): the ceiling of the e2e
    leg, whose every step uploads that many bytes."""
    import torch
    src = torch.empty(int(nbytes), dtype=torch.uint8).pin_memory()
    dst = torch.empty(int(nbytes), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    best = None
    for _ in range(reps + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dst.copy_(src, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del src, dst
    return nbytes / (best / 1e3) / 1e9


def with_issue_roofline(roofline, clk, peaks):
    """The fused pass is bound by instruction issue, not HBM: beside the HBM
    fraction, its warp instructions per launch (ncu smsp__inst_executed.sum of
    a capture, scaled to the bench launch by the pairs it processes) over the
    issue peak at the SM clock sampled during the timed region (148 SMs x 4
    schedulers x one warp instruction per cycle)."""
    winst = roofline.get("warp_instructions_per_launch")
    mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz")
    ms = roofline["kernel_ms"]["fused"]
    if winst and mhz and ms > 0:
        peak = 148 * 4 * mhz * 1e6
        achieved = winst / (ms / 1e3)
        roofline["issue"] = {"bound": "issue", "achieved": achieved / 1e9, "peak": peak / 1e9,
                             "unit": "G warp instructions/s", "frac": achieved / peak, "sm_mhz": mhz,
                             "source": "instructions from the ncu capture in profiles/, clock sampled"}
    return roofline


def serve_pool_candidate(args):
    import synth
    ref, i = args
    return synth.c4_pool_candidate(ref, i)


def c1_candidate(args):
    import synth
    ref, k = args
    return synth.nv12_candidate(ref, synth.c1_candidate_step(k))


def cached_reference_bench(tmb, ref, n_cands, steps, warmup, value, peak):
    """One C1 reference frame + n_cands distorted versions of it (8x8 DCT
    quantisation, steps spread over [2, 48]) per step, through the batch's
    cached reference (s2_batch_set_reference + submit_with_reference, the
    semantics of ssim2-gpu's Ssim2Batch): the reference's XYB pyramid and
    stays resident, so each candidate's prep converts one frame."""
    import multiprocessing as mp
    import torch
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        cands = pool.map(c1_candidate, [(ref, k) for k in range(n_cands)])
    dy = [torch.from_numpy(c[0]).cuda() for c in cands]
    duv = [torch.from_numpy(c[1]).cuda() for c in cands]
    b = tmb.Ssim2Batch(n_cands, n_cands * W * H)
    b.set_reference(torch.from_numpy(ref[0]).cuda(), "nv12", ref_uv=torch.from_numpy(ref[1]).cuda())
    stream = torch.cuda.current_stream()
    for _ in range(max(warmup, 3)):
        b.submit_with_reference(dy, "nv12", dis_uv=duv)
    res = b.results()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        b.submit_with_reference(dy, "nv12", dis_uv=duv)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    tmb.lib.s2_batch_set_profiling(b._h, 1)
    kt = (ctypes.c_float * 3)()
    acc = np.zeros(3)
    for _ in range(3):
        b.submit_with_reference(dy, "nv12", dis_uv=duv)
        tmb.lib.s2_batch_last_timings(b._h, kt)
        acc += np.array(kt[:])
    tmb.lib.s2_batch_set_profiling(b._h, 0)
    acc /= 3
    sn = sum_pixels()
    tile_bytes = n_cands * 2 * 12 * sn  # ref XYB, dis XYB (3 planes f32 each) read
    prep_bytes = n_cands * (1.5 * W * H + 12 * sn)  # NV12 of the candidate in, its XYB planes out
    b.close()
    rate = n_cands / (ms / 1e3)
    return {"workload": "1 x 1920x1080 NV12 reference (cached) + %d DCT-quantised candidates per step" % n_cands,
            "pairs_per_s": rate, "vs_value": rate / value, "ms_per_step": ms,
            "score_range": [float(min(r[0] for r in res)), float(max(r[0] for r in res))],
            "kernel_ms": {"prep": float(acc[0]), "tile": float(acc[1]), "finalize": float(acc[2])},
            "bytes_per_step": {"prep (NV12 in + candidate XYB out)": prep_bytes,
                               "tile (reference XYB + candidate XYB in)": tile_bytes},
            "tile_gbs": tile_bytes / (acc[1] / 1e3) / 1e9, "tile_frac": tile_bytes / (acc[1] / 1e3) / 1e9 / peak}


def c2_pair(i):
    import synth
    return synth.c2_pair(i)


def uneven_bench(tmb, n=256, steps=3):
    """Uneven-size batch: n sRGB8 pairs with width and height each uniform in
    [64, 2048], scored (a) as one submission -- one prep, one persistent tile
    launch over every (pair, scale, tile, channel), one finalize, the tile
    height autotuned -- and (b) as a chain of one-pair submissions, the way a
    per-size instance scores them one at a time."""
    import multiprocessing as mp
    import torch
    with mp.get_context("spawn").Pool(os.cpu_count() or 1) as pool:
        raw = pool.map(c2_pair, range(n))
    dev = [(torch.from_numpy(r).cuda(), torch.from_numpy(d).cuda()) for r, d in raw]
    descs = [tmb.PairDesc(r, d, "srgb8") for r, d in dev]
    px = sum(r.shape[0] * r.shape[1] for r, _ in raw)
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch = tmb.Ssim2Batch(n, px)
    for _ in range(2):
        batched = batch.compute_batch(descs)  # the first one also tunes the tile height
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        batch.submit(descs)
        batched = batch.results()
    ev1.record(stream)
    torch.cuda.synchronize()
    batched_ms = ev0.elapsed_time(ev1) / steps
    one = tmb.Ssim2Batch(1, max(r.shape[0] * r.shape[1] for r, _ in raw))
    chain = [one.compute_batch([d])[0] for d in descs]  # warm-up: graphs and tuning per size class
    torch.cuda.synchronize()
    ev0.record(stream)
    chain = [one.compute_batch([d])[0] for d in descs]
    ev1.record(stream)
    torch.cuda.synchronize()
    chain_ms = ev0.elapsed_time(ev1)
    worst = max(abs(a[0] - b[0]) for a, b in zip(batched, chain))
    assert worst < 1e-9, "batched and per-pair scores differ by %g" % worst
    batch.close()
    one.close()
    return {"pairs": n, "megapixels": px / 1e6, "sizes": "W, H uniform in [64, 2048], sRGB8 (C0 content)",
            "batched_ms": batched_ms, "batched_pairs_per_s": n / (batched_ms / 1e3),
            "per_pair_chain_ms": chain_ms, "per_pair_chain_pairs_per_s": n / (chain_ms / 1e3),
            "batched_vs_chain": chain_ms / batched_ms, "max_score_diff": worst}


def serving_bench(tmb, rates=(200, 1000, 5000), jobs_per_rate=10000, server_kw=None):
    """Serving workload: `jobs_per_rate` Poisson arrivals at each offered rate;
    job sizes continuous log-uniform between 128x128 and 3840x2160, 1..16
    candidates per job with DCT steps uniform in [2, 48]; 40 GB admission
    budget; latency = arrival -> all candidates scored.  Images are crops of a
    pregenerated 3840x2160 pool (one reference, 16 candidates whose steps are
    the midpoints of 16 bins of [2, 48]) at a per-job offset; a job's
    candidates are the pool candidates of its steps' bins.  They sit in pinned
    host memory and are passed with the pool's row pitch (no copies).  Jobs
    the server refuses (Busy: 128 unfinished jobs) are counted, not retried."""
    import multiprocessing as mp
    import synth
    import torch
    ref = synth.c4_pool_reference()
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        cands = pool.map(serve_pool_candidate, [(ref, i) for i in range(synth.C4_POOL_CANDS)])
    pinned = [torch.from_numpy(a).pin_memory() for a in [ref] + cands]
    pool_imgs = [t.numpy() for t in pinned]
    out = {"workload": "C4: %d Poisson jobs per rate, sizes log-uniform 128x128..3840x2160 (continuous), "
                       "1-16 candidates, DCT step U[2,48]" % jobs_per_rate,
           "pool": "crops of one 3840x2160 reference + %d candidates (DCT step bin midpoints), pinned host "
                   "memory" % synth.C4_POOL_CANDS}
    for rate in rates:
        jobs = synth.c4_jobs(jobs_per_rate, rate, seed_index=rate)
        crops = [synth.c4_job_crop(jb) for jb in jobs]
        kw = dict(hbm_budget=40 << 30)
        kw.update(server_kw or {})
        sv = tmb.Ssim2Server(**kw)
        # warm-up: a few jobs of assorted sizes
        for jb, (ox, oy, idx) in list(zip(jobs, crops))[:8]:
            w, h = jb["w"], jb["h"]
            sv.wait(sv.submit(pool_imgs[0][oy:oy + h, ox:ox + w], [pool_imgs[1 + idx[0]][oy:oy + h, ox:ox + w]]))
        sv.reset_stats()
        ids, pairs, rejected = [], 0, 0
        t0 = time.perf_counter()
        for jb, (ox, oy, idx) in zip(jobs, crops):
            w, h = jb["w"], jb["h"]
            dt = jb["t"] - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            try:
                ids.append(sv.submit(pool_imgs[0][oy:oy + h, ox:ox + w],
                                     [pool_imgs[1 + c][oy:oy + h, ox:ox + w] for c in idx]))
                pairs += jb["k"]
            except tmb.Busy:
                rejected += 1
        for i in ids:
            sv.wait(i, timeout_ms=600000)
        wall = time.perf_counter() - t0
        rep = sv.stats()
        sv.close()
        out["rate_%d" % rate] = {"offered_jobs_per_s": rate, "jobs": jobs_per_rate, "accepted_jobs": len(ids),
                                 "rejected_busy": rejected, "pairs": pairs,
                                 "pairs_per_s": pairs / wall, "p50_ms": rep["p50_ms"], "p99_ms": rep["p99_ms"],
                                 "max_ms": rep["max_ms"], "rounds": rep["rounds"], "wall_s": wall,
                                 "gpu_busy_s": rep["gpu_busy_s"], "worker_wait_s": rep["worker_wait_s"],
                                 "worker_upload_s": rep["worker_upload_s"],
                                 "worker_submit_s": rep["worker_submit_s"], "copy_busy_s": rep["copy_busy_s"],
                                 "upload_gb": rep["bytes_uploaded"] / 1e9}
    return out


def cpu_baseline(seconds=15.0, threads=None):
    """Oracle cpu32 mode (the CPU crate's arithmetic) on 1080p pairs, one pair per
    thread on all host cores, for about `seconds`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import synth
    from concurrent.futures import ThreadPoolExecutor
    threads = threads or os.cpu_count() or 1
    (ry, ruv), (dy, duv) = synth.c1_pair(0, W, H)
    rl, dl = oracle.nv12_to_linear(ry, ruv), oracle.nv12_to_linear(dy, duv)
    t0 = time.time()
    oracle.ssim2_linear(rl, dl, "cpu32")
    one = time.time() - t0
    n = max(threads, int(round(seconds / max(one, 1e-3) * threads / max(threads, 1))))
    n = max(threads, min(n, threads * 4))
    t0 = time.time()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda _: oracle.ssim2_linear(rl, dl, "cpu32"), range(n)))
    dt = time.time() - t0
    return {"value": n / dt, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": "%d x 1920x1080 pairs (NV12 converted to linear f32 outside the timed region), "
                      "oracle cpu32 = scalar C port of ssimulacra2-cuda/examples/cpu.rs (-O3 -march=x86-64-v3, "
                      "one pair per thread); single-thread %.2f s/pair" % (n, one)}


def zensim_bench(tmb, n_cands=16, reps=3):
    """zensim features (the other sibling metric of the shared pyramid row):
    one 1920x1080 sRGB8 reference cached with Zensim::set_reference, then
    n_cands distorted versions through compute_with_reference (each call
    returns its 228 features to the host, so the time includes the readback);
    and the oracle restatement on one host thread for one pair."""
    import synth
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ref, _ = synth.srgb_pair(W, H, synth.pair_seed(0, 5000))
    cands = [synth.srgb_pair(W, H, synth.pair_seed(0, 5000), 2.0 + 46.0 * k / n_cands)[1] for k in range(n_cands)]
    dref = torch.from_numpy(ref).cuda()
    dcs = [torch.from_numpy(c).cuda() for c in cands]
    z = tmb.Zensim(W, H)
    z.set_reference(dref)
    for c in dcs[:2]:
        z.compute_with_reference(c)
    torch.cuda.synchronize()
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        for c in dcs:
            z.compute_with_reference(c)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    z.close()
    t0 = time.perf_counter()
    oracle.zensim_features_srgb8(ref, cands[0])
    cpu_s = time.perf_counter() - t0
    return {"workload": "1 x 1920x1080 sRGB8 reference (cached) + %d candidates, 228 features each" % n_cands,
            "pairs_per_s": n_cands / best, "ms_per_pair": best / n_cands * 1e3,
            "cpu_baseline": {"value": 1.0 / cpu_s, "unit": "pairs/s", "cores": 1, "kind": "port",
                             "sample": "1 pair, oracle zensim_oracle.c (-O3 -march=x86-64-v3), one thread"},
            "score": "unavailable: the zensim weight table is not in the reference tree"}


def dssim_bench(tmb, descs, n_pairs, steps, warmup, s2_value, peak):
    """DSSIM, the sibling metric, on the same batch: both metrics from one
    prep pass, and DSSIM alone; device-timed like the main leg, with the
    DSSIM passes' kernel time and their declared I/O (Lab planes of both
    images read, SSIM map written by the tile pass and read by the MAD pass:
    32 bytes per pixel over the five levels)."""
    import torch
    b = tmb.Ssim2Batch(n_pairs, n_pairs * W * H)
    out = {}
    stream = torch.cuda.current_stream()
    for key, metrics in (("both", ("ssimulacra2", "dssim")), ("dssim_only", "dssim")):
        b.set_metrics(metrics)
        for _ in range(max(warmup, 3)):
            b.submit(descs)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            b.submit(descs)
        e1.record(stream)
        torch.cuda.synchronize()
        out[key + "_pairs_per_s"] = n_pairs * steps / (e0.elapsed_time(e1) / 1e3)
    res = b.results()
    out["dssim_mean"] = float(np.mean([r[5] for r in res]))
    tmb.lib.s2_batch_set_profiling(b._h, 1)
    kt = (ctypes.c_float * 3)()
    dms = ctypes.c_float()
    acc = np.zeros(4)
    for _ in range(3):
        b.submit(descs)
        tmb.lib.s2_batch_last_timings(b._h, kt)
        tmb.lib.s2_batch_last_dssim_ms(b._h, ctypes.byref(dms))
        acc += np.array(list(kt[:]) + [dms.value])
    tmb.lib.s2_batch_set_profiling(b._h, 0)
    acc /= 3
    npx = sum(max((W + (1 << s) - 1) >> s, 8) * max((H + (1 << s) - 1) >> s, 8) for s in range(5))
    ab = 32 * npx * n_pairs
    out["kernel_ms"] = {"prep_lab": float(acc[0]), "dssim_passes": float(acc[3])}
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "dssim_traffic.json")) as f:
            traffic = json.load(f).get("bytes_per_launch") * n_pairs // 64
    except (OSError, ValueError, TypeError):
        traffic = None
    out["roofline"] = {"bound": "hbm", "achieved": ab / (acc[3] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                       "frac": ab / (acc[3] / 1e3) / 1e9 / peak, "algorithmic_bytes_per_launch": ab,
                       "kernel": "dssim clamp+tile+mean+mad+final",
                       # ncu DRAM bytes of the tile launch (the passes' dominant kernel), per launch
                       "traffic_tile_kernel": traffic}
    out["both_vs_ssimulacra2_only"] = out["both_pairs_per_s"] / s2_value
    b.close()
    return out


def dssim_cpu_baseline(seconds=10.0, threads=None):
    """Oracle f32 mirror of dssim-cuda on 1080p pairs, one pair per thread on
    all host cores, for about `seconds` (bounded sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import synth
    from concurrent.futures import ThreadPoolExecutor
    threads = threads or os.cpu_count() or 1
    (ry, ruv), (dy, duv) = synth.c1_pair(0, W, H)
    rl, dl = oracle.nv12_to_linear(ry, ruv), oracle.nv12_to_linear(dy, duv)
    t0 = time.time()
    oracle.dssim_linear(rl, dl, "cuda32")
    one = time.time() - t0
    n = max(threads, min(threads * 4, int(seconds / max(one, 1e-3)) * threads // max(threads, 1)))
    t0 = time.time()
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda _: oracle.dssim_linear(rl, dl, "cuda32"), range(n)))
    dt = time.time() - t0
    return {"value": n / dt, "unit": "pairs/s", "cores": threads, "kind": "port",
            "sample": "%d x 1920x1080 pairs (NV12 converted to linear f32 outside the timed region), oracle f32 "
                      "mirror of dssim-cuda (dssim_oracle.c); single-thread %.2f s/pair" % (n, one)}


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU path (oracle port), all host threads."""
    if rank != 0:
        return
    steps, warm = args.steps, args.warmup
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    import synth
    from concurrent.futures import ThreadPoolExecutor
    threads = os.cpu_count() or 1
    (ry, ruv), (dy, duv) = synth.c1_pair(0, W, H)
    rl, dl = oracle.nv12_to_linear(ry, ruv), oracle.nv12_to_linear(dy, duv)
    per_step = threads  # one 1080p pair per host thread per step (bounded sample of the 64)
    with ThreadPoolExecutor(threads) as ex:
        for _ in range(warm):
            oracle.ssim2_linear(rl, dl, "cpu32")
        t0 = time.time()
        for _ in range(steps):
            list(ex.map(lambda _: oracle.ssim2_linear(rl, dl, "cpu32"), range(per_step)))
        dt = time.time() - t0
    v = steps * per_step / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "pairs/s", "n_gpus": world,
            "steps": steps, "warmup": warm, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "1920x1080 NV12 pairs, reference CPU path, %d pairs per step" % per_step},
            "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": threads, "kind": "port",
                             "sample": "%d steps x %d 1080p pairs; oracle cpu32 = scalar C port of "
                                       "ssimulacra2-cuda/examples/cpu.rs (-O3 -march=x86-64-v3, one pair per "
                                       "thread; the reference's Rust/NPP code cannot be built here)"
                                       % (steps, per_step)},
            "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def sum_pixels(w=W, h=H, scales=6):
    n = 0
    for _ in range(scales):
        n += w * h
        w, h = (w + 1) // 2, (h + 1) // 2
    return n


def algorithmic_bytes_fused(n_pairs, storage_bytes=4):
    """Declared I/O of one fused launch over n_pairs pairs: it reads the XYB
    planes of both frames at every scale (3 planes x storage bytes x sum of
    the scale sizes) and writes 6 doubles per (tile, channel) (negligible)."""
    return n_pairs * 2 * 3 * storage_bytes * sum_pixels()


def algorithmic_bytes_prep(n_pairs, storage_bytes=4):
    """prep: reads the NV12 frames (1.5 B/px each), writes the XYB planes."""
    return n_pairs * (2 * 1.5 * W * H + 2 * 3 * storage_bytes * sum_pixels())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-pairs", type=int, default=64)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-cached", action="store_true", help="skip the cached-reference leg")
    ap.add_argument("--serve-jobs", type=int, default=10000, help="jobs per offered rate of the serving leg")
    ap.add_argument("--no-uneven", action="store_true", help="skip the 256-pair uneven-size batch leg")
    ap.add_argument("--no-dssim", action="store_true", help="skip the DSSIM (sibling metric) leg")
    ap.add_argument("--no-zensim", action="store_true", help="skip the zensim features leg")
    ap.add_argument("--strip", type=int, default=0,
                    help="tile height of the main leg (16, 32, 64; 0 = autotuned, the default)")
    ap.add_argument("--pairs", type=int, default=N_PAIRS,
                    help="pairs per step (64 is the workload; smaller only for profiler captures)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    NP = args.pairs
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    tmb = import_pkg()

    pairs_np = gen_pairs(NP, offset=replica_offset(rank, NP))
    dev = []
    for ry, ruv, dy, duv in pairs_np:
        dev.append(tuple(torch.from_numpy(a).cuda() for a in (ry, ruv, dy, duv)))
    descs = [tmb.PairDesc(r, d, "nv12", ru, du) for r, ru, d, du in dev]
    stream = torch.cuda.current_stream()

    batch = tmb.Ssim2Batch(NP, NP * W * H, strip_rows=args.strip)
    batch.submit(descs)
    scores = [r[0] for r in batch.results()]
    lib = tmb.lib

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- batched, inputs resident ---------------------------------------
    for _ in range(args.warmup):
        batch.submit(descs)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for _ in range(args.steps):
            batch.submit(descs)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dist, "cuda")
    value = whole_job_rate(world, NP, args.steps, ms)

    # ---- fused-kernel roofline (CUDA events around each launch) ----------
    lib.s2_batch_set_profiling(batch._h, 1)
    kt = (ctypes.c_float * 3)()
    acc = np.zeros(3)
    nprof = max(3, min(args.steps, 10))
    for _ in range(nprof):
        batch.submit(descs)
        lib.s2_batch_last_timings(batch._h, kt)
        acc += np.array(kt[:])
    lib.s2_batch_set_profiling(batch._h, 0)
    acc /= nprof
    fused_ms = float(acc[1])
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    ab = algorithmic_bytes_fused(NP)
    achieved = ab / (fused_ms / 1e3) / 1e9
    traffic = None
    winst = None
    tpath = os.path.join(ROOT, "profiles", "fused_traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            # both were measured for the 64-pair launch; each pair's planes
            # are read once and its items are the same, so they scale with
            # the pairs of this run
            traffic = tj.get("bytes_per_launch")
            traffic = None if traffic is None else int(traffic * NP / N_PAIRS)
            winst = tj.get("warp_instructions_per_launch")
            winst = None if winst is None else int(winst * NP / N_PAIRS)
        except (OSError, ValueError):
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "fused_kernel<float>",
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                "kernel_ms": {"prep": float(acc[0]), "fused": fused_ms, "finalize": float(acc[2])},
                "fused_blocks_per_sm": int(lib.s2_fused_blocks_per_sm(0)),
                "algorithmic_bytes_per_launch": ab,
                "warp_instructions_per_launch": winst,
                "prep_gbs": algorithmic_bytes_prep(NP) / (float(acc[0]) / 1e3) / 1e9,
                # every pass's declared I/O over the sum of their times (prep: NV12 in + XYB
                # planes out; fused: XYB planes in; finalize: negligible)
                "all_passes": {"bytes": algorithmic_bytes_prep(NP) + ab, "ms": float(acc.sum()),
                               "gbs": (algorithmic_bytes_prep(NP) + ab) / (float(acc.sum()) / 1e3) / 1e9,
                               "frac": (algorithmic_bytes_prep(NP) + ab) / (float(acc.sum()) / 1e3) / 1e9 / peak}}

    # ---- plain: the drop-in, one pair at a time ----------------------------
    ctx = tmb.Ssimulacra2(W, H)
    npl = min(args.plain_pairs, NP)
    for i in range(3):
        r, ru, d, du = dev[i]
        ctx.compute_nv12(r, ru, d, du)
        ctx.get_score()
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    plain_scores = []
    for i in range(npl):
        r, ru, d, du = dev[i]
        ctx.compute_nv12(r, ru, d, du)
        plain_scores.append(ctx.get_score())
    plain_s = time.perf_counter() - t0
    plain = npl / plain_s
    assert np.allclose(plain_scores, scores[:npl], rtol=0, atol=1e-9), "plain vs batched scores differ"

    # ---- e2e: host buffers through the public API ---------------------------
    host = []
    for ry, ruv, dy, duv in pairs_np:
        host.append(tuple(torch.from_numpy(a).pin_memory() for a in (ry, ruv, dy, duv)))
    hdescs = [tmb.PairDesc(r, d, "nv12", ru, du) for r, ru, d, du in host]
    h2d = sum(a.numel() for h in host for a in h)
    d2h = NP * ctypes.sizeof(tmb.capi.Result)

    def e2e_run(steps):
        # s2_batch_submit_host: each step's planes are uploaded in groups that
        # overlap earlier groups' compute, and step k+1 is submitted before
        # step k's results are read, so its uploads overlap step k's tile pass
        res = None
        batch.submit_host(hdescs)
        for _ in range(steps - 1):
            batch.submit_host(hdescs)
            res = batch.results()
        res = batch.results()
        return res

    e2e_run(args.warmup)
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    res = e2e_run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    e2e = whole_job_rate(world, NP, args.steps, e2e_ms)
    assert np.allclose([r[0] for r in res], scores, atol=1e-9)
    link = h2d_link_rate(h2d)

    cached = None
    if not args.no_cached:
        cached = cached_reference_bench(tmb, pairs_np[0][:2], NP - 1, args.steps, args.warmup, value / world, peak)

    served = None
    if not args.no_serving:
        served = serving_bench(tmb, jobs_per_rate=args.serve_jobs)
    uneven = None
    if not args.no_uneven and world == 1:
        uneven = uneven_bench(tmb)

    dssim = None
    if not args.no_dssim:
        dssim = dssim_bench(tmb, descs, NP, args.steps, args.warmup, value / world, peak)

    zensim = None
    if not args.no_zensim and world == 1:
        zensim = zensim_bench(tmb)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline()
        if dssim is not None:
            dssim["cpu_baseline"] = dssim_cpu_baseline()

    if rank == 0:
        clk = clocks.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{NP} x 1920x1080 NV12 BT.709 limited pairs per step (batched, one submission)",
                       "pairs_per_step": NP, "storage": "f32", "blur": "fir (fused, shifted moments)",
                       "l2": "inputs 398 MB per step > 126 MB L2 (no flush)",
                       "parallelism": "replicas" if world > 1 else "single"},
            "plain_pairs_per_s": plain, "batched_vs_plain": value / world / plain,
            "e2e": {"value": e2e, "unit": "pairs/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    # the step's upload over the host link: its rate inside the
                    # e2e run against a plain pinned copy of the same bytes
                    "upload_gbs": h2d * e2e / NP / world / 1e9, "link_h2d_gbs": link,
                    "link_frac": (h2d * e2e / NP / world / 1e9) / link if link else None},
            "roofline": with_issue_roofline(roofline, clk, peaks),
            "gpu_launches": 3 * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
            "cached_reference": cached,
            "served": served,
            "uneven": uneven,
            "dssim": dssim,
            "zensim": zensim,
            "score_mean": float(np.mean(scores)),
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
