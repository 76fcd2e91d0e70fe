"""Benchmark: voxel-view updates/s of the tilt WBP hot path on B200.

Workload (one "step" = one pass of the hot path over one tilt series, inputs
resident in HBM): large plain WBP, 121 views at -60..+60 deg in 1 deg steps
with N(0, 0.1 deg) jitter, 2048x2048 float32 projections of a seeded phantom
(5000 ellipsoids + 200 beads, Poisson-like noise), reconstructed to
2048 x 2048 x 800 (13.4 GB resident).  The pass is R-weighting + cosine stretch
(filter stage) and back-projection.  It runs in two forms: FP16-stored
filtered projections (the headline `value`) and plain FP32 (`plain_fp32`);
both accumulate in FP32.  Inputs (2 GB projections, 2-4 GB staged rows, 13.4 GB
volume) are far larger than L2, so no flush is needed between steps.

`e2e` goes through the public C ABI with pinned host buffers: upload the
projections, reconstruct, download the whole volume, every step.

--impl reference: the CPU restatement of the reference's own algorithm (the
Rust reference cannot be built here) on a bounded sample of the same workload,
all host threads.

Multi-GPU (torchrun): one independent series per rank (weak scaling), no
data-path collective; the time is the max over ranks.
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
sys.path.insert(0, os.path.join(ROOT, "imod-rs_b200"))

METRIC = "voxel-view updates/s"
SM_COUNT = 148
SMEM_BYTES_PER_CLK = 128  # per SM


def c2_workload(jitter_seed=2):
    rng = np.random.default_rng(jitter_seed)
    ang = (np.arange(-60, 61, 1.0) + rng.normal(0.0, 0.1, 121)).astype(np.float32)
    return dict(name="large plain WBP: 121 views 2048x2048 -> 2048x2048x800, RADIAL 0.35/0.035",
                nx=2048, ny=2048, onx=2048, onz=800, angles=ang, radial=(0.35, 0.035), n_ell=5000,
                n_beads=200)


def c1_workload():
    """Config-1 shape, used for small profiling captures."""
    ang = np.arange(-60, 61, 2.0).astype(np.float32)
    return dict(name="plain WBP: 61 views 512x512 -> 512x512x200, RADIAL 0.35/0.035",
                nx=512, ny=512, onx=512, onz=200, angles=ang, radial=(0.35, 0.035), n_ell=300,
                n_beads=40)


def c2strip_workload():
    """The large WBP geometry (2048 wide, 121 jittered views, thickness 800) on 256 rows:
    the same per-slice work as the full series, with 2.3 GB on the device, for counter
    captures (their DRAM bytes scale to the full series by 2048 / 256 rows)."""
    w = c2_workload()
    w.update(name="large plain WBP strip: 121 views 2048x256 -> 2048x256x800, RADIAL 0.35/0.035", ny=256)
    return w


WORKLOADS = {"c2": c2_workload, "c1": c1_workload, "c2strip": c2strip_workload}


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def max_over_ranks(x, dist, world):
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, dist, world):
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def barrier(dist, world):
    if world > 1:
        dist.barrier()


def hbm_peak():
    """Measured HBM copy bandwidth of the B200s (GB/s) and where it came from."""
    for path in (os.path.join(ROOT, "MEASURED_PEAKS.json"),):
        try:
            with open(path) as f:
                v = json.load(f).get("hbm_gbs")
            if v:
                return float(v), "of measured (MEASURED_PEAKS.json hbm_gbs)"
        except (OSError, ValueError, AttributeError):
            pass
    return 6650.0, "of fallback (6.65 TB/s, MEASURED_PEAKS.json absent)"


def read_traffic(variant_name, storage="fp16"):
    """Per-launch DRAM bytes of the back-projection kernel at the large configuration,
    from the committed ncu summary of that tile variant (a 256-row strip of the same
    geometry, scaled by 2048 / 256 rows), or None when the timed variant has none.
    The summary lists one or more captures, each a `variant:` line followed by its
    `traffic_bytes_per_launch:` line."""
    path = os.path.join(ROOT, "profiles", f"bp_fast_c2strip_{storage}.md")
    traffic, cur = {}, None
    try:
        for line in open(path):
            key, _, val = line.partition(":")
            if key == "variant":
                cur = val.strip()
            elif key == "traffic_bytes_per_launch" and cur is not None:
                traffic[cur] = float(val.strip())
    except OSError:
        return None
    return traffic.get(variant_name)


def run_ours(args):
    import torch

    import tiltgpu as T

    world, rank, local, dist = dist_setup(args)
    torch.cuda.set_device(local)
    w = WORKLOADS[args.workload]()
    nx, ny, onx, onz, ang = w["nx"], w["ny"], w["onx"], w["onz"], w["angles"]
    nz = len(ang)
    n_proj = nz * ny * nx
    # seeded phantom projections, generated on this rank's device (independent series per rank)
    proj_d = torch.empty(n_proj, dtype=torch.float32, device=f"cuda:{local}")
    T.synth_projections(ang, nx=nx, ny=ny, vol_nx=onx, vol_nz=onz, n_ell=w["n_ell"], rmin=3, rmax=40,
                        dmin=0.2, dmax=1.0, n_beads=w["n_beads"], bead_r=5, bead_d=5.0, noise_kind=2,
                        noise=20000.0, seed=1000 + rank, device=local, out_device_ptr=proj_d.data_ptr())
    # a dedicated stream: the session runs on it and the CUDA events below time it
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    results = {}
    launches = 0
    forms = [f for f in ("fp32", "fp16") if f in args.forms.split(",")]
    for form in forms:
        s = T.Session(nx, ny, nz, ang, width=onx, thickness=onz, radial=w["radial"], log=True,
                      storage=form, device=local)
        s.set_stream(stream.cuda_stream)
        s.set_device(proj_d.data_ptr(), n_proj)
        for _ in range(args.warmup):
            s.reconstruct(sync=False)
        torch.cuda.synchronize()
        barrier(dist, world)
        clocks = ClockSampler(local)
        if form == "fp16":
            clocks.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        bp_ms = []
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            s.reconstruct(sync=False)
            info = s.last_run()
            launches += info["kernel_launches"] if form == "fp16" else 0
        e1.record(stream)
        torch.cuda.synchronize()
        # per-stage device times of the last step (events on the launching stream)
        s.synchronize()
        info = s.last_run()
        barrier(dist, world)
        ms = e0.elapsed_time(e1)
        ms_max = max_over_ranks(ms, dist, world)
        upd = info["updates"] * args.steps
        results[form] = dict(ms=ms_max, updates=sum_over_ranks(upd, dist, world), info=info,
                             kernel=s.kernel_info(),
                             clocks=clocks.stop() if form == "fp16" else None)
        # back-projection kernel alone, timed on the launching stream
        bp = []
        for _ in range(3):
            s.reconstruct(sync=True)
            bp.append(s.last_run()["ms_backproject"])
        results[form]["bp_ms"] = float(np.median(bp))
        results[form]["filter_ms"] = float(s.last_run()["ms_filter"])
        if form == "fp16":
            sess16 = s
        else:
            sess32 = s
    # the first slices of both forms, for the accuracy check against the oracle below
    acc_rows = 16
    first = {}
    for form, s_ in (("fp32", locals().get("sess32")), ("fp16", locals().get("sess16"))):
        if s_ is not None:
            s_.reconstruct(sync=True)
            first[form] = s_.download(0, min(acc_rows, s_.out_shape[0]))[0].copy()
    if "sess32" in locals():
        sess32.close()
    if args.profile:  # small-case profiling run: stage times only
        if rank == 0:
            print(json.dumps({f: {k: r[k] for k in ("ms", "bp_ms", "filter_ms")} | {"kernel": r["kernel"]}
                              for f, r in results.items()}), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    # ---- e2e through the public API with pinned host buffers.  Two sessions on
    # two streams take the steps in turn, so one step's download (PCIe D2H) runs
    # while the next step uploads (H2D) and computes; every step still copies its
    # projections in and its whole volume out.
    import ctypes as C
    L = T.lib()
    streams = [stream, torch.cuda.Stream(device=local)]
    sess = [sess16, T.Session(nx, ny, nz, ang, width=onx, thickness=onz, radial=w["radial"], log=True,
                              storage="fp16", device=local)]
    sess[1].set_stream(streams[1].cuda_stream)
    sess[1].set_variant(sess16.kernel_info()["variant"])
    host_in = torch.empty(n_proj, dtype=torch.float32, pin_memory=True)
    host_in.copy_(proj_d.cpu())
    out_shape = sess16.out_shape
    n_out = int(np.prod(out_shape))
    host_out = [torch.empty(n_out, dtype=torch.float32, pin_memory=True) for _ in range(2)]

    e2e_steps = max(2, min(args.steps, 8))
    for i in range(2):  # warm both sessions (tuning, graphs)
        T.check(L.tg_upload_projections(sess[i].h, C.c_void_p(host_in.data_ptr()), n_proj))
        T.check(L.tg_reconstruct(sess[i].h))
        T.check(L.tg_synchronize(sess[i].h))
    torch.cuda.synchronize()
    barrier(dist, world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev_end = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev0.record(streams[0])
    streams[1].wait_event(ev0)
    for i in range(e2e_steps):
        s_, o_ = sess[i % 2], host_out[i % 2]
        T.check(L.tg_upload_projections(s_.h, C.c_void_p(host_in.data_ptr()), n_proj))
        T.check(L.tg_reconstruct(s_.h))
        T.check(L.tg_download_slices_async(s_.h, 0, out_shape[0], C.c_void_p(o_.data_ptr())))
    for k in range(2):
        ev_end[k].record(streams[k])
    st = T.Stats()
    for s_ in sess:
        T.check(L.tg_synchronize(s_.h))
        T.check(L.tg_get_stats(s_.h, C.byref(st)))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(max(ev0.elapsed_time(e) for e in ev_end) * 1e-3, dist, world)
    e2e_upd = sum_over_ranks(sess16.last_run()["updates"] * e2e_steps, dist, world)
    for s_ in sess:
        s_.close()
    del host_in, host_out

    r16, r32 = results["fp16"], results["fp32"]
    value = r16["updates"] / (r16["ms"] * 1e-3)
    plain = r32["updates"] / (r32["ms"] * 1e-3)
    clk = r16["clocks"] or {}
    sm_mhz = clk.get("sm_mhz") or 1965.0
    # roofline of the dominant kernel (back-projection): shared-memory bytes per update
    # (4 B FP16 pair, 8 B FP32 pair) against 148 SMs x 128 B/clk x measured SM clock
    upd_pass = r16["info"]["updates"]
    bp_s = r16["bp_ms"] * 1e-3
    ach = upd_pass * 4.0 / bp_s / 1e9
    peak = SM_COUNT * SMEM_BYTES_PER_CLK * sm_mhz * 1e6 / 1e9
    traffic = read_traffic(r16["kernel"]["variant_name"])
    line = {
        "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r16["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "storage": "fp16",
        "data": "synthetic (seeded ellipsoid+bead phantom, Poisson noise, --log)",
        "config": {"workload": w["name"],
                   "views": nz, "proj": [nx, ny], "volume": [onx, ny, onz],
                   "l2": "inputs larger than L2 (no flush needed)", "parallelism": f"replicas{world}",
                   "bp_kernel": r16["kernel"]["variant_name"]},
        "plain_fp32": {"value": plain, "ms_per_step": r32["ms"] / args.steps,
                       "bp_ms": r32["bp_ms"], "filter_ms": r32["filter_ms"],
                       "bp_kernel": r32["kernel"]["variant_name"],
                       "roofline_frac": upd_pass * 8.0 / (r32["bp_ms"] * 1e-3) / 1e9 / peak},
        "fp16_over_fp32": value / plain,
        "stage_ms": {"filter": r16["filter_ms"], "backproject": r16["bp_ms"]},
        "roofline": {"bound": "smem", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": traffic,
                     "note": "shared-memory bytes of the back-projection kernel (4 B/update FP16 pair); "
                             "peak = 148 SMs x 128 B/clk x median SM clock sampled in the run; traffic = "
                             "DRAM bytes per launch of this tile variant from profiles/bp_fast_c2strip_fp16.md "
                             "(ncu on a 256-row strip of the same geometry, x 2048/256), null if untuned"},
        "roofline_hbm": {"bound": "hbm", "achieved": (4.0 * nz * nx * ny + 4.0 * onx * onz * ny) / bp_s / 1e9,
                         "peak": hbm_peak()[0], "unit": "GB/s",
                         "note": "back-projection kernel: FP16 staged rows (4 B per sample: value and "
                                 "difference) read + volume written; "
                                 + hbm_peak()[1]},
        "e2e": {"value": e2e_upd / e2e_s, "unit": "updates/s", "h2d_bytes_per_step": n_proj * 4,
                "d2h_bytes_per_step": int(np.prod(out_shape)) * 4 + 12},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"], ref_rows = cpu_baseline(args, w, proj_d, nslices=acc_rows, want_rows=True)
        # error of both forms on those slices against the oracle's f32 restatement of the reference
        # and against the oracle's FP64 data path with the reference's f32 geometry (ref64g),
        # the bound of the FP16 form (rel-L2 <= 2e-3)
        ref64 = oracle_rows64(w, proj_d, acc_rows)
        line["accuracy"] = {}
        for form, got in first.items():
            for name, ref in (("ref32", ref_rows), ("ref64g", ref64)):
                d = got.astype(np.float64) - ref.astype(np.float64)
                line["accuracy"][f"{form}_vs_{name}"] = {
                    "rel_l2": float(np.linalg.norm(d) / np.linalg.norm(ref.astype(np.float64))),
                    "max_abs": float(np.abs(d).max()), "ref_max_abs": float(np.abs(ref).max()),
                    "slices": acc_rows}
    if rank == 0 and world == 1 and args.workload == "c2" and not args.no_serving:
        # the metric's latency half and the target comparison: served FP16 against
        # serial plain FP32, end to end (host copies included), on the same series
        del proj_d
        torch.cuda.empty_cache()
        keys = ("workload", "jobs", "done", "failed", "failures", "latency_ms", "value",
                "device_busy_updates_per_s", "serial_plain_fp32", "ratio_vs_serial_plain_fp32")
        try:
            sv, pool = serve_stream(20.0, args.serve_seconds, 0.05, 150.0, 16, n_large=1)
            line["serving"] = {k: sv[k] for k in keys} | {"unit": "updates/s"}
            sat, _ = serve_stream(40.0, args.saturated_seconds, 0.05, 150.0, 16, n_large=1, pool=pool, seed=21)
            line["serving_saturated"] = {k: sat[k] for k in keys} | {"unit": "updates/s"}
            del pool
            line["c4_end_to_end"] = c4_at_once()
        except Exception as exc:  # the throughput line above stands on its own
            line["serving_error"] = repr(exc)[:200]
        try:
            line["c3_sirt"] = c3_summary()
        except Exception as exc:
            line["c3_error"] = repr(exc)[:200]
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline(args, w, proj_d=None, nslices=16, want_rows=False):
    """The oracle port (ref32, all host threads) on slices [0, nslices) of the workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nx, ny, onx, onz, ang = w["nx"], w["ny"], w["onx"], w["onz"], w["angles"]
    nz = len(ang)
    if proj_d is not None:
        proj = proj_d.cpu().numpy().reshape(nz, ny, nx)
    else:
        proj = seeded_rows(nz, ny, nx, nslices)
    p = O.Params(nx, ny, nz, ang, width=onx, thickness=onz, radial=w["radial"], log=True)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    rows = O.wbp_rows(p, proj, 0, nslices, nthreads=cores)
    dt = time.perf_counter() - t0
    upd = float(onx) * onz * nslices * nz
    res = {"value": upd / dt, "unit": "updates/s", "cores": cores, "kind": "port",
           "sample": f"slices 0..{nslices} of the workload (filter of their rows + stretch + WBP), "
                     f"{upd:.3g} updates in {dt:.2f} s"}
    return (res, rows) if want_rows else res


def oracle_rows64(w, proj_d, nslices):
    """ref64g (FP64 data path, the reference's f32 sampling geometry) of slices [0, nslices)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    nx, ny, onx, onz, ang = w["nx"], w["ny"], w["onx"], w["onz"], w["angles"]
    nz = len(ang)
    proj = proj_d.cpu().numpy().reshape(nz, ny, nx)
    p = O.Params(nx, ny, nz, ang, width=onx, thickness=onz, radial=w["radial"], log=True)
    return O.wbp_rows(p, proj, 0, nslices, nthreads=os.cpu_count() or 1, precision="64g")


def seeded_rows(nz, ny, nx, nrows, seed=5):
    """Seeded Poisson-like counts for the rows a bounded CPU sample reads (timing is data-independent)."""
    rng = np.random.default_rng(seed)
    proj = np.full((nz, ny, nx), 20000.0, np.float32)
    proj[:, :nrows, :] = rng.poisson(20000.0 * np.exp(-rng.random((nz, nrows, nx)))).astype(np.float32)
    return proj


def run_reference(args):
    world, rank, local, dist = dist_setup(args)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    w = c2_workload()
    nx, ny, onx, onz, ang = w["nx"], w["ny"], w["onx"], w["onz"], w["angles"]
    nz = len(ang)
    cores = os.cpu_count() or 1
    # the oracle parallelises over slices (as the reference's rayon loop over Y does):
    # two slices per host thread keep every core busy
    nsl = max(8, 2 * cores)
    proj = seeded_rows(nz, ny, nx, nsl)
    p = O.Params(nx, ny, nz, ang, width=onx, thickness=onz, radial=w["radial"], log=True)
    for _ in range(args.warmup):
        O.wbp_rows(p, proj, 0, nsl, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.wbp_rows(p, proj, 0, nsl, nthreads=cores)
    dt = time.perf_counter() - t0
    upd = float(onx) * onz * nsl * nz * args.steps
    v = upd / dt
    line = {"metric": METRIC, "value": v, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded counts)",
            "impl": "reference",
            "config": {"workload": "large plain WBP: 121 views 2048x2048 -> 2048x2048x800, RADIAL 0.35/0.035",
                       "views": nz, "proj": [nx, ny], "volume": [onx, ny, onz], "parallelism": "host threads"},
            "cpu_baseline": {"value": v, "unit": "updates/s", "cores": cores, "kind": "port",
                             "sample": f"each step: slices 0..{nsl} (filter of their rows, stretch, WBP)"},
            "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def c4_jobs(n=64, seed=4):
    """Batched uneven series: width in {256,384,512,768,1024} (square projections),
    views U{41..121}, ranges +-U(50,70) deg with uneven steps, thickness U{100..500},
    WBP:SIRT(10) = 3:1, each with its own seeded phantom and noise level."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        w = int(rng.choice([256, 384, 512, 768, 1024]))
        nv = int(rng.integers(41, 122))
        rmax = float(rng.uniform(50, 70))
        steps = rng.uniform(0.5, 1.5, nv - 1)
        steps = steps / steps.sum() * 2 * rmax
        ang = (-rmax + np.concatenate([[0.0], np.cumsum(steps)])).astype(np.float32)
        thick = int(rng.integers(100, 501))
        jobs.append(dict(w=w, nv=nv, ang=ang, thick=thick, sirt=10 if i % 4 == 3 else 0,
                         seed=1000 + i, noise=float(rng.uniform(0.2, 0.8))))
    return jobs


def job_updates(j):
    return float(j["w"]) * j["w"] * j["thick"] * len(j["ang"]) * (1 + 2 * j["sirt"])


def synth_job(T, torch, j, device_only=False):
    """Seeded ellipsoid phantom projections of one job (device tensor, or pinned host)."""
    ne = max(10, int(300 * (j["w"] / 512) ** 2 * j["thick"] / 200))
    d = torch.empty((len(j["ang"]), j["w"], j["w"]), dtype=torch.float32, device="cuda")
    T.synth_projections(j["ang"], nx=j["w"], ny=j["w"], vol_nz=j["thick"], n_ell=ne,
                        n_beads=max(4, ne // 8), noise_kind=1, noise=j.get("noise", 0.5),
                        seed=j["seed"], out_device_ptr=d.data_ptr())
    if device_only:
        return d
    h = torch.empty(d.shape, dtype=torch.float32, pin_memory=True)
    h.copy_(d)
    del d
    return h


def run_c3(args):
    """SIRT with x-axis tilt: 61 views at -60..+60 deg in 2 deg steps, 1024x1024, x-tilt
    1.5 deg in every view, Poisson counts (base 20000) with --log, phantom 1024x1024x400;
    WBP start then --sirt iterations (one CUDA graph per iteration).  Forms: FP32,
    FP16 and BF16 staging of the filtered projections and residuals, all accumulating
    in FP32."""
    import torch

    import tiltgpu as T
    torch.cuda.set_device(0)
    nx = ny = 1024
    onz = 400
    ang = np.arange(-60, 61, 2.0).astype(np.float32)
    xt = np.full(len(ang), args.xtilt, np.float32)
    n_proj = len(ang) * ny * nx
    proj_d = torch.empty(n_proj, dtype=torch.float32, device="cuda")
    T.synth_projections(ang, nx=nx, ny=ny, vol_nz=onz, n_ell=300, rmin=3, rmax=40, dmin=0.2, dmax=1.0,
                        n_beads=40, bead_r=5, bead_d=5.0, noise_kind=2, noise=20000.0, xtilt_deg=args.xtilt,
                        seed=3, out_device_ptr=proj_d.data_ptr())
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    res, vols = {}, {}
    forms = [f for f in ("fp32", "fp16", "bf16") if f in (args.forms or "fp32,fp16,bf16").split(",")]
    for form in forms:
        s = T.Session(nx, ny, len(ang), ang, thickness=onz, radial=(0.35, 0.035), log=True, xtilt=xt,
                      sirt=args.sirt, sirt_relax=args.sirt_relax, storage=form)
        s.set_stream(stream.cuda_stream)
        s.set_device(proj_d.data_ptr(), n_proj)
        for _ in range(args.warmup if not args.profile else 1):
            s.reconstruct(sync=False)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            s.reconstruct(sync=False)
        e1.record(stream)
        torch.cuda.synchronize()
        s.synchronize()
        info = s.last_run()
        ms = e0.elapsed_time(e1) / args.steps
        res[form] = {"value": info["updates"] / (ms * 1e-3), "ms_per_step": ms,
                     "stage_ms": {k: info[k] for k in ("ms_filter", "ms_backproject", "ms_reproject")},
                     "updates_per_step": info["updates"], "kernel": s.kernel_info()["variant_name"]}
        if not args.profile:
            vol, st = s.download()
            vols[form] = vol
            fin = np.isfinite(vol)
            res[form]["max_abs"] = float(np.abs(vol[fin]).max()) if fin.any() else None
            res[form]["nonfinite_voxels"] = int((~fin).sum())
        s.close()
    line = {"metric": METRIC, "unit": "updates/s", "n_gpus": 1, "workload":
            f"c3: SIRT {args.sirt} iterations, x-tilt {args.xtilt} deg, 61 views 1024x1024 -> 1024x1024x400, --log",
            "forms": res, "steps": args.steps, "data": "synthetic seeded phantom, Poisson counts, resident in HBM"}
    if "fp32" in vols:
        a = vols["fp32"].astype(np.float64)
        for f in ("fp16", "bf16"):
            if f in vols:
                b = vols[f].astype(np.float64)
                e = float(np.linalg.norm(a - b) / np.linalg.norm(a))
                line[f + "_rel_l2_vs_fp32"] = e if np.isfinite(e) else None  # FP16 overflows once SIRT diverges
    line["sirt_relax"] = args.sirt_relax
    print(json.dumps(line), flush=True)


def c3_summary(sirt=20, xtilt=1.5, relax=0.3, steps=2):
    """The SIRT configuration in all three staging forms, inputs resident (each
    iteration one CUDA graph): seconds per reconstruction and updates/s.  Relaxation
    0.3: at the reference's default 1.0 its un-normalised update diverges on this
    thick phantom, and the FP16 form then stops with TG_ERR_RANGE."""
    import torch

    import tiltgpu as T
    nx = ny = 1024
    onz = 400
    ang = np.arange(-60, 61, 2.0).astype(np.float32)
    xt = np.full(len(ang), xtilt, np.float32)
    n_proj = len(ang) * ny * nx
    proj_d = torch.empty(n_proj, dtype=torch.float32, device="cuda")
    T.synth_projections(ang, nx=nx, ny=ny, vol_nz=onz, n_ell=300, rmin=3, rmax=40, dmin=0.2, dmax=1.0,
                        n_beads=40, bead_r=5, bead_d=5.0, noise_kind=2, noise=20000.0, xtilt_deg=xtilt,
                        seed=3, out_device_ptr=proj_d.data_ptr())
    stream = torch.cuda.Stream()
    out = {"workload": f"c3: SIRT {sirt} iterations (relax {relax}) from the WBP start, x-tilt {xtilt} deg in "
                       "every view, 61 views 1024x1024 -> 1024x1024x400, Poisson counts with --log",
           "unit": "updates/s"}
    for form in ("fp32", "fp16", "bf16"):
        s = T.Session(nx, ny, len(ang), ang, thickness=onz, radial=(0.35, 0.035), log=True, xtilt=xt,
                      sirt=sirt, sirt_relax=relax, storage=form)
        s.set_stream(stream.cuda_stream)
        s.set_device(proj_d.data_ptr(), n_proj)
        try:
            s.reconstruct()  # tuning, graph capture
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                s.reconstruct(sync=False)
            e1.record(stream)
            s.synchronize()
            ms = e0.elapsed_time(e1) / steps
            info = s.last_run()
            out[form] = {"value": info["updates"] / (ms * 1e-3), "s_per_reconstruction": ms * 1e-3,
                         "ms_per_iteration": (ms - info["ms_filter"] - info["ms_backproject"]) / sirt}
        except T.TiltGpuError as exc:  # e.g. FP16 staging range exceeded by a diverging run
            out[form] = {"status": exc.code, "error": str(exc)[:160]}
        finally:
            s.close()
    return out


def run_c4(args):
    """64 uneven series: one persistent launch per round (FP16 staging, FP32
    accumulation) against the plain FP32 form (one series at a time)."""
    import torch

    import tiltgpu as T
    torch.cuda.set_device(0)
    jobs = c4_jobs()
    projs = [synth_job(T, torch, j, device_only=True) for j in jobs]
    upd = sum(job_updates(j) for j in jobs)

    def sessions(storage):
        out = []
        for j, d in zip(jobs, projs):
            s = T.Session(j["w"], j["w"], len(j["ang"]), j["ang"], **job_kw(j, storage))
            s.set_device(d.data_ptr(), d.numel())
            out.append(s)
        return out

    res = {}
    ss = sessions("fp32")
    for s in ss:  # tunes every shape once
        s.reconstruct()
    times = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s in ss:
            s.reconstruct(sync=True)
        times.append(time.perf_counter() - t0)
    res["plain_fp32"] = upd / min(times)
    for s in ss:
        s.close()
    for storage in ("fp16", "fp32"):
        ss = sessions(storage)
        b = T.Batch()
        for s in ss:
            b.add(s)
        b.reconstruct()
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            b.reconstruct()
            times.append(time.perf_counter() - t0)
        res["batched_" + storage] = upd / min(times)
        if args.profile:  # per-kernel device time of one batched run (CUPTI through torch.profiler)
            from torch.profiler import ProfilerActivity, profile
            with profile(activities=[ProfilerActivity.CUDA]) as prof:
                b.reconstruct()
            res["kernels_ms_" + storage] = {e.key[:60]: round(e.device_time_total / 1000.0, 2)
                                            for e in prof.key_averages() if e.device_time_total > 0}
        b.close()
        for s in ss:
            s.close()
    line = {"metric": METRIC, "value": res["batched_fp16"], "unit": "updates/s", "n_gpus": 1,
            "workload": "c4: 64 uneven series, WBP:SIRT(10) 3:1, one persistent launch per round",
            "plain_fp32": res["plain_fp32"], "batched_fp32": res["batched_fp32"],
            "batched_fp16_over_plain_fp32": res["batched_fp16"] / res["plain_fp32"],
            "updates_per_step": upd, "steps": args.steps, "timing": "best of steps, wall clock with sync",
            **{k: v for k, v in res.items() if k.startswith("kernels_ms_")},
            "data": "synthetic seeded phantoms, projections resident in HBM"}
    print(json.dumps(line), flush=True)


def make_pool(T, torch, jobs):
    """Seeded projections of each job in pinned host memory, every shape tuned in both
    forms (FP16 staging, plain FP32) outside any timed region."""
    t0 = time.perf_counter()
    pool = [(j, synth_job(T, torch, j)) for j in jobs]
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    for j, h in pool:
        for storage in ("fp16", "fp32"):
            with T.Session(j["w"], j["w"], len(j["ang"]), j["ang"], **job_kw(j, storage, sirt=0)) as s:
                s.upload(h.numpy())
                s.reconstruct()
    torch.cuda.empty_cache()
    print(f"# pool of {len(pool)} seeded series ready in {time.perf_counter() - t0:.1f}s", file=sys.stderr,
          flush=True)
    return pool


# SIRT relaxation of the batched and served series: at the reference's default 1.0 its
# un-normalised update diverges on the thicker series, and the FP16 staging form then
# stops with TG_ERR_RANGE instead of producing infinities
C4_RELAX = 0.3


def job_kw(j, storage, sirt=None):
    return dict(thickness=j["thick"], sirt=j["sirt"] if sirt is None else sirt, radial=(0.35, 0.035),
                storage=storage, sirt_relax=C4_RELAX)


class OutRings:
    """Pinned host output buffers: every result is copied out in full; contents are not
    checked here (jobs that share a ring slot overwrite each other's bytes)."""

    def __init__(self, torch, pool, n=4):
        small = [j["w"] * j["w"] * j["thick"] for j, _ in pool if j["w"] < 2048]
        large = [j["w"] * j["w"] * j["thick"] for j, _ in pool if j["w"] >= 2048]
        self.small = [torch.empty(max(small or [1]), dtype=torch.float32, pin_memory=True) for _ in range(n)]
        self.large = torch.empty(max(large), dtype=torch.float32, pin_memory=True) if large else None

    def out(self, i, j):
        n = j["w"] * j["w"] * j["thick"]
        buf = self.large if j["w"] >= 2048 else self.small[i % len(self.small)]
        return buf[:n].numpy().reshape(j["w"], j["thick"], j["w"])


def served_run(T, pool, arrivals, budget_gb, rings):
    """Submit pool[k] at each arrival time (seconds from the start) to one tg_server
    (FP16 staging, continuous batching, HBM admission budget); wait for all."""
    sampler = ClockSampler(0)
    sv = T.Server(device=0, budget_bytes=int(budget_gb * 1e9), max_active=64)
    ids = []
    sampler.start()
    start = time.perf_counter()
    for i, (ta, k) in enumerate(arrivals):
        now = time.perf_counter() - start
        if ta > now:
            time.sleep(ta - now)
        j, h = pool[k]
        ids.append(sv.submit(h.numpy(), j["ang"], out=rings.out(i, j), tag=k, **job_kw(j, "fp16")))
    results = [sv.wait(jid) for jid in ids]
    wall = time.perf_counter() - start
    clocks = sampler.stop()
    info = sv.info()
    sv.close()
    done = [r for r in results if r["state"] == "done"]
    lat = np.array([r["done_ms"] - r["submit_ms"] for r in done]) if done else np.zeros(1)
    span_ms = (max(r["done_ms"] for r in done) - min(r["submit_ms"] for r in done)) if done else 1.0
    upd = sum(r["updates"] for r in done)
    return {"value": upd / (span_ms / 1e3), "jobs": len(arrivals), "done": len(done),
            "failed": len(results) - len(done),
            "failures": sorted({f'{r["status"]}: {r["message"]}' for r in results if r["state"] != "done"})[:5],
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "max": float(lat.max())},
            "wall_s": wall, "rounds": info["rounds"], "bp_launches": info["bp_launches"],
            "gpu_round_s": info["gpu_round_ms"] / 1e3, "host_round_s": info["host_round_ms"] / 1e3,
            "host_admit_s": info["host_admit_ms"] / 1e3, "oom_requeues": info["oom_requeues"],
            "bytes_peak": info["bytes_peak"],
            "device_busy_updates_per_s": upd / max(info["gpu_round_ms"] / 1e3, 1e-9), "clocks": clocks}


def serial_service_times(T, torch, pool, rings):
    """Plain FP32, one series at a time, end to end: upload from pinned memory,
    reconstruct, download the whole volume (seconds per pool series)."""
    service = []
    for i, (j, h) in enumerate(pool):
        out = rings.out(i, j)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        with T.Session(j["w"], j["w"], len(j["ang"]), j["ang"], **job_kw(j, "fp32")) as s:
            s.upload(h.numpy())
            s.reconstruct()
            s.download(out=out)
        service.append(time.perf_counter() - t1)
    return service


def serve_stream(rate, duration, large_frac, budget_gb, pool_small, n_large=2, pool=None, seed=20):
    """Poisson request stream through tg_server (continuous batching, HBM admission
    budget) with p50/p99 latency; beside it the same arrivals served one at a time
    by plain FP32 sessions (each pool series timed once end to end, the arrivals
    replayed through one first-in first-out server with those service times)."""
    import torch

    import tiltgpu as T
    rng = np.random.default_rng(seed)
    if pool is None:
        small = c4_jobs(pool_small, seed=5)
        big_ang = np.arange(-60, 61, 1.0).astype(np.float32)
        large = [dict(w=2048, nv=121, ang=big_ang, thick=800, sirt=0, seed=9000 + k, noise=0.5)
                 for k in range(n_large)]
        pool = make_pool(T, torch, small + large)
    small_idx = [k for k, (j, _) in enumerate(pool) if j["w"] < 2048]
    large_idx = [k for k, (j, _) in enumerate(pool) if j["w"] >= 2048]
    arrivals, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        if large_idx and rng.random() < large_frac:
            k = large_idx[int(rng.integers(0, len(large_idx)))]
        else:
            k = small_idx[int(rng.integers(0, len(small_idx)))]
        arrivals.append((t, k))
    rings = OutRings(torch, pool)
    sv = served_run(T, pool, arrivals, budget_gb, rings)
    service = serial_service_times(T, torch, pool, rings)
    free_at, serial_lat = 0.0, []
    for ta, k in arrivals:
        begin = max(ta, free_at)
        free_at = begin + service[k]
        serial_lat.append(free_at - ta)
    arr_upd = sum(job_updates(pool[k][0]) for _, k in arrivals)
    serial_busy = sum(service[k] for _, k in arrivals)
    serial = {"value": arr_upd / serial_busy, "unit": "updates/s", "utilisation": serial_busy / duration,
              "latency_ms_fifo_replay": {"p50": float(np.percentile(serial_lat, 50)) * 1e3,
                                         "p99": float(np.percentile(serial_lat, 99)) * 1e3},
              "how": "each pool series timed once end to end (upload, reconstruct, download); "
                     "the arrivals replayed through one FIFO server"}
    n_small = len(small_idx)
    line = {"metric": METRIC, "unit": "updates/s", "n_gpus": 1,
            "workload": (f"serve: Poisson {rate} jobs/s for {duration:.0f} s, C4 sizes "
                         f"({n_small} seeded series) + {large_frac:.0%} 2048^2x121-view WBP jobs "
                         f"(thickness 800), FP16 staging, SIRT relax {C4_RELAX}, budget {budget_gb:.0f} GB"),
            **sv, "serial_plain_fp32": serial, "ratio_vs_serial_plain_fp32": sv["value"] / serial["value"],
            "data": "synthetic seeded phantoms, projections from pinned host memory"}
    return line, pool


def c4_at_once(budget_gb=150.0, pool=None):
    """The 64 uneven C4 series (WBP:SIRT(10) 3:1) submitted together to the server
    (FP16 staging, continuous batching, every projection copied in from pinned host
    memory and every volume copied out) against plain FP32 series run one after
    another end to end (upload, reconstruct, download)."""
    import torch

    import tiltgpu as T
    if pool is None:
        pool = make_pool(T, torch, c4_jobs())
    rings = OutRings(torch, pool)
    sv = served_run(T, pool, [(0.0, k) for k in range(len(pool))], budget_gb, rings)
    service = serial_service_times(T, torch, pool, rings)
    upd = sum(job_updates(j) for j, _ in pool)
    plain = upd / sum(service)
    return {"workload": "c4: 64 uneven series (widths 256-1024, 41-121 views, thickness 100-500, "
                        "WBP:SIRT(10) 3:1), all submitted at once, host copies included",
            "batched_fp16_served": sv["value"], "plain_fp32_serial": plain,
            "ratio_vs_plain_fp32": sv["value"] / plain, "done": sv["done"], "failed": sv["failed"],
            "failures": sv["failures"], "sirt_relax": C4_RELAX,
            "wall_s": sv["wall_s"], "serial_s": sum(service), "unit": "updates/s"}


def run_cli(args):
    """The drop-in `tilt` command on the large WBP series, files in and out: a 2.0 GB
    float MRC stack and its .tlt written to a scratch directory, then `bin/tilt` run
    (overlapped read/upload and download/write) with mode-2 and mode-12 output; wall
    clock of the whole command against the device-resident rate."""
    import shutil
    import tempfile

    import torch

    import tiltgpu as T
    torch.cuda.set_device(0)
    w = c2_workload()
    nx, ny, onz, ang = w["nx"], w["ny"], w["onz"], w["angles"]
    nz = len(ang)
    d = torch.empty(nz * ny * nx, dtype=torch.float32, device="cuda")
    T.synth_projections(ang, nx=nx, ny=ny, vol_nx=nx, vol_nz=onz, n_ell=w["n_ell"], rmin=3, rmax=40, dmin=0.2,
                        dmax=1.0, n_beads=w["n_beads"], bead_r=5, bead_d=5.0, noise_kind=2, noise=20000.0,
                        seed=1000, out_device_ptr=d.data_ptr())
    proj = d.cpu().numpy().reshape(nz, ny, nx)
    del d
    torch.cuda.empty_cache()
    tmp = tempfile.mkdtemp(prefix="tilt_cli_", dir=args.scratch or None)
    res = {"workload": w["name"] + ", through bin/tilt (MRC in, MRC out, --log)", "unit": "updates/s"}
    try:
        src, tlt = os.path.join(tmp, "in.mrc"), os.path.join(tmp, "in.tlt")
        T.mrc_write_f32(src, T.mrc_header_new(nx, ny, nz, "Float"), proj)
        T.write_tilt_file(tlt, ang)
        upd = float(nx) * onz * ny * nz
        for mode in (2, 12):
            out = os.path.join(tmp, f"out{mode}.rec")
            t0 = time.perf_counter()
            r = subprocess.run([T.CLI_PATH, "-i", src, "-o", out, "-t", tlt, "-z", str(onz), "--radial",
                                "0.35,0.035", "--log", "--storage", "fp16", "--mode", str(mode)],
                               capture_output=True, text=True)
            wall = time.perf_counter() - t0
            stages = [ln for ln in r.stderr.splitlines() if ln.startswith("tilt: read+upload")]
            res[f"mode{mode}"] = {"rc": r.returncode, "wall_s": wall, "value": upd / wall,
                                  "output_bytes": os.path.getsize(out) if os.path.exists(out) else None,
                                  "stages": stages[-1] if stages else r.stderr[-300:]}
            if os.path.exists(out):
                os.remove(out)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    print(json.dumps(res), flush=True)


def run_serve(args):
    import torch
    torch.cuda.set_device(0)
    line, _ = serve_stream(args.rate, args.duration, args.large_frac, args.budget_gb, args.pool)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c3", "c4", "serve", "cli"])
    ap.add_argument("--sirt", type=int, default=20, help="c3: SIRT iterations")
    ap.add_argument("--xtilt", type=float, default=1.5, help="c3: x-axis tilt of every view (deg)")
    ap.add_argument("--sirt-relax", type=float, default=1.0, help="c3: SIRT relaxation (the reference's default 1.0)")
    ap.add_argument("--rate", type=float, default=20.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=120.0, help="serve: seconds of arrivals")
    ap.add_argument("--large-frac", type=float, default=0.05, help="serve: share of 2048^2 jobs")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: HBM admission budget")
    ap.add_argument("--pool", type=int, default=32, help="serve: distinct seeded C4-size series")
    ap.add_argument("--serve-seconds", type=float, default=10.0,
                    help="default run: seconds of the short served stream reported under 'serving'")
    ap.add_argument("--saturated-seconds", type=float, default=15.0,
                    help="default run: seconds of the saturated (40 jobs/s) served stream")
    ap.add_argument("--no-serving", action="store_true", help="default run: skip the served streams and C4")
    ap.add_argument("--scratch", default=None, help="cli: directory for the MRC files (default: the system temp)")
    ap.add_argument("--forms", default=None, help="staging precisions to time (c1/c2: fp32,fp16; c3: fp32,bf16)")
    ap.add_argument("--profile", action="store_true",
                    help="time the requested forms only (no e2e, no CPU baseline); for ncu captures")
    args = ap.parse_args()
    if args.workload in WORKLOADS and args.forms is None:
        args.forms = "fp32,fp16"
    if not args.profile and args.workload in WORKLOADS and set(args.forms.split(",")) != {"fp32", "fp16"}:
        ap.error("--forms other than fp32,fp16 needs --profile")
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "c3":
        run_c3(args)
        return
    if args.workload == "c4":
        run_c4(args)
        return
    if args.workload == "serve":
        run_serve(args)
        return
    if args.workload == "cli":
        run_cli(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
