"""Benchmark of the B200 `nextevent_path_tracer` (plain NEE+MIS) on the 1M-triangle workload.

One step = one full render of the heightfield-and-spheres scene (512x512-vertex
fBm floor + 2000 icospheres, 50% Oren-Nayar / 50% Lambert+Phong, 4 area
lights, 1,162,250 triangles) at 1024x512, 64 spp, max depth 16
(num_path_vertices 18): 33.5M camera paths. Inputs are synthetic and seeded
(wurstrenderer_b200/scenes.py); the scene is resident in HBM before timing.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun every rank renders the whole image with its own random streams
(weak scaling: per-GPU work fixed) and the FP64 films are summed onto rank 0
with one NCCL reduce per step. Rank 0 prints one JSON line.

`value` is device time (CUDA events on the renderer's stream, summed over the K
steps, max over ranks; at N > 1 each step also includes the FP64 film reduce,
timed by CUDA events on the stream it is issued on); `e2e` is the same metric
through the public C ABI call with host output (wr_render: film copied
device->host into pinned host memory inside the timed region; at N > 1 render,
reduce and read-back of the reduced film).

The default run also carries the guided-vs-plain equal-time studies of the two
guided workloads against their FP64 reference crops: the door-gap room (config 4,
`equal_time_relmse`) and the 10M-triangle full combination (config 5, `c5`, with
its plain Mpaths/s). Both train with config 4's Adam learning rate, 1e-3; each
also repeats its guided renders at 2e-3 under `lr_0.002` (same plain renders).
The `lbvh` key renders the same workload on the device-built LBVH tree.
The CPU baseline runs the oracle (the reference's own renderer code compiled
here, or its FP64 restatement) on the box's host cores on a bounded sample of
the same workload (full frame at reduced spp; per-path work is unchanged).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "heightfield_spheres_1M: 1024x512, 64 spp, num_path_vertices 18 (max depth 16), 1,162,250 triangles"
WORKLOAD_JOBS = ("jobs128: 128 jobs over the 36-triangle Cornell box, random cameras, resolutions {64,128,256,512}^2, "
                 "spp log-uniform in [4, 256], num_path_vertices 14, one wavefront / one graph launch per step")
METRIC = "Mpaths/s"


WORKLOAD_PHONG = ("heightfield_phong: 1024x512, 16 spp, num_path_vertices 18; the heightfield workload's 522k-triangle "
                  "floor and 4 lights as triangles, its 2000 spheres as 160,000 Phong tessellation patches "
                  "(80-face icospheres with radial vertex normals, FP64 patch test)")


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def scene_path(rank, world, dist, workload="heightfield"):
    """Writes the seeded workload once per node (rank 0), shared by the other ranks."""
    from wurstrenderer_b200 import scenes
    if workload == "jobs128":
        d = os.path.join(tempfile.gettempdir(), "wurst_b200_bench_cornell_v2")
        p = os.path.join(d, "cornell.json")
        writer = lambda: scenes.write_cornell(d)
    elif workload in ("door", "c5"):
        d, p = workload_dir(workload)
        writer = lambda: scenes.write_guided_workload(workload, d, spp=WORKLOAD_SPP[workload])
    elif workload == "phong":
        d = os.path.join(tempfile.gettempdir(), "wurst_b200_bench_heightfield_phong_v1")
        p = os.path.join(d, "heightfield_phong.json")
        writer = lambda: scenes.write_heightfield_phong(d)
    else:
        d = os.path.join(tempfile.gettempdir(), "wurst_b200_bench_heightfield_v1")
        p = os.path.join(d, "heightfield_spheres.json")
        writer = lambda: scenes.write_heightfield_spheres(d)
    if rank == 0 and not os.path.exists(p + ".done"):
        writer()
        open(p + ".done", "w").write("ok")
    if world > 1:
        dist.barrier()
    while not os.path.exists(p + ".done"):
        time.sleep(0.1)
    return p


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region.

    Read-only NVML queries every 10 ms on the device this rank renders on (matched by UUID, so
    CUDA_VISIBLE_DEVICES remapping does not matter); where NVML is not usable, nvidia-smi every
    200 ms on the local-rank index."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    PERIOD_S = 0.01

    def __init__(self, gpu_index, cuda_device=None):
        self.rows = []
        self.proc = None
        self.gpu = gpu_index
        self.nvml = None
        self.stop_evt = threading.Event()
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(cuda_device if cuda_device is not None else 0).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            bits = (pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap)
            self.nvml = (pynvml, h, bits, float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)))
        except Exception:
            self.nvml = None

    def _poll_nvml(self):
        pynvml, h, bits, _ = self.nvml
        while not self.stop_evt.is_set():
            try:
                sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, [n for n, b in zip(self.NAMES, bits) if r & b]))
            except Exception:
                pass
            self.stop_evt.wait(self.PERIOD_S)

    def start(self):
        if self.nvml is not None:
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.nvml is not None:
            self.stop_evt.set()
            self.t.join(timeout=2)
            sm = sorted(r[0] for r in self.rows)
            reasons = sorted({n for r in self.rows for n in r[1]})
            return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": self.nvml[3], "reasons": reasons,
                    "samples": len(sm), "sm_mhz_min": sm[0] if sm else None, "source": "nvml, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = self.NAMES
        for r in self.rows:
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_ray():
    """DRAM bytes per traced ray of the traversal kernels from the committed ncu capture summary
    (keys "k_extend" and "k_trace_pair"), when present."""
    p = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def l1_profile():
    """L1/TEX figures of the traversal kernel from the committed single-launch ncu capture."""
    p = os.path.join(ROOT, "profiles", "k_trace_pair_l1.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(path, budget_s=20.0):
    """The reference's renderer code (oracle/_ref) or the oracle's restatement on the host cores."""
    import oracle
    cores = os.cpu_count() or 1
    try:
        import oracle as o
        if o.reference_available():
            out = os.path.join(tempfile.gettempdir(), "wurst_ref_bench.pfm")
            spp = 1
            rep = o.run_reference(path, out, spp=spp)
            # grow the sample until it takes a few seconds of the budget
            while rep["seconds"] < budget_s / 4 and spp < 64:
                spp *= 2
                rep = o.run_reference(path, out, spp=spp)
            # one core: the same per-tile loop on one thread over the full frame at 1 spp
            one = o.run_reference(path, out, spp=1, serial=True, threads=1)
            return {"value": rep["paths"] / rep["seconds"] / 1e6, "unit": METRIC, "cores": rep["threads"],
                    "kind": "reference", "cpu_model": cpu_model(),
                    "value_1core": one["paths"] / one["seconds"] / 1e6,
                    "sample": "full %dx%d frame at %d spp (%d paths), reference PathNeeRenderer::render() with "
                              "Embree replaced by the oracle's FP32 BVH ray caster; value_1core: the same per-tile "
                              "loop on one thread, full frame at 1 spp" % (rep["width"], rep["height"], spp,
                                                                           rep["paths"])}
    except Exception as e:  # fall through to the restatement
        print("reference baseline unavailable: %s" % e, file=sys.stderr)
    sc = oracle.OracleScene(path)
    spp = 1
    _, sec, paths = sc.render(spp=spp, threads=cores)
    while sec < budget_s / 4 and spp < 64:
        spp *= 2
        _, sec, paths = sc.render(spp=spp, threads=cores)
    return {"value": paths / sec / 1e6, "unit": METRIC, "cores": cores, "kind": "port", "cpu_model": cpu_model(),
            "sample": "full %dx%d frame at %d spp (%d paths), FP64 oracle restatement" % (sc.width, sc.height, spp,
                                                                                             paths)}


def run_reference_arm(args, rank):
    """--impl reference: the reference's CPU implementation on the host cores (rank 0 only)."""
    if rank != 0:
        return
    import oracle
    path = scene_path(0, 1, None)
    cores = os.cpu_count() or 1
    use_ref = oracle.reference_available()
    kind = "reference" if use_ref else "port"
    spp_sample = 1
    times, paths_total = [], 0
    sc = None if use_ref else oracle.OracleScene(path)
    out = os.path.join(tempfile.gettempdir(), "wurst_ref_arm.pfm")
    for i in range(args.warmup + args.steps):
        if use_ref:
            rep = oracle.run_reference(path, out, spp=spp_sample, salt=i + 1)
            sec, paths, threads = rep["seconds"], rep["paths"], rep["threads"]
        else:
            _, sec, paths = sc.render(spp=spp_sample, salt=i + 1, threads=cores)
            threads = cores
        if i >= args.warmup:
            times.append(sec)
            paths_total += paths
    total = sum(times)
    value = paths_total / total / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / max(1, args.steps),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "sample": "each step: full 1024x512 frame at %d spp (same scene, same per-path work)" % spp_sample},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": kind, "cpu_model": cpu_model(),
                             "sample": "full 1024x512 frame at %d spp per step, %d steps" % (spp_sample, args.steps)},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def relmse(x, ref, eps=1e-2):
    import numpy as np
    return float(np.mean((x - ref) ** 2 / (ref ** 2 + eps)))


DOOR_WORKLOAD = ("door_room_200k: closed 6x3x6 m room, 1x1 emitter behind a partition with a 0.2 m door gap, "
                 "300 seeded Phong / Oren-Nayar boxes (197,782 triangles), 1024x1024, num_path_vertices 10")
C5_WORKLOAD = ("full_combination_10M: 2048^2 fBm floor + 20000 icospheres (80 faces) + 16 area lights "
               "(9,980,450 triangles), 2048x1024 FP32 sky (3 Gaussian suns + gradient), Phong exponents up "
               "to 2000, 3840x2160, num_path_vertices 26 (max depth 24)")
STUDY_WORKLOADS = {"door": DOOR_WORKLOAD, "c5": C5_WORKLOAD}


WORKLOAD_SPP = {"door": 256, "c5": 1024}


def workload_dir(name):
    d = os.path.join(tempfile.gettempdir(), "wurst_b200_bench_%s_v1" % name)
    return d, os.path.join(d, "door.json" if name == "door" else "full_combination.json")


def workload_scene(name):
    """Writes (once per box) the full-size scene of a guided-vs-plain workload; returns its JSON path."""
    from wurstrenderer_b200 import scenes
    d, p = workload_dir(name)
    if not os.path.exists(p + ".done"):
        scenes.write_guided_workload(name, d, spp=WORKLOAD_SPP[name])
        open(p + ".done", "w").write("ok")
    return p


def guided_vs_plain(wr, name="door", plain_spp=256, seeds=2, extra_lrs=()):
    """Equal-time relMSE of the learned proposal against plain NEE+MIS on a full-size workload,
    both measured against the reference's own FP64 render of a crop at 16384 spp
    (tests/golden/<name>_crop_ref_{a,b}.npy, two independent 8192-spp halves). The guided render
    (training on its first 32 spp included) gets the device time of the plain render. The guided
    renders train with the workload's Adam learning rate (1e-3); each rate in `extra_lrs` adds the
    same guided study at that rate under "lr_<rate>" (same plain renders)."""
    import numpy as np
    gdir = os.path.join(ROOT, "tests", "golden")
    meta_p = os.path.join(gdir, "%s_crop_meta.json" % name)
    if not os.path.exists(meta_p):
        return {"unavailable": "reference crop not generated (tests/golden/make_crop_golden.py)"}
    meta = json.load(open(meta_p))
    ref_a = np.load(os.path.join(gdir, "%s_crop_ref_a.npy" % name)).astype(np.float64)
    ref_b = np.load(os.path.join(gdir, "%s_crop_ref_b.npy" % name)).astype(np.float64)
    ref = 0.5 * (ref_a + ref_b)
    x0, y0, x1, y1 = meta["crop"]
    p = workload_scene(name)
    out = {"workload": STUDY_WORKLOADS[name],
           "oracle": "reference PathNeeRenderer (FP64 CPU), 16384 spp, crop %s" % meta["crop"],
           "relmse_def": "mean over crop pixels and channels of (x - ref)^2 / (ref^2 + 1e-2)",
           "oracle_noise_relmse": relmse(ref_a, ref_b) / 4.0}
    with wr.Scene.from_file(p) as sc:
        sc.render(spp=1, seed=1)                       # warm-up (allocations, graph paths)
        sc.render(spp=2, seed=2, guiding=1, guide_train_spp=2, guide_steps=16)
        plain_err, plain_err3, plain_ms = [], [], []
        for i in range(seeds):
            img = sc.render(spp=plain_spp, seed=100 + i)
            plain_ms.append(sc.stats["render_ms"])
            plain_err.append(relmse(img[y0:y1, x0:x1], ref))
            plain_err3.append(relmse(img[y0:y1, x0:x1], ref, eps=1e-3))
        t_budget = float(np.mean(plain_ms))

        def guided(lr):
            img = sc.render(spp=plain_spp, seed=200, guiding=1, guide_lr=lr)   # calibration: guided time per spp
            st = sc.stats
            per_spp = (st["render_ms"] - st["guide_train_ms"]) / plain_spp
            g_spp = max(33, int((t_budget - st["guide_train_ms"]) / per_spp))
            r = {"spp": g_spp, "err": [], "err3": [], "ms": [], "train": []}
            for i in range(seeds):
                img = sc.render(spp=g_spp, seed=300 + i, guiding=1, guide_lr=lr)
                st = sc.stats
                r["ms"].append(st["render_ms"])
                r["train"].append(st["guide_train_ms"])
                r["err"].append(relmse(img[y0:y1, x0:x1], ref))
                r["err3"].append(relmse(img[y0:y1, x0:x1], ref, eps=1e-3))
                r["steps"], r["records"] = st["guide_steps"], st["guide_records"]
            return r, img

        res, img = guided(None)
        g_spp, g_err, g_err3, g_ms, g_train = res["spp"], res["err"], res["err3"], res["ms"], res["train"]
        steps, records = res["steps"], res["records"]
        extra = {lr: guided(lr)[0] for lr in extra_lrs}
    pe, ge = float(np.mean(plain_err)), float(np.mean(g_err))
    pm, gm = float(np.mean(plain_ms)), float(np.mean(g_ms))
    npix = img.shape[0] * img.shape[1]
    out.update({"plain": {"spp": plain_spp, "relmse": pe, "ms": pm, "runs": seeds,
                          "mpaths_s": npix * plain_spp / (pm * 1e3)},
                "guided": {"spp": g_spp, "relmse": ge, "ms": gm, "train_ms": float(np.mean(g_train)),
                           "adam_steps": steps, "records": records, "runs": seeds,
                           "mpaths_s": npix * g_spp / (gm * 1e3)},
                "relmse_ratio_equal_time": (ge * gm) / (pe * pm),
                # the same with the 1e-3 epsilon of the reference's error image (util/errorimage.h:18)
                "relmse_eps1e-3": {"plain": float(np.mean(plain_err3)), "guided": float(np.mean(g_err3)),
                                   "ratio_equal_time": (float(np.mean(g_err3)) * gm) / (float(np.mean(plain_err3)) * pm)},
                "adam_lr": 1e-3,
                "note": "ratio = (relMSE_guided x time_guided) / (relMSE_plain x time_plain); relMSE of an "
                        "unbiased estimator scales as 1/time, so this is the equal-time ratio"})
    for lr, r in extra.items():
        e, m = float(np.mean(r["err"])), float(np.mean(r["ms"]))
        out["lr_%g" % lr] = {"adam_lr": lr, "spp": r["spp"], "relmse": e, "ms": m,
                             "train_ms": float(np.mean(r["train"])), "adam_steps": r["steps"],
                             "relmse_ratio_equal_time": (e * m) / (pe * pm)}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--queue-capacity", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0, help="override the workload's spp (profiling runs only)")
    ap.add_argument("--quick", action="store_true", help="skip e2e, profile and CPU baseline (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="use the default wavefront settings")
    ap.add_argument("--bvh-width", type=int, default=0, choices=[0, 2, 8],
                    help="2: binary BVH, 8: compressed 8-wide BVH, 0: the library default")
    ap.add_argument("--no-guiding", action="store_true", help="skip the guided-vs-plain equal-time studies")
    ap.add_argument("--no-c5", action="store_true", help="skip the config-5 (10M triangles) study of the default run")
    ap.add_argument("--no-graph", action="store_true",
                    help="host-driven launches instead of one graph per render (profiling runs: ncu does not "
                         "profile kernels inside conditional graph nodes)")
    ap.add_argument("--workload", default="heightfield", choices=["heightfield", "jobs128", "door", "c5", "phong"],
                    help="heightfield: the 1M-triangle single render (headline); jobs128: 128 batched jobs "
                         "over the Cornell box, one graph launch per step; door: one guided render (learned "
                         "proposal trained on its first 32 spp) of the 200k-triangle door-gap room at 256 spp; "
                         "c5: one plain render of the 10M-triangle full combination at 3840x2160, 1024 spp, "
                         "with the guided-vs-plain study on it; phong: the heightfield scene with its spheres "
                         "as Phong tessellation patches, 16 spp")
    args = ap.parse_args()

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local_rank = env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return

    import numpy as np
    import torch
    import wurstrenderer_b200 as wr

    dist = None
    torch.cuda.set_device(local_rank)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    wr.set_device(local_rank)
    path = scene_path(rank, world, dist, args.workload)

    t0 = time.perf_counter()
    scene = wr.Scene.from_file(path, bvh_width=args.bvh_width)
    load_s = time.perf_counter() - t0
    info = scene.info
    W, H = info["width"], info["height"]
    spp, nverts = info["num_spp"], info["num_path_vertices"]
    if args.spp:
        spp = args.spp
    film = torch.empty((H, W, 3), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")   # > 126 MB L2
    tune = {}
    tune_ms = None
    tune_probe = None
    batch_jobs = None
    if args.workload == "jobs128":
        from wurstrenderer_b200 import scenes
        batch_jobs = scenes.batch_jobs(seed=1003, n_jobs=128, num_path_vertices=14)
        paths_batch = sum(j["camera"]["resolution"][0] * j["camera"]["resolution"][1] * j["num_spp"]
                          for j in batch_jobs)
    if not args.no_autotune:
        if batch_jobs is None:
            tune, tune_ms = scene.autotune(probe_spp=16)
            tune_probe = "the scene's camera at 16 spp"
        else:
            # the batch itself is the probe: every 4th job (a quarter of the cameras and resolutions)
            # at a quarter of its spp, about 1/16 of the batch's paths
            probe = [dict(j, num_spp=max(1, j["num_spp"] // 4), seed=77 + k) for k, j in enumerate(batch_jobs[::4])]
            tune, tune_ms = scene.autotune_batch(probe)
            tune_probe = "wr_autotune_batch over every 4th job of the batch at 1/4 of its spp (%d jobs, %d paths)" % (
                len(probe), sum(j["camera"]["resolution"][0] * j["camera"]["resolution"][1] * j["num_spp"]
                                for j in probe))
        tune = {k: v for k, v in tune.items() if k != "use_graph"}
    if args.queue_capacity:
        tune["queue_capacity"] = args.queue_capacity
    qc = tune.get("queue_capacity")
    knobs = dict(grid_trace=tune.get("grid_trace"), grid_shade=tune.get("grid_shade"),
                 trace_block=tune.get("trace_block"), fetch_threshold=tune.get("fetch_threshold"),
                 use_graph=not args.no_graph)

    from wurstrenderer_b200.distributed import combine_films, max_over_ranks, rank_seed

    red0, red1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step(seed):
        seed = rank_seed(seed, rank)
        if batch_jobs is not None:
            for k, j in enumerate(batch_jobs):
                j["seed"] = seed + k
            scene.render_batch(batch_jobs, queue_capacity=qc, **knobs)
            return scene.stats
        scene.render_device(film.data_ptr(), spp=spp, seed=seed, queue_capacity=qc,
                            guiding=1 if args.workload == "door" else 0, **knobs)
        st = scene.stats
        if world > 1:
            # the one exchange of the step: the FP64 film reduce (NCCL), timed with CUDA events on the
            # stream it is issued on, after the render (which has synchronised its own stream)
            red0.record()
            combine_films(film, world, dist)
            red1.record()
            red1.synchronize()
            st["reduce_ms"] = red0.elapsed_time(red1)
            st["render_ms"] += st["reduce_ms"]
        return st

    for i in range(args.warmup):
        step(1000 * rank + i)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank, torch.cuda.current_device())
    clocks.start()
    dev_ms, reduce_ms, launches, iters = 0.0, 0.0, 0, 0
    wall0 = time.perf_counter()
    for i in range(args.steps):
        flush.fill_(float(i))               # evict L2 between timed steps (outside the per-step device timing)
        torch.cuda.synchronize()
        st = step(7919 * (rank + 1) + i)
        dev_ms += st["render_ms"]
        reduce_ms += st.get("reduce_ms", 0.0)
        launches += st["kernel_launches"]
        iters += st["iterations"]
    torch.cuda.synchronize()
    wall_ms = (time.perf_counter() - wall0) * 1e3
    if world > 1:
        dist.barrier()
    clk = clocks.stop()

    max_ms = max_over_ranks(dev_ms, world, dist, device="cuda")
    paths_per_rank = W * H * spp if batch_jobs is None else paths_batch
    value = paths_per_rank * world * args.steps / (max_ms / 1e3) / 1e6

    if args.quick:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "ms_per_step": max_ms / args.steps, "spp": spp, "quick": True}
        if args.steps == 1 and args.warmup == 0 and batch_jobs is None:
            # the timed render once more, with its per-kernel launch and ray counts (profiling runs: an
            # ncu capture limited to the first extend launches sees only the timed render's)
            scene.render_device(film.data_ptr(), spp=spp, seed=rank_seed(7919 * (rank + 1), rank),
                                queue_capacity=qc, profile=2, guiding=1 if args.workload == "door" else 0,
                                **knobs)
            pst = scene.stats
            line["extend_launches"] = dict(zip(wr.KERNELS, pst["kernel_count"]))["extend"]
            line["extend_rays"] = dict(zip(wr.KERNELS, pst["kernel_items"]))["extend"]
            line["shadow_rays"] = dict(zip(wr.KERNELS, pst["kernel_items"]))["shadow"]
        if rank == 0:
            print(json.dumps(line), flush=True)
        scene.close()
        if world > 1:
            dist.destroy_process_group()
        return

    # end to end through the public C ABI with host output (device->host copy of the film inside)
    host_t = torch.empty((H, W, 3), dtype=torch.float64, pin_memory=True)   # pinned host film
    host = host_t.numpy()
    e2e_ms = 0.0
    for i in range(args.steps):
        torch.cuda.synchronize()
        a = time.perf_counter()
        if batch_jobs is not None:
            step(424242 + 1000 * i)
        elif world > 1:
            # per rank: render into device memory, reduce the films onto rank 0, read the film back
            scene.render_device(film.data_ptr(), spp=spp, seed=rank_seed(424242 + i, rank), queue_capacity=qc,
                                guiding=1 if args.workload == "door" else 0, **knobs)
            combine_films(film, world, dist)
            host_t.copy_(film)
        else:
            scene.render(spp=spp, seed=424242 + i, out=host, queue_capacity=qc,
                         guiding=1 if args.workload == "door" else 0, **knobs)
        e2e_ms += (time.perf_counter() - a) * 1e3
    e2e_value = paths_per_rank * world * args.steps / (max_over_ranks(e2e_ms, world, dist, device="cuda") / 1e3) / 1e6

    # one profiled render (per-kernel events + traversal counters) for the roofline, outside the timed region
    if batch_jobs is not None:
        for k, j in enumerate(batch_jobs):
            j["seed"] = 99 + k
        scene.render_batch(batch_jobs, queue_capacity=qc, profile=2, **knobs)
    else:
        scene.render_device(film.data_ptr(), spp=spp, seed=99, queue_capacity=qc, profile=2,
                            guiding=1 if args.workload == "door" else 0, **knobs)
    prof = scene.stats
    kn = wr.KERNELS
    k_ms = dict(zip(kn, prof["kernel_ms"]))
    k_cnt = dict(zip(kn, prof["kernel_count"]))
    k_items = dict(zip(kn, prof["kernel_items"]))
    rays = k_items["extend"]
    nv, nt = prof["extend_node_visits"], prof["extend_tri_tests"]
    alg_bytes = 48 * rays + 64 * nv + 48 * nt            # 32 B ray in + 16 B hit out + 64 B/node + 48 B/triangle
    launches_e = max(1, k_cnt["extend"])
    avg_ms = k_ms["extend"] / launches_e
    achieved = (alg_bytes / launches_e) / (avg_ms / 1e3) / 1e9
    peak, peak_kind = measured_peaks()
    tr = traffic_per_ray()
    traffic = tr["k_extend"]["dram_bytes_per_ray"] * rays / launches_e if "k_extend" in tr else None
    extend_alone = {"kernel": "k_extend (closest hit only, separate-kernel schedule)", "achieved": achieved,
                    "frac": achieved / peak, "traffic": traffic,
                    "dram_gbs": None if traffic is None else traffic / (avg_ms / 1e3) / 1e9,
                    "alg_bytes_per_launch": alg_bytes / launches_e, "avg_launch_ms": avg_ms,
                    "rays_per_launch": rays / launches_e, "node_visits_per_ray": nv / max(1, rays),
                    "tri_tests_per_ray": nt / max(1, rays)}

    # the same render with the fused schedule the timed renders use: per-launch device time of
    # k_trace_pair (this iteration's extend rays + the previous iteration's shadow rays)
    if batch_jobs is not None:
        scene.render_batch(batch_jobs, queue_capacity=qc, profile=3, **knobs)
    else:
        scene.render_device(film.data_ptr(), spp=spp, seed=99, queue_capacity=qc, profile=3,
                            guiding=1 if args.workload == "door" else 0, **knobs)
    p3 = scene.stats
    k3_ms = dict(zip(kn, p3["kernel_ms"]))
    k3_cnt = dict(zip(kn, p3["kernel_count"]))
    k3_items = dict(zip(kn, p3["kernel_items"]))
    rays_e, rays_s = k3_items["extend"], k3_items["shadow"]
    # shadow ray: 32 B in + 4 B visibility out; same node / triangle terms
    alg_pair = (48 * rays_e + 36 * rays_s + 64 * (p3["extend_node_visits"] + p3["shadow_node_visits"]) +
                48 * (p3["extend_tri_tests"] + p3["shadow_tri_tests"]))
    launches_p = max(1, k3_cnt["extend"] + k3_cnt["shadow"])      # pair launches + the final shadow launch
    pair_ms = (k3_ms["extend"] + k3_ms["shadow"]) / launches_p
    achieved_p = (alg_pair / launches_p) / (pair_ms / 1e3) / 1e9
    traffic_p = (tr["k_trace_pair"]["dram_bytes_per_ray"] * (rays_e + rays_s) / launches_p
                 if "k_trace_pair" in tr else None)
    roofline = {"bound": "hbm", "achieved": achieved_p, "peak": peak, "unit": "GB/s", "frac": achieved_p / peak,
                "traffic": traffic_p, "peak_kind": peak_kind,
                "kernel": "k_trace_pair (closest hit of this iteration's rays + any hit of the previous "
                          "iteration's shadow rays, one persistent launch; the timed renders' traversal kernel)",
                "dram_gbs": None if traffic_p is None else traffic_p / (pair_ms / 1e3) / 1e9,
                # measured DRAM bytes over the same time: the HBM share actually used (the
                # algorithmic bytes are mostly L1 / L2 hits, so `frac` can exceed 1)
                "dram_frac": None if traffic_p is None else traffic_p / (pair_ms / 1e3) / 1e9 / peak,
                "alg_bytes_per_launch": alg_pair / launches_p, "avg_launch_ms": pair_ms,
                "extend_rays_per_launch": rays_e / launches_p, "shadow_rays_per_launch": rays_s / launches_p,
                "node_visits_per_ray": (p3["extend_node_visits"] + p3["shadow_node_visits"]) / max(1, rays_e + rays_s),
                "tri_tests_per_ray": (p3["extend_tri_tests"] + p3["shadow_tri_tests"]) / max(1, rays_e + rays_s),
                "traversal_share_fused": (k3_ms["extend"] + k3_ms["shadow"]) / max(1e-9, sum(k3_ms.values())),
                "k_extend_alone": extend_alone,
                # the bound the traversal actually meets: L1/TEX throughput (one ncu capture, one launch)
                "l1": (lambda l1: None if l1 is None else {
                    "bound": "l1tex", "frac": l1["l1tex_data_pipe_lsu_wavefronts_pct_of_peak_elapsed"] / 100.0,
                    "unit": "fraction of the L1/TEX data-pipe LSU wavefront peak (elapsed)",
                    "throughput_active": l1["l1tex_throughput_pct_of_peak_active"] / 100.0,
                    "global_ld_bytes_per_launch": 32 * l1["global_ld_sectors"],
                    "global_ld_gbs": 32 * l1["global_ld_sectors"] / (l1["duration_us"] * 1e-6) / 1e9,
                    "l1_hit_rate": l1["l1tex_sector_hit_rate_pct"] / 100.0,
                    "active_threads_per_instruction": l1["active_threads_per_instruction"],
                    "source": l1["source"]})(l1_profile()),
                "kernel_share": {k: k_ms[k] / max(1e-9, sum(k_ms.values())) for k in kn}}

    if batch_jobs is None:
        h2d, d2h = 104, W * H * 3 * 8     # render request (camera, spp, seed) in, FP64 film out
    else:
        h2d = 160 * len(batch_jobs)       # job table (camera + spp + depth + offsets per job)
        d2h = sum(j["camera"]["resolution"][0] * j["camera"]["resolution"][1] * 24 for j in batch_jobs)
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (FP64 film + CDF build)", "data": "synthetic (seeded procedural scene)",
            "config": {"workload": {"heightfield": WORKLOAD, "jobs128": WORKLOAD_JOBS,
                                    "door": DOOR_WORKLOAD + ", 256 spp, guided (learned proposal trained on its "
                                                            "first 32 spp)",
                                    "c5": C5_WORKLOAD + ", 1024 spp, plain NEE+MIS",
                                    "phong": WORKLOAD_PHONG}[args.workload],
                       "parallelism": "replicas x%d, FP64 film reduce" % world,
                       "reduce_ms_per_step": reduce_ms / args.steps if world > 1 else None,
                       "autotuned": tune, "autotune_probe_ms": tune_ms, "autotune_probe": tune_probe,
                       "l2": "256 MB buffer written between timed steps; path state > L2",
                       "queue_capacity": prof["queue_capacity"], "grid_trace": prof["grid_trace"],
                       "grid_shade": prof["grid_shade"], "scene_load_s": load_s,
                       "bvh_nodes": info["bvh_nodes"], "bvh_depth": info["bvh_depth"],
                       "bvh_width": args.bvh_width or "library default",
                       "iterations_per_step": iters / args.steps, "wall_ms_per_step": wall_ms / args.steps},
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": launches,
            "roofline": roofline,
            "clocks": clk,
            "mrays_per_s": (k_items["extend"] + k_items["shadow"]) * world * args.steps / (max_ms / 1e3) / 1e6}
    if world == 1 and args.workload == "heightfield" and args.bvh_width in (0, 2):
        # the on-device LBVH build (Morton codes, radix sort, Karras topology, refit) of the same
        # scene: its device build time and the throughput of renders on that tree
        with wr.Scene.from_file(path, bvh_builder=wr.BVH_DEVICE_LBVH) as ls:
            li = ls.info
            for i in range(2):
                ls.render_device(film.data_ptr(), spp=spp, seed=31 + i, queue_capacity=qc, **knobs)
            lms = []
            for i in range(3):
                flush.fill_(float(i))
                torch.cuda.synchronize()
                ls.render_device(film.data_ptr(), spp=spp, seed=41 + i, queue_capacity=qc, **knobs)
                lms.append(ls.stats["render_ms"])
        line["lbvh"] = {"build_ms_device": li["bvh_ms"], "scene_create_ms": li["build_ms"], "bvh_nodes": li["bvh_nodes"],
                        "bvh_depth": li["bvh_depth"], "mpaths_s": W * H * spp / (sorted(lms)[1] * 1e3),
                        "host_sah": {"build_ms": info["bvh_ms"], "bvh_nodes": info["bvh_nodes"],
                                     "bvh_depth": info["bvh_depth"], "mpaths_s": value},
                        "note": "same workload and settings, tree built on the device instead of by the host binned SAH"}
    if rank == 0 and not args.no_cpu_baseline and batch_jobs is None:
        line["cpu_baseline"] = cpu_baseline(path)
    if world == 1 and not args.no_guiding and args.workload in ("heightfield", "c5"):
        study = "c5" if args.workload == "c5" else "door"
        line["equal_time_relmse"] = guided_vs_plain(wr, study, plain_spp=1024 if study == "c5" else 256,
                                                    seeds=1 if study == "c5" else 3,
                                                    extra_lrs=() if study == "c5" else (2e-3,))
        if args.workload == "heightfield" and not args.no_c5:
            # the second guided-vs-plain target (config 5, 10M triangles): plain Mpaths/s and the
            # equal-time ratio at 256 spp, two seeds
            line["c5"] = guided_vs_plain(wr, "c5", plain_spp=256, seeds=2, extra_lrs=(2e-3,))
    if rank == 0:
        print(json.dumps(line), flush=True)
    scene.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
