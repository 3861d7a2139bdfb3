"""Encode throughput of the B200 NNTC encoder hot path: one step = one whole encode of the workload material.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--form adjoint|plain] [--config C]

Metric: encode Mpix/s = base W x H of the material / encode seconds (the reference's `time ... s total` definition,
src/main.cpp:1788-2948, with the base extent), for the adjoint + mixed-precision form against the plain form on the
same GPU. N > 1 runs under torchrun as REPLICAS: every rank encodes its own seeded material of the same configuration
on its own GPU, with no collective on the data path (the encode does not shard; one material per GPU); the whole-job
value is the pixels of every rank over the slowest rank's time.

- `value`: the `--form` encode (default adjoint) on a device model whose source chain is already resident in HBM,
  timed by the library's CUDA events on its own stream around the whole encode (nntc_b200_encode_result.ms_total), K
  steps bracketed by a barrier and a synchronize, max over ranks. Every encode forms its own per-material caches.
- `forms`: both forms on the same material and GPU - ms per encode, PSNR per texture, the adjoint / plain speed ratio,
  the PSNR delta, and whether the adjoint form's joint pass was kept; the other form is timed over --compare-steps.
- `e2e`: the `--form` encode through the C ABI with host buffers: device_create_from_base (the base plane's H2D copy
  from pinned host memory, the rest of the source chain built on the device), the encode, the D2H read of its result
  (indices, BC endpoints/selectors, decoder) and the asset written to disk, every step.
- `roofline`: the dominant kernel's achieved rate from per-launch CUDA events over the timed steps
  (nntc_b200_kernel_stats), against MEASURED_PEAKS.json.
- `reference_cuda`: the reference's own CUDA encoder (oracle/_ref/nntc_encode_cuda, its sources unmodified, compiled
  for sm_100) on the same material on the same GPU, once: its own `time ... s total` and per-texture PSNR.
- `cpu_baseline`: the reference's own CPU encoder (oracle/_ref/nntc_encode_cpu, built from the reference sources) on
  a bounded crop of the same material, on this host's cores, with this library's encode of the same crop beside it.
- `--impl reference`: that reference CPU encoder alone, timed per step on the crop (rank 0; other ranks exit 0).
The inputs are seeded synthetic textures with the shapes of the configuration (nntc_b200/materials.py); every step's
working set is far larger than the 126 MB L2, so no flush is needed between steps.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from nntc_b200 import abi, check, lib, materials  # noqa: E402

CONFIG_NAMES = {0: "1x256x256 noise+rects c0=2 c1=4", 1: "4x512x512 pbr c0=2 c1=4", 2: "4x1024x1024 pbr c0=2 c1=4",
                3: "4x2048x1024 pbr c0=4 c1=4", 4: "6x4096x4096 pbr c0=4 c1=4"}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9 for i in range(4) if r[5 + i] == "Active"})
        load = [s for s in sm if s > 0.5 * (max(mx) if mx else 1)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def crop_material(mat, size):
    tex = [t[:size, :size].copy() for t in mat.textures]
    return materials.Material(f"{size}x{size} crop of {mat.name}", tex, mat.c0, mat.c1, mat.k).build()


def reference_cpu(mat, steps, warmup, threads):
    """The reference's CPU encoder on `mat` (PNG inputs), each run's own `time ... s total` (Mpix/s of the base)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "nntc_encode_cpu")
    if not os.path.exists(exe):
        return None, "oracle/_ref/nntc_encode_cpu is not built"
    tmp = tempfile.mkdtemp(prefix="nntc_ref_")
    pngs = materials.save_material(mat, os.path.join(tmp, "in"))
    cmd = [exe, *pngs, "-o", os.path.join(tmp, "out") + "/", "--backend", "cpu", "--c0", str(mat.c0), "--c1",
           str(mat.c1), "-j", str(threads)]
    secs = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return None, "reference encoder failed: " + (p.stdout + p.stderr)[-300:]
        # the reference's own span (src/main.cpp:1788 -> 2948), else the process's wall clock
        m = re.search(r"time\s+([\d.]+) s total", p.stdout)
        if i >= warmup:
            secs.append(float(m.group(1)) if m else wall)
    shutil.rmtree(tmp, ignore_errors=True)
    return secs, None


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    mat = crop_material(materials.config(args.config, seed=0) if args.config != 4 else big_material(0), args.crop)
    threads = os.cpu_count() or 1
    secs, err = reference_cpu(mat, args.steps, args.warmup, threads)
    if err:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    mpix = mat.width * mat.height / 1e6
    value = mpix * len(secs) / sum(secs)
    sample = f"{mat.name} (a {args.crop}x{args.crop} crop of the workload), whole encode, {threads} threads"
    print(json.dumps({
        "impl": "reference", "metric": "encode Mpix/s", "value": round(value, 6), "unit": "Mpix/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * sum(secs) / len(secs), 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": CONFIG_NAMES[args.config], "sample": sample},
        "cpu_baseline": {"value": round(value, 6), "unit": "Mpix/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 6), "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
    return 0


def slowest(world, times_ms, device):
    """Every rank's times, the max over ranks of each (the replicas' whole-job time is the slowest rank's)."""
    import torch

    t = torch.tensor(times_ms, dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist

        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_value(world, mpix, steps, ms):
    """Whole-job Mpix/s: every replica encodes `mpix` of base `steps` times within the slowest rank's `ms`."""
    return world * mpix * steps / (ms / 1000.0)


def big_material(seed):
    return materials.config(4, seed=seed)


KERNELS = ["objective", "normal_equations", "assemble_level1", "assemble_level0", "cg_product_level1",
           "quant_sweep", "bc_refine", "cg_product_level0"]   # nntc_b200_kernel ids 0..7
FORMS = {"plain": 0, "adjoint": 1}


def encode_args(L, form):
    ea = abi.EncodeArgs()
    L.nntc_b200_encode_defaults(C.byref(ea))
    ea.form = FORMS[form]
    return ea


def reference_cuda(mat, threads):
    """The reference's own CUDA encoder (oracle/_ref/nntc_encode_cuda, its unmodified sources compiled for sm_100) on
    the same material and layout, once: its `time ... s total` and per-texture PSNR."""
    exe = os.path.join(ROOT, "oracle", "_ref", "nntc_encode_cuda")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/nntc_encode_cuda is not built"}
    tmp = tempfile.mkdtemp(prefix="nntc_refcuda_")
    try:
        pngs = materials.save_material(mat, os.path.join(tmp, "in"), level=1)
        cmd = [exe, *pngs, "-o", os.path.join(tmp, "out") + "/", "--backend", "cuda", "--c0", str(mat.c0), "--c1",
               str(mat.c1), "--png", "0", "-j", str(threads)]
        t0 = time.perf_counter()
        p = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        wall = time.perf_counter() - t0
        if p.returncode != 0:
            return {"unavailable": "the reference CUDA encoder failed: " + (p.stdout + p.stderr)[-300:]}
        m = re.search(r"time\s+([\d.]+) s total", p.stdout)
        secs = float(m.group(1)) if m else wall
        psnr = [float(x) for x in re.findall(r"psnr\s+texture \d+\s+([\d.]+) dB", p.stdout)]
        return {"value": round(mat.width * mat.height / 1e6 / secs, 6), "unit": "Mpix/s", "s_total": round(secs, 3),
                "psnr": psnr, "span": "the reference's own time ... s total (PNG decode, encode, asset write)",
                "build": "the reference's sources unmodified, kernels compiled for sm_100 with -fmad=false"}
    except subprocess.TimeoutExpired:
        return {"unavailable": "the reference CUDA encoder did not finish in 900 s"}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="adjoint", choices=["adjoint", "plain"],
                    help="the form timed for `value` and `e2e`; the other form is timed beside it")
    ap.add_argument("--compare-steps", type=int, default=3, help="timed encodes of the other form")
    ap.add_argument("--config", type=int, default=4)
    ap.add_argument("--crop", type=int, default=256, help="edge of the CPU-baseline crop")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true")
    ap.add_argument("--no-precision", action="store_true", help="skip the mixed-precision error report")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    mat = materials.config(args.config, seed=rank) if args.config != 4 else big_material(rank)
    model = abi.make_model(mat)
    L = lib()
    per_site = (C.c_double * len(mat.per_site))(*mat.per_site)
    # a pinned host copy of the base plane: what the e2e leg copies to the device every step (the rest of the source
    # chain is built on the device from it)
    pinned = torch.from_numpy(np.ascontiguousarray(mat.chain[0], np.float32).ravel()).pin_memory()
    base_ptr = C.cast(pinned.data_ptr(), C.POINTER(C.c_float))
    h2d = pinned.numel() * 4

    def outputs():
        k0 = [np.zeros(p[0] * p[1] * mat.c0, np.uint8) for p in mat.planes]
        k1 = [np.zeros(p[2] * p[3] * mat.c1, np.uint8) for p in mat.planes]
        ep = [np.zeros(((p[0] + 3) // 4) * ((p[1] + 3) // 4) * mat.c0 * 2, np.uint8) for p in mat.planes]
        sel = [np.zeros(e.size * 8, np.uint8) for e in ep]
        return k0, k1, ep, sel

    out = outputs()
    d2h = sum(a.size for grp in out for a in grp) + (model.nout * (model.nin + 1)) * 4

    handle = C.c_void_p()
    check(L.nntc_b200_device_create_from_base(C.byref(model), base_ptr, C.byref(handle)), "device_create_from_base")

    def encode_resident(ea):
        r = abi.EncodeResult()
        m = abi.make_model(mat)
        check(L.nntc_b200_encode_on_device(handle, C.byref(m), C.byref(ea), per_site, C.byref(r), None, None, None,
                                           None), "encode")
        return r

    headline, other = args.form, ("plain" if args.form == "adjoint" else "adjoint")
    ea = encode_args(L, headline)
    # the other form first, a few encodes, for the form ratio and the PSNR delta (none with --compare-steps 0)
    ea_other = encode_args(L, other)
    other_results = []
    if args.compare_steps > 0:
        encode_resident(ea_other)
        other_results = [encode_resident(ea_other) for _ in range(args.compare_steps)]
    other_ms = statistics.median(r.ms_total for r in other_results) if other_results else None

    for _ in range(args.warmup):
        encode_resident(ea)
    check(L.nntc_b200_kernel_timing(handle, 1), "timing")
    check(L.nntc_b200_kernel_stats(handle, 0, None, None, 1), "reset")
    launches0 = L.nntc_b200_launch_count()
    results = []
    with Clocks(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            results.append(encode_resident(ea))
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if world > 1:
            dist.barrier()
    launches = L.nntc_b200_launch_count() - launches0
    device_ms = sum(r.ms_total for r in results)
    stats = {}
    for kid, name in enumerate(KERNELS):
        n = C.c_longlong()
        ms = C.c_double()
        check(L.nntc_b200_kernel_stats(handle, kid, C.byref(n), C.byref(ms), 0), "stats")
        stats[name] = (n.value, ms.value)
    check(L.nntc_b200_kernel_timing(handle, 0), "timing")

    # e2e: through the C ABI with host buffers, every step's H2D of the base plane, the encode, the D2H of the shipped
    # state and the asset written to disk (the .dds files and the descriptor); the resident model is released first,
    # and one untimed step warms the path up
    L.nntc_b200_device_destroy(handle)
    e2e_ms = []
    asset_dir = tempfile.mkdtemp(prefix="nntc_asset_")

    def e2e_step():
        h = C.c_void_p()
        m = abi.make_model(mat)
        check(L.nntc_b200_device_create_from_base(C.byref(m), base_ptr, C.byref(h)), "device_create_from_base")
        r = abi.EncodeResult()
        k0, k1, ep, sel = out
        check(L.nntc_b200_encode_on_device(h, C.byref(m), C.byref(ea), per_site, C.byref(r), abi.u8_ptrs(k0),
                                           abi.u8_ptrs(k1), abi.u8_ptrs(ep), abi.u8_ptrs(sel)), "encode")
        L.nntc_b200_device_destroy(h)
        check(L.nntc_b200_write_asset(C.byref(m), abi.u8_ptrs(k0), abi.u8_ptrs(k1), abi.u8_ptrs(ep), abi.u8_ptrs(sel),
                                      mat.width, mat.height, os.path.join(asset_dir, "bench").encode(), None, None),
              "write_asset")

    e2e_step()
    if world > 1:
        dist.barrier()
    for _ in range(args.steps):
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        e2e_step()
        ev1.record()
        ev1.synchronize()
        e2e_ms.append(ev0.elapsed_time(ev1))
    shutil.rmtree(asset_dir, ignore_errors=True)

    device_ms, e2e_total = slowest(world, [device_ms, sum(e2e_ms)], "cuda")
    mpix = mat.width * mat.height / 1e6
    value = job_value(world, mpix, args.steps, device_ms)
    e2e_value = job_value(world, mpix, args.steps, e2e_total)

    if rank == 0:
        hbm, tf, src = peaks()
        fp64 = C.c_double()
        fp32 = C.c_double()
        check(L.nntc_b200_measure_fma_peaks(C.byref(fp64), C.byref(fp32)), "measure_fma_peaks")
        pipes = {"fp64_tflops": round(fp64.value, 2), "fp32_tflops": round(fp32.value, 2),
                 "how": "nntc_b200_measure_fma_peaks: 8 independent FMA chains per thread, 4 blocks per SM, CUDA events"}
        dom = max(stats, key=lambda k: stats[k][1])
        roof = roofline(dom, stats[dom], mat, hbm, tf, src, headline)
        fractions = {}
        for name, st in stats.items():
            if st[0] == 0:
                continue
            per_launch_s = st[1] / st[0] / 1000.0
            entry = {"ms_per_launch": round(st[1] / st[0], 4),
                     "hbm_frac": round(algorithmic_bytes(name, mat, headline) / per_launch_s / 1e9 / hbm, 4),
                     "binding": BINDING[headline].get(name)}
            fl = algorithmic_flops(name, mat)
            if fl:
                pipe = "fp32" if headline == "adjoint" else "fp64"
                peak = fp32.value if pipe == "fp32" else fp64.value
                entry["compute"] = {"pipe": pipe, "achieved_tflops": round(fl / per_launch_s / 1e12, 3),
                                    "peak_tflops": round(peak, 2), "frac": round(fl / per_launch_s / 1e12 / peak, 4)}
            fractions[name] = entry
        nt = len(mat.textures)
        psnr_h = [round(x, 3) for x in results[-1].psnr[:nt]]
        head_ms = device_ms / args.steps
        forms = {headline: {"ms_per_encode": round(head_ms, 2), "mpix_s": round(mpix / (head_ms / 1000), 6),
                            "psnr": psnr_h, "e_ship": results[-1].e_ship}}
        if other_results:
            psnr_o = [round(x, 3) for x in other_results[-1].psnr[:nt]]
            forms[other] = {"ms_per_encode": round(other_ms, 2), "mpix_s": round(mpix / (other_ms / 1000), 6),
                            "psnr": psnr_o, "e_ship": other_results[-1].e_ship, "steps": args.compare_steps}
            adj, pln = forms["adjoint"], forms["plain"]
            forms["adjoint_over_plain"] = round(pln["ms_per_encode"] / adj["ms_per_encode"], 4)
            forms["psnr_delta_db"] = [round(a - b, 3) for a, b in zip(adj["psnr"], pln["psnr"])]
        adj_res = results[-1] if headline == "adjoint" else (other_results[-1] if other_results else None)
        if adj_res is not None:
            forms["joint_pass"] = {"taken": adj_res.joint_taken, "e_before": adj_res.e_before_joint,
                                   "e_reached": adj_res.e_joint, "ms": round(adj_res.ms_joint, 2)}
        line = {
            "metric": "encode Mpix/s", "value": round(value, 6), "unit": "Mpix/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(head_ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3+f32+f64" if headline == "adjoint" else "f32+f64",
            "data": "synthetic (seeded, nntc_b200/materials.py)",
            "config": {"workload": CONFIG_NAMES[args.config], "form": headline, "base": [mat.width, mat.height],
                       "textures": nt, "c0": mat.c0, "c1": mat.c1, "k": mat.k,
                       "chain_pixels": mat.chain_pixels, "parallelism": f"replicas x{world}",
                       "l2": "working set > 126 MB L2 every step, no flush needed",
                       "caches": "the per-material target caches are re-formed inside every encode",
                       "psnr": psnr_h, "rounds": results[-1].rounds_used,
                       "wall_s_per_step": round(wall / args.steps, 3),
                       "phase_ms": {k: round(getattr(results[-1], "ms_" + k), 2) for k in
                                    ("a", "b", "c", "e", "pack", "refine", "joint", "total")},
                       "kernel_ms": {k: [v[0], round(v[1], 2)] for k, v in stats.items()}},
            "forms": forms,
            "e2e": {"value": round(e2e_value, 6), "unit": "Mpix/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "span": "base plane H2D from pinned memory, chain built on the device, encode, D2H of the shipped "
                            "state, asset (.dds + JSON) written to disk"},
            "gpu_launches": launches,
            "roofline": roof,
            "kernel_fractions": fractions,
            "pipe_peaks": pipes,
            "clocks": clocks.summary(),
        }
        if world == 1 and not args.no_precision:
            # the adjoint form's errors against the FP64 form at the state an adjoint-form encode ships
            from nntc_b200.session import Session
            with Session(mat) as s:
                s.encode(encode_args(L, "adjoint"))
                line["precision_vs_fp64"] = {k: float(f"{v:.3g}") for k, v in s.precision_report(mat.k).items()}
                line["precision_vs_fp64"]["what"] = (
                    "max relative error against the FP64 form from the same state: decoder coefficients (tensor-core "
                    "sums vs FP64 sums, per output row), one block (b) / (c') correction (FP32 vs FP64 stencil)")
        if world == 1 and not args.no_reference_cuda:
            line["reference_cuda"] = reference_cuda(mat, os.cpu_count() or 1)
            if "psnr" in line["reference_cuda"]:
                line["reference_cuda"]["psnr_delta_db"] = [round(a - b, 3) for a, b in
                                                           zip(psnr_h, line["reference_cuda"]["psnr"])]
        if not args.no_cpu_baseline and world == 1:
            crop = crop_material(mat, args.crop)
            secs, err = reference_cpu(crop, 1, 0, os.cpu_count() or 1)
            if err:
                line["cpu_baseline"] = {"unavailable": err}
            else:
                # this library on the same crop, the like-for-like ratio's other side
                with_crop = crop_gpu_mpix(L, crop, ea)
                line["cpu_baseline"] = {
                    "value": round(crop.width * crop.height / 1e6 / secs[0], 6), "unit": "Mpix/s",
                    "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"{args.crop}x{args.crop} crop of the workload ({nt} textures, c0 {mat.c0} c1 {mat.c1}), "
                              f"whole encode by the reference CPU encoder, one run",
                    "same_crop_gpu_mpix_s": round(with_crop, 6)}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def crop_gpu_mpix(L, crop, ea):
    """This library's encode of the CPU baseline's crop (resident, median of three after one warm-up)."""
    per_site = (C.c_double * len(crop.per_site))(*crop.per_site)
    chain = [np.ascontiguousarray(c, np.float32).ravel() for c in crop.chain]
    model = abi.make_model(crop)
    h = C.c_void_p()
    check(L.nntc_b200_device_create(C.byref(model), abi.float_ptrs(chain), C.byref(h)), "device_create")
    ms = []
    for i in range(4):
        r = abi.EncodeResult()
        m = abi.make_model(crop)
        check(L.nntc_b200_encode_on_device(h, C.byref(m), C.byref(ea), per_site, C.byref(r), None, None, None, None),
              "encode")
        if i:
            ms.append(r.ms_total)
    L.nntc_b200_device_destroy(h)
    return crop.width * crop.height / 1e6 / (statistics.median(ms) / 1000.0)


# DRAM bytes (read + write) per launch of each timed kernel group, per level-0 pixel of the chain, from ncu captures
# (one launch of each kernel, its sections and dram__bytes_{read,write}.sum) of the 4 x 2048 x 1024 material (2796160
# level-0 pixels); a launch's traffic grows with the pixels it covers, so the bench scales these to its own workload.
# A group of two kernels (the assembly: site terms, then the gather) adds both. Per form: the two forms run different
# kernels for most groups.
_PIX3 = 2796160
TRAFFIC_PER_UNIT = {
    "adjoint": {
        "normal_equations": (723597056 + 8700928) / _PIX3,                    # k_ls_accumulate_tc<12>
        "objective": (718641152 + 4395008) / _PIX3,                           # k_objective_f32<12>
        "assemble_level0": (718829056 + 627887616 + 671188992 + 944002048) / _PIX3,
        "assemble_level1": (718788608 + 627927552 + 885506560 + 71808000) / _PIX3,
        "quant_sweep": (610947328 + 42693888) / _PIX3,                        # a level-0 colour launch
        "bc_refine": (1279862000 + 43057664) / _PIX3,                         # one colour
    },
    "plain": {
        "normal_equations": (722979328 + 8198656) / _PIX3,                    # k_ls_accumulate_mma<12>
        "objective": (1255526000 + 4267264) / _PIX3,                          # k_objective_p<12>
        "assemble_level0": (718652928 + 626347520 + 671268096 + 1827433000) / _PIX3,
        "quant_sweep": (1030932000 + 46642944) / _PIX3,
        "bc_refine": (1279862000 + 43057664) / _PIX3,
    },
}

# What bounds each group, from the same captures: the roofline the HBM fraction alone does not show.
BINDING = {
    "adjoint": {
        "assemble_level0": "issue: the fused FP32 site terms at ~88% issue; the gather's L2 latency (one visit ahead)",
        "assemble_level1": "issue: the fused FP32 site terms at ~88% issue; the gather at ~50% issue (cp.async ring)",
        "objective": "issue: FP32 decode with fused multiply-adds, ~72% issue, FP32 pipe ~36%",
        "normal_equations": "latency of the site rows' loads at 16 warps per SM; the tensor pipe (tcgen05) ~14% busy",
        "bc_refine": "latency: the set-up (block-major stencil copy, coalesced), then the ordered selector steps",
        "quant_sweep": "HBM (FP32 per-block stencil, a level-0 colour at ~67% of the copy bandwidth)",
        "cg_product_level0": "HBM (FP32 stencil)",
        "cg_product_level1": "DRAM latency (small launches)",
    },
    "plain": {
        "assemble_level0": "FP32/ALU issue (site terms, the reference's unfused arithmetic) and FP64 issue plus stencil "
                           "stores (gather)",
        "assemble_level1": "FP32/ALU issue (site terms) and L2 latency (gather)",
        "objective": "FP64 pipe (~50% of peak)",
        "normal_equations": "the FP64 tensor pipe (mma.sync m8n8k4, ~76% busy)",
        "bc_refine": "latency: the set-up (block-major stencil copy, coalesced), then the ordered selector steps",
        "quant_sweep": "HBM (FP64 stencil, a level-0 colour at ~78% of the copy bandwidth)",
        "cg_product_level0": "HBM (FP64 stencil)",
        "cg_product_level1": "DRAM latency (small launches)",
    },
}


def roofline(name, stat, mat, hbm, tf, src, form):
    """The dominant kernel against the HBM roofline: its algorithmic bytes per launch over its mean launch time."""
    launches, ms = stat
    if launches == 0:
        return None
    per = algorithmic_bytes(name, mat, form)
    achieved = per / (ms / launches / 1000.0) / 1e9
    t0 = sum(p[0] * p[1] for p in mat.planes)
    unit = TRAFFIC_PER_UNIT[form].get(name)
    traffic = round(unit * t0) if unit else None
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "traffic": traffic, "peak_source": src,
            "traffic_source": "ncu DRAM bytes of the 4x2048x1024 workload scaled by level-0 pixels" if traffic
            else "no ncu DRAM figure recorded for this group's current kernels",
            "binding": BINDING[form].get(name), "bytes_per_launch": per, "launches": launches,
            "ms_per_launch": round(ms / launches, 4)}


def algorithmic_flops(name, mat):
    """Floating-point operations a launch of a pipe-bound group does (every plane of the chain), where they are the
    work that matters: the objective's per-site sampling, decode and squared residuals."""
    c0, c1, nout, k = mat.c0, mat.c1, 3 * len(mat.textures), mat.k
    nin = c1 + c0 + c0 * c1
    t0 = sum(p[0] * p[1] for p in mat.planes)
    if name == "objective":
        per_site = 2 * nout * nin + c0 * c1 + 5 * nout
        return t0 * ((1 + k) * per_site + 8 * c1 * (1 + k) + 8 * c0 * k)
    return 0


def algorithmic_bytes(name, mat, form):
    """Bytes a launch must read and write at least (every plane of the chain): its inputs once and its outputs once.
    The stencil is FP64 in the plain form, FP32 in the adjoint form; the targets are the centre sites' source and the
    fractional sites' cached float targets."""
    c0, c1, nout, k = mat.c0, mat.c1, 3 * len(mat.textures), mat.k
    t0 = sum(p[0] * p[1] for p in mat.planes)
    t1 = sum(p[2] * p[3] for p in mat.planes)
    sb = 4 if form == "adjoint" else 8   # bytes per stencil entry
    targets = 4 * nout * (1 + k)
    if name == "assemble_level0":   # reads the targets, v0 and v1, writes the stencil and the gradient
        return t0 * (targets + 4 * c0 + 5 * c0 * c0 * sb + 8 * c0) + t1 * 4 * c1
    if name == "assemble_level1":
        return t0 * (targets + 4 * c0) + t1 * (4 * c1 + 5 * c1 * c1 * sb + 8 * c1)
    if name == "objective" or name == "normal_equations":
        return t0 * (targets + 4 * c0) + t1 * 4 * c1
    if name == "cg_product_level0":   # the stencil's 5 blocks + x in + y out per level-0 texel
        return t0 * (5 * c0 * c0 * sb + 3 * 8 * c0)
    if name == "cg_product_level1":
        return t1 * (5 * c1 * c1 * sb + 3 * 8 * c1)
    if name == "quant_sweep":   # one colour: a quarter of the texels, their 5 own blocks, gradient and state
        return max(t0 * (5 * c0 * c0 * sb + 2 * 8 * c0 + 9 * c0) // 4, t1 * (5 * c1 * c1 * sb) // 4)
    if name == "bc_refine":   # one colour: a quarter of the blocks read their FP64 stencil, grad, planes
        return t0 * (5 * c0 * c0 * 8 + 8 * c0 + 4 * c0 + 4 * c0 + 8 * c0) // 4
    return 0


if __name__ == "__main__":
    sys.exit(main())
