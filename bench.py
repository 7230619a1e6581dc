"""Benchmark: Gpairs/s of the shear-scalar (xi_t) pair sums at 10M objects.

Workload (the tomography workload of synth.py, number 5): 5 shear bins of
0.2/0.5/1.0/1.9/4.0 M sources x 5 scalar bins of 0.1/0.2/0.4/0.7/1.0 M lenses,
10.0 M objects on a 1000 deg^2 flat patch (clustered: Gaussian blobs on a
Poisson background), 25 cross-correlations in one persistent launch, 20 log
bins from 1 to 300 arcmin, 100 lens patches (per-patch sums for the
bootstrap).  Synthetic, seeded (numpy PCG64, seed 1005).

One step = one tpcf_batch_shear_scalar call: grid and lens-group build on the
device, the pair kernel over all 25 tasks, the per-patch reduction, outputs.
``value`` uses inputs resident in HBM; ``e2e`` the same call with pinned host
inputs (H2D copies and the result D2H inside the timed region).  Times are CUDA
events on the stream the library launches on; for N > 1 ranks the work items
are sharded (no data-path collective except one all-reduce of the per-patch
sums) and the time is the max over ranks.

--impl reference times the reference algorithm's CPU path (the FP32 OpenMP
restatement of tangential_shear_tpcf with its kd-tree, oracle/) on the host
cores on a bounded lens sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpairs/s for xi_t at 10M objects, plain vs batched+adjoint form at 1e-6 rel. error"
UNIT = "Gpairs/s"
FLOP_PER_PAIR = 26  # shear-scalar, FMA = 2, MUFU = 1 (per binned pair)
# DRAM bytes read + written by one pair-kernel launch of the default workload,
# per grid cell side theta_max/D (one-pass ncu captures of
# dram__bytes_read.sum + dram__bytes_write.sum)
K_PAIRS_DRAM_BYTES = {16: 69.567e9 + 0.403e9, 24: 68.311e9 + 0.409e9, 32: 65.525e9 + 0.403e9}
SPH_FLOP_PER_PAIR = 52  # spherical shear-scalar: hi/lo unit-vector differences, east/north projection, angle series
WORKLOAD_DESC = ("tomography: 5 shear bins (0.2,0.5,1.0,1.9,4.0 M) x 5 scalar bins "
                 "(0.1,0.2,0.4,0.7,1.0 M) = 10.0 M objects, 25 cross-pairs in one launch, "
                 "20 log bins 1-300 arcmin, 1000 deg^2 clustered, 100 lens patches")


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def window(self, t0, t1):
        """Restrict the summary to samples taken between wall times t0 and t1."""
        self.t0, self.t1 = t0, t1

    def summary(self):
        import datetime
        sm, mx, reasons = [], None, set()
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(p[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                if hasattr(self, "t0") and not (self.t0 - 0.3 <= ts <= self.t1 + 0.3):
                    continue
            except ValueError:
                pass
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"),
                               p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- workload --
def workload(scale):
    synth = importlib.import_module("2pcf_b200.synth")
    return synth.make_workload(5, scale=scale)


def cpu_baseline(w, seconds, nthreads, steps=1, warmup=0):
    """Reference algorithm (FP32 restatement + kd-tree, OpenMP) on a lens sample:
    every k-th lens of each scalar bin, concatenated, against each full shear
    bin (the 25 task pairs).  Rate = binned pairs / pair-loop seconds (tree
    builds excluded, which favours the CPU).  k is calibrated so one step takes
    about ``seconds`` of pair-loop time."""
    from oracle import oracle as O
    lo, hi, nb = w["bins"]
    lenses, shapes = w["lens_bins"], w["shape_bins"]

    def sample(stride):
        return {k: np.concatenate([L[k][::stride] for L in lenses]) for k in ("x", "y", "z", "val", "w")}

    def run(stride):
        Ls = sample(stride)
        pairs, loop = 0, 0.0
        for S in shapes:
            r = O.ref_pairs(O.SHEAR, Ls, S, lo, hi, nb, num_threads=nthreads)
            pairs += int(r["n_pairs"].sum())
            loop += O.last_timing()[1]
        return pairs, loop, len(Ls["x"])

    cal = 20000 if nthreads >= 4 else 200000     # calibration (~120 / ~12 lenses)
    p0, t0, _ = run(cal)
    rate = p0 / max(t0, 1e-6)
    pairs_per_lens = p0 / len(sample(cal)["x"])
    n_tot = sum(len(L["x"]) for L in lenses)
    want = max(1.0, seconds * rate / pairs_per_lens)
    stride = max(1, int(n_tot / want))
    for _ in range(warmup):
        run(stride * 10)
    tot_p, tot_t, nl = 0, 0.0, 0
    for _ in range(steps):
        p, t, nl = run(stride)
        tot_p += p
        tot_t += t
    return {"value": tot_p / tot_t / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"every {stride}-th lens of each scalar bin ({nl} lenses) against all "
                      f"{sum(len(S['x']) for S in shapes) / 1e6:.1f} M sources, all 25 tasks; {tot_p:.3e} binned pairs; rate over the OpenMP pair "
                      f"loop ({tot_t:.1f} s), kd-tree builds excluded",
            "seconds": tot_t}


def adjoint_timing(w, ctx, bins, pairs, pair_ms, stream, peak):
    """The batched + adjoint form: xi_t and xi_x of all 25 tasks from one
    differentiable forward launch (raw per-lens sums kept on the device), a
    chi^2 against a seeded target, and the backward (one batched adjoint
    launch over all tasks), against the plain batched forward.  One untimed
    pass first."""
    import torch
    ag = importlib.import_module("2pcf_b200.autograd")
    d = lambda a: torch.from_numpy(a).cuda()
    geo_L = [dict(x=d(L["x"]), y=d(L["y"]), z=d(L["z"])) for L in w["lens_bins"]]
    geo_S = [dict(x=d(S["x"]), y=d(S["y"]), z=d(S["z"]), m=d(S["m"])) for S in w["shape_bins"]]
    target = torch.from_numpy(np.random.default_rng(1004).normal(0, 1e-4, (len(w["tasks"]), bins.n_bin))).cuda()
    t_fwd = t_all = 0.0
    for rep in range(2):
        leaves = ([d(L["val"]).requires_grad_(True) for L in w["lens_bins"]],
                  [d(L["w"]).requires_grad_(True) for L in w["lens_bins"]],
                  [d(S["e1"]).requires_grad_(True) for S in w["shape_bins"]],
                  [d(S["e2"]).requires_grad_(True) for S in w["shape_bins"]],
                  [d(S["w"]).requires_grad_(True) for S in w["shape_bins"]])
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        xi_t, _ = ag.xi_shear_batch(w["tasks"], geo_L, geo_S, *leaves, bins, ctx)
        e1.record(stream)
        loss = (((xi_t - target) / 1e-3) ** 2).sum()
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        t_fwd, t_all = e0.elapsed_time(e1), e0.elapsed_time(e2)
        adj_ms = ctx.stats()["pair_kernel_ms"]   # the adjoint kernel of the backward launch
        del leaves, xi_t, loss
    ach = pairs * ADJ_FLOP_PER_PAIR / (adj_ms * 1e-3) / 1e12
    return {"value": pairs / (t_all * 1e-3) / 1e9, "unit": UNIT,
            "forward_ms": t_fwd, "forward_plus_adjoint_ms": t_all,
            "fwd_adj_over_plain_fwd": t_all / pair_ms,
            "fwd_adj_over_fwd": t_all / t_fwd,
            "adjoint_roofline": {"bound": "fp32", "achieved": ach, "peak": peak, "unit": "TFLOP/s",
                                 "frac": ach / peak, "kernel": "k_adj", "kernel_ms": adj_ms,
                                 "flop_per_pair": ADJ_FLOP_PER_PAIR},
            "note": "25 tasks in one differentiable forward launch (raw per-lens sums kept on the device) and "
                    "one backward launch (tpcf_batch_shear_scalar_adjoint); plain forward = the pair kernel of "
                    "the batched step"}


def sky_patch(x, y, box, lam0_deg=40.0, phi0_deg=-30.0):
    """Flat arcmin coordinates of a box of side ``box`` mapped onto a sky
    patch centred at (lam0, phi0): latitude offset = y, longitude offset =
    x / cos(latitude) (radians, FP32)."""
    d2r = np.pi / 180.0
    phi = phi0_deg * d2r + (np.asarray(y, np.float64) - box / 2) / 60.0 * d2r
    lam = lam0_deg * d2r + (np.asarray(x, np.float64) - box / 2) / 60.0 * d2r / np.cos(phi)
    return lam.astype(np.float32), phi.astype(np.float32)


def marks_timing(tpcf, stream, nb):
    """xi from precomputed marks for 16 maps over 1.0 M lenses (HBM roofline
    on the algorithmic bytes) and a 1000-resample marks bootstrap (FP64 FMA
    roofline); CUDA events on the launch stream, each timed call after an
    untimed one."""
    import torch
    out = {}
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    # xi from marks: 1.0 M lenses x 20 bins, 16 maps
    rng = np.random.default_rng(77)
    n, nbm, n_map = 1_000_000, nb, 16
    mk = tpcf.MarksField(x=dev(rng.normal(size=n).astype(np.float32)), y=dev(rng.normal(size=n).astype(np.float32)),
                         w=dev(rng.uniform(0.5, 1.5, n).astype(np.float32)),
                         xi_E=dev(rng.normal(size=(n, nbm)).astype(np.float32)),
                         xi_B=dev(rng.normal(size=(n, nbm)).astype(np.float32)),
                         K=dev(rng.uniform(0.5, 1.5, (n, nbm)).astype(np.float32)))
    val = dev(rng.normal(size=(n_map, n)).astype(np.float32))
    wm = dev(rng.uniform(0.5, 1.5, (n_map, n)).astype(np.float32))
    mctx = tpcf.Context(0)
    mctx.set_stream(stream.cuda_stream)
    mctx.set_timing(True)  # CUDA events around the partial-sum kernel(s) of each call
    _, ms = timed(lambda: tpcf.calculate_tpcf_from_marks([mk], [val], [wm], ctx=mctx))
    kms = mctx.stats()["pair_kernel_ms"]
    # algorithmic bytes: the marks once (xi_E, xi_B, K [n][n_bin] and the marks
    # weight, FP32) and the maps' val and w [n_map][n] (FP32); 2 FLOP per lens,
    # marks row and map
    byt = (3 * 4 * n * nbm + 4 * n) + n_map * 8 * n
    peaks = load_peaks()
    hbm = peaks.get("hbm_gbs") or 6650.0
    hbm_src = "measured (MEASURED_PEAKS.json)" if peaks.get("hbm_gbs") else \
        "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"
    p64 = mctx.measure_fp64_peak()
    out["marks_reweight"] = {"maps": n_map, "lenses": n, "n_bin": nbm, "call_ms": ms, "kernel_ms": kms,
                             "kernel": "k_marks_dmma (FP64 mma.sync m8n8k4)",
                             "call_hbm_frac": byt / (ms * 1e-3) / 1e9 / hbm,
                             "fp64_frac": n * (3 * nbm + 1) * n_map * 2 / (kms * 1e-3) / 1e12 / p64,
                             "roofline": {"bound": "hbm", "achieved": byt / (kms * 1e-3) / 1e9, "peak": hbm,
                                          "unit": "GB/s", "frac": byt / (kms * 1e-3) / 1e9 / hbm,
                                          "bytes": byt, "peak_source": hbm_src}}
    _, ms = timed(lambda: tpcf.marks_bootstrap([mk], 1000, seed=5, covariance=True, ctx=mctx))
    kms = mctx.stats()["pair_kernel_ms"]
    # each resample re-weights every lens's 3 n_bin + 1 marks: one FP64 FMA
    # each (the multiplicities are drawn on the device), so FP64-bound; the
    # FP64 tensor instruction and the FP64 FMA pipe have the same peak here
    flop = 1000 * n * (3 * nbm + 1) * 2
    # its HBM side: every pass of 16 resamples streams the marks once and the
    # 16 multiplicity rows (INT32 per lens), ceil(1000 / 16) passes
    boot_bytes = -(-1000 // 16) * (3 * 4 * n * nbm + 4 * n) + 1000 * 4 * n
    out["marks_bootstrap"] = {"resamples": 1000, "lenses": n, "call_ms": ms, "kernel_ms": kms,
                              "call_fp64_frac": flop / (ms * 1e-3) / 1e12 / p64,
                              "hbm": {"bytes": boot_bytes, "achieved_gbs": boot_bytes / (kms * 1e-3) / 1e9,
                                      "frac": boot_bytes / (kms * 1e-3) / 1e9 / hbm, "peak_source": hbm_src},
                              "roofline": {"bound": "fp64", "achieved": flop / (kms * 1e-3) / 1e12, "peak": p64,
                                           "unit": "TFLOP/s", "frac": flop / (kms * 1e-3) / 1e12 / p64,
                                           "flop": flop, "peak_source": "FP64 FMA loop measured in this run"}}
    del mk, val, wm
    mctx.close()
    return out


def widened_timing(tpcf, w, peak_fp32, stream, cpu_threads, with_cpu=True):
    """Measurements of the rows around the pair sum: the spherical pair sum on
    the tomography catalogues projected onto a sky patch, xi from precomputed
    marks for 16 maps, a 1000-resample bootstrap of marks, the equal-weight
    k-means, and the text catalogue reader.  CUDA events on the launch stream;
    each timed call follows an untimed one."""
    import tempfile
    import torch
    out = {}
    d2r = np.pi / 180.0
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1)

    # the same 25 planar tasks with redshifts that make the z cut bite
    # (lens z ~ U(0, 1), source z ~ U(0.3, 1.5): ~19% of the pairs are dropped)
    rz = np.random.default_rng(9)
    Lz = [tpcf.LensCatalog(x=dev(l["x"]), y=dev(l["y"]), val=dev(l["val"]), w=dev(l["w"]),
                           z=dev(rz.uniform(0, 1, len(l["x"])).astype(np.float32))) for l in w["lens_bins"]]
    Sz = [tpcf.ShapeCatalog(x=dev(s_["x"]), y=dev(s_["y"]), e1=dev(s_["e1"]), e2=dev(s_["e2"]), w=dev(s_["w"]),
                            z=dev(rz.uniform(0.3, 1.5, len(s_["x"])).astype(np.float32)), m=dev(s_["m"]))
          for s_ in w["shape_bins"]]
    zbins = tpcf.create_bins(*w["bins"])
    zctx = tpcf.Context(0)
    zctx.set_timing(True)
    zctx.set_stream(stream.cuda_stream)
    zctx.set_cell_size(zbins.x_max / 64)
    outs, ms = timed(lambda: tpcf.batch_shear_2pcf(Lz, Sz, w["tasks"], zbins, ctx=zctx))
    zp = sum(int(o.n_pairs.sum()) for o in outs)
    out["z_cut"] = {"value": zp / (ms * 1e-3) / 1e9, "unit": UNIT, "binned_pairs": zp, "call_ms": ms,
                    "kernel_ms": zctx.stats()["pair_kernel_ms"]}
    zctx.close()
    del Lz, Sz

    # spherical pair sum: the 25 tomography tasks on a 31.6 x 31.6 deg patch at
    # Dec -30 (flat arcmin coordinates mapped to longitude / latitude)
    def sph(c):
        return sky_patch(c["x"], c["y"], w["box"])

    Ls, Ss = [], []
    for l in w["lens_bins"]:
        lam, phi = sph(l)
        Ls.append(tpcf.LensCatalog(x=dev(lam), y=dev(phi), val=dev(l["val"]), w=dev(l["w"]), z=dev(l["z"])))
    for s_ in w["shape_bins"]:
        lam, phi = sph(s_)
        Ss.append(tpcf.ShapeCatalog(x=dev(lam), y=dev(phi), e1=dev(s_["e1"]), e2=dev(s_["e2"]), w=dev(s_["w"]),
                                    z=dev(s_["z"]), m=dev(s_["m"])))
    lo, hi, nb = w["bins"]
    sbins = tpcf.create_bins(lo / 60 * d2r, hi / 60 * d2r, nb)
    sctx = tpcf.Context(0)
    sctx.set_timing(True)
    sctx.set_stream(stream.cuda_stream)
    sctx.set_cell_size(sbins.x_max / 64)
    outs, ms = timed(lambda: tpcf.batch_shear_2pcf(Ls, Ss, w["tasks"], sbins, spherical_coords=True, ctx=sctx))
    pairs = sum(int(o.n_pairs.sum()) for o in outs)
    kms = sctx.stats()["pair_kernel_ms"]
    ach = pairs * SPH_FLOP_PER_PAIR / (kms * 1e-3) / 1e12
    out["sphere"] = {"value": pairs / (ms * 1e-3) / 1e9, "unit": UNIT, "binned_pairs": pairs, "call_ms": ms,
                     "roofline": {"bound": "fp32", "achieved": ach, "peak": peak_fp32, "unit": "TFLOP/s",
                                  "frac": ach / peak_fp32, "kernel": "k_pairs_sph",
                                  "flop_per_pair": SPH_FLOP_PER_PAIR, "kernel_ms": kms}}
    if with_cpu:
        from oracle import oracle as O
        Lh = {k: np.ascontiguousarray(v.cpu().numpy()[::2000]) for k, v in vars(Ls[4]).items()}
        Sh = {k: np.ascontiguousarray(v.cpu().numpy()) for k, v in vars(Ss[2]).items()}
        t0 = time.time()
        r = O.ref_sphere_f32(O.SHEAR, Lh, Sh, sbins.x_min, sbins.x_max, nb, num_threads=cpu_threads)
        dt = time.time() - t0
        out["sphere"]["cpu_baseline"] = {
            "value": int(r["n_pairs"].sum()) / dt / 1e9, "unit": UNIT, "cores": cpu_threads, "kind": "port",
            "sample": f"every 2000-th lens of scalar bin 5 ({len(Lh['x'])}) against shear bin 3 "
                      f"({len(Sh['x'])}), the reference's spherical loop (acos, all pairs) in FP32"}
    sctx.close()
    del Ls, Ss

    out.update(marks_timing(tpcf, stream, nb))

    # equal-weight k-means on all lens positions, 100 blocks
    ux = np.concatenate([l["x"] for l in w["lens_bins"]])
    uy = np.concatenate([l["y"] for l in w["lens_bins"]])
    uw = np.concatenate([l["w"] for l in w["lens_bins"]])
    uw = (0.01 + uw / uw.max()).astype(np.float32)
    U = [dev(a) for a in (ux, uy, uw)]
    mctx = tpcf.Context(0)
    mctx.set_stream(stream.cuda_stream)
    (lab, _, it, devw), ms = timed(lambda: tpcf.partition_data_equal(U[0], U[1], U[2], 100, seed=3, ctx=mctx))
    out["kmeans_equal"] = {"points": int(len(ux)), "k": 100, "iterations": it, "max_weight_deviation": devw,
                           "call_ms": ms}
    mctx.close()

    # text catalogue: 0.5 M shape rows
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "shapes.txt")
        S0 = w["shape_bins"][3]
        m = 500_000
        np.savetxt(path, np.stack([S0[k][:m] for k in ("x", "y", "z", "e1", "e2", "w", "m")], 1), fmt="%.8g")
        size = os.path.getsize(path)
        t0 = time.time()
        tpcf.load_standard_shape_catalog(path)
        dt = time.time() - t0
        out["text_reader"] = {"rows": m, "bytes": size, "seconds": dt, "MB_per_s": size / dt / 1e6,
                              "threads": host_threads()}
    return out


# ------------------------------------------------------- configurations 1-4 --
CONFIG_WORKLOADS = {
    1: "config 1: shear-scalar + scalar-scalar, 20k x 20k uniform on 600' x 600', 15 log bins 1-100'",
    2: "config 2: scalar-scalar auto-correlation, 1.0 M points on 600' x 600' (Gaussian random kappa, "
       "P(k) ~ k^-1.5), w ~ U(0.5, 1.5), 30 log bins 0.5-250'",
    3: "config 3: shear-scalar with errors, 2.0 M shear x 0.5 M scalar on 1200' x 1200', clustered, "
       "100 k-means patches, 1000 resamples, 20 log bins 1-200'",
    4: "config 4: differentiable xi_t on the clustered 2.0 M x 0.5 M catalogues, chi^2 against a seeded "
       "target, forward + adjoint (torch.autograd, device tensors)",
}
ADJ_FLOP_PER_PAIR = 20   # adjoint of a loss on xi_t, per binned pair (sources as owners)
KAPPA_FLOP_PER_PAIR = 14


def cpu_rate(mode, L, S, bins, seconds, nthreads, full=False):
    """The FP32 OpenMP restatement of the reference loop (kd-tree) on every
    k-th lens (k calibrated to about ``seconds`` of pair loop; all lenses when
    ``full``) against all sources: binned pairs per second of pair loop."""
    from oracle import oracle as O
    lo, hi, nb = bins

    def run(stride):
        Ls = {k: np.ascontiguousarray(v[::stride]) for k, v in L.items()}
        r = O.ref_pairs(mode, Ls, S, lo, hi, nb, num_threads=nthreads)
        return int(r["n_pairs"].sum()), O.last_timing()[1], len(Ls["x"])

    n = len(L["x"])
    stride = 1
    if not full:
        cal = max(1, n // (200 if nthreads >= 4 else 20))
        p0, t0, n0 = run(cal)
        per_lens_s = t0 / max(n0, 1)
        stride = max(1, int(n / max(1.0, seconds / max(per_lens_s, 1e-9))))
    p, t, nl = run(stride)
    return {"value": p / max(t, 1e-9) / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": (f"all {nl} lenses" if stride == 1 else f"every {stride}-th lens ({nl})") +
                      f" against all {len(S['x'])} sources; {p:.3e} binned pairs; rate over the OpenMP pair loop "
                      f"({t:.1f} s), kd-tree build excluded"}


def config_timing(k, tpcf, stream, peak, steps=3, warmup=2, with_cpu=True, cpu_seconds=8.0):
    """One configuration of the benchmark suite at its stated size: `value` =
    binned pairs per second of the whole step with inputs in HBM, `e2e` the same
    step through the public API from pinned host arrays, the pair kernel's
    roofline, the autotuned cell side and tile shape, and the CPU port on all
    host threads and on one."""
    import torch
    synth = importlib.import_module("2pcf_b200.synth")
    at = importlib.import_module("2pcf_b200.autotune")
    w = synth.make_workload(k)
    bins = tpcf.create_bins(*w["bins"])
    ctx = tpcf.Context(0)
    ctx.set_timing(True)
    ctx.set_stream(stream.cuda_stream)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    L = w["lenses"]
    S = w.get("shapes")
    K = w.get("kappa_map")
    lens_cat = [tpcf.LensCatalog(**{q: L[q] for q in ("x", "y", "val", "w", "z")})]
    if k == 2:   # the kappa map is the lens catalogue itself (auto-correlation)
        tune_src = [tpcf.ShapeCatalog(x=K["x"], y=K["y"], e1=K["kappa_E"], e2=K["kappa_B"], w=K["w"],
                                      z=np.ones_like(K["x"]), m=np.zeros_like(K["x"]))]
    else:
        tune_src = [tpcf.ShapeCatalog(**{q: S[q] for q in ("x", "y", "e1", "e2", "w", "z", "m")})]
    tune = at.autotune(lens_cat, tune_src, [(0, 0)], bins, ctx, corner=1.0 if k == 1 else 0.5)
    n_patch = w.get("n_patch", 100)
    wt = (0.01 + L["w"] / L["w"].max()).astype(np.float32)
    kernel_ms, flops, adj_ms = [0.0], [0.0], [0.0]
    state = {}

    def shear(A, B, **kw):
        return tpcf.tangential_shear_tpcf(A["x"], A["y"], A["z"], A["val"], A["w"], B["x"], B["y"], B["z"],
                                          B["e1"], B["e2"], B["w"], B["m"], bins, calculate_marks=False,
                                          ctx=ctx, **kw)

    def kappa(A, B):
        return tpcf.scalar_kappa_tpcf(A["x"], A["y"], A["val"], A["w"], B["x"], B["y"], B["kappa_E"],
                                      B["kappa_B"], B["w"], bins, calculate_marks=False, ctx=ctx)

    def step(A, B, C, U):
        kernel_ms[0] = flops[0] = adj_ms[0] = 0.0
        if k == 1:
            r1 = shear(A, B)
            k1 = ctx.stats()["pair_kernel_ms"]
            r2 = kappa(A, C)
            k2 = ctx.stats()["pair_kernel_ms"]
            p1, p2 = int(r1.n_pairs.sum()), int(r2.n_pairs.sum())
            kernel_ms[0], flops[0] = k1 + k2, p1 * FLOP_PER_PAIR + p2 * KAPPA_FLOP_PER_PAIR
            return p1 + p2
        if k == 2:
            r = kappa(A, C)
            p = int(r.n_pairs.sum())
            kernel_ms[0], flops[0] = ctx.stats()["pair_kernel_ms"], p * KAPPA_FLOP_PER_PAIR
            return p
        if k == 3:
            lab, _, _ = tpcf.partition_data(U[0], U[1], U[2], n_patch, ctx=ctx)
            r = shear(A, B, patch_A=lab, n_patch=n_patch)
            p = int(r.n_pairs.sum())
            kernel_ms[0], flops[0] = ctx.stats()["pair_kernel_ms"], p * FLOP_PER_PAIR
            tpcf.block_bootstrap(r.patch_sums, w["n_boot"], seed=1003, ctx=ctx)
            return p
        # k == 4: the differentiable form (torch.autograd on device tensors: the
        # raw per-lens sums stay in device memory), chi^2 against a seeded
        # target, backward through the adjoint; the loss is read back
        ag = importlib.import_module("2pcf_b200.autograd")
        cu = lambda t: t if t.is_cuda else t.cuda(non_blocking=True)
        g = {q: cu(t) for q, t in A.items()}
        h = {q: cu(t) for q, t in B.items()}
        geo = dict(x_A=g["x"], y_A=g["y"], z_A=g["z"], x_B=h["x"], y_B=h["y"], z_B=h["z"], m_B=h["m"])
        leaves = [t.detach().requires_grad_(True) for t in (g["val"], g["w"], h["e1"], h["e2"], h["w"])]
        xi_t, _ = ag.xi_shear(*leaves, geo, bins, ctx)
        kernel_ms[0], flops[0] = ctx.stats()["pair_kernel_ms"], state["pairs"] * FLOP_PER_PAIR
        if state.get("forward_only"):
            xi_t.sum().item()
            return state["pairs"]
        loss = (((xi_t - state["target"]) / state["sig"]) ** 2).sum()
        loss.backward()
        adj_ms[0] = ctx.stats()["pair_kernel_ms"]
        loss.item()
        return state["pairs"]

    def cats(to):
        A = {q: to(v) for q, v in L.items()}
        B = {q: to(v) for q, v in S.items()} if S is not None else None
        C = {q: to(v) for q, v in K.items()} if K is not None else None
        U = [to(L["x"]), to(L["y"]), to(wt)]
        return A, B, C, U

    def timed(A, B, C, U, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kms = fl = ams = 0.0
        e0.record(stream)
        for _ in range(n):
            pairs = step(A, B, C, U)
            kms += kernel_ms[0]
            fl += flops[0]
            ams += adj_ms[0]
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, pairs, kms / n, fl / n, ams / n

    Ad, Bd, Cd, Ud = cats(dev)
    if k == 4:  # binned pairs and the seeded target, from one plain forward call
        r = shear(Ad, Bd)
        state["pairs"] = int(r.n_pairs.sum())
        xi = r.sum_gt / r.sum_K
        sig = np.abs(xi) * 0.1 + 1e-6
        state["sig"] = torch.from_numpy(sig).cuda()
        state["target"] = torch.from_numpy(np.random.default_rng(1004).normal(xi, sig)).cuda()
    for _ in range(warmup):
        step(Ad, Bd, Cd, Ud)
    ms, pairs, kms, fl, ams = timed(Ad, Bd, Cd, Ud, steps)
    Ah, Bh, Ch, Uh = cats(pin)
    step(Ah, Bh, Ch, Uh)
    ms_e2e, pairs_e2e, _, _, _ = timed(Ah, Bh, Ch, Uh, steps)
    h2d = sum(int(t.numel()) * t.element_size() for d in (Ah, Bh, Ch) if d for t in d.values())
    if k == 3:
        h2d += sum(int(t.numel()) * t.element_size() for t in Uh)
    ach = fl / (kms * 1e-3) / 1e12
    out = {"workload": CONFIG_WORKLOADS[k], "value": pairs / (ms * 1e-3) / 1e9, "unit": UNIT,
           "ms_per_step": ms, "steps": steps, "warmup": warmup, "binned_pairs": pairs,
           "e2e": {"value": pairs_e2e / (ms_e2e * 1e-3) / 1e9, "unit": UNIT, "ms_per_step": ms_e2e,
                   "h2d_bytes_per_step": int(h2d)},
           "roofline": {"bound": "fp32", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                        "kernel": "k_pairs", "kernel_ms": kms,
                        "flop_per_pair": KAPPA_FLOP_PER_PAIR if k == 2 else
                        ("26 shear, 14 scalar" if k == 1 else FLOP_PER_PAIR)},
           "autotune_ms_per_gpair": {"cell": {f"theta_max/{d}": round(v, 3) for d, v in tune["cell"].items()},
                                     "tile": {g: round(v, 3) for g, v in tune["tile"].items()},
                                     "choice": tune["choice"]}}
    if k == 4:
        state["forward_only"] = True
        fwd_ms, _, _, _, _ = timed(Ad, Bd, Cd, Ud, steps)
        state["forward_only"] = False
        adj_ach = pairs * ADJ_FLOP_PER_PAIR / (ams * 1e-3) / 1e12
        out["forward_plus_adjoint_over_forward"] = ms / max(fwd_ms, 1e-9)
        out["adjoint_roofline"] = {"bound": "fp32", "achieved": adj_ach, "peak": peak, "unit": "TFLOP/s",
                                   "frac": adj_ach / peak, "kernel": "k_adj", "kernel_ms": ams,
                                   "flop_per_pair": ADJ_FLOP_PER_PAIR}
        out["forward_value"] = pairs / (fwd_ms * 1e-3) / 1e9
    if with_cpu:
        cw = w["bins"]
        nt = host_threads()
        if k == 1:
            parts = [cpu_rate(O_SHEAR, L, S, cw, cpu_seconds, nt, full=True),
                     cpu_rate(O_KAPPA, L, K, cw, cpu_seconds, nt, full=True)]
            one = [cpu_rate(O_SHEAR, L, S, cw, cpu_seconds, 1, full=True)]
        elif k == 2:
            parts = [cpu_rate(O_KAPPA, L, K, cw, cpu_seconds, nt)]
            one = [cpu_rate(O_KAPPA, L, K, cw, cpu_seconds / 2, 1)]
        else:
            parts = [cpu_rate(O_SHEAR, L, S, cw, cpu_seconds, nt)]
            one = [cpu_rate(O_SHEAR, L, S, cw, cpu_seconds / 2, 1)]
        cb = dict(parts[0])
        if len(parts) > 1:
            cb["value"] = float(np.mean([c["value"] for c in parts]))
            cb["sample"] = "shear-scalar: " + parts[0]["sample"] + "; scalar-scalar: " + parts[1]["sample"] + \
                           "; value = mean of the two rates"
        cb["single_thread"] = {q: one[0][q] for q in ("value", "unit", "cores", "sample")}
        out["cpu_baseline"] = cb
        out["speedup_vs_cpu_all_threads"] = out["value"] / cb["value"]
    ctx.close()
    return out


O_SHEAR, O_KAPPA = 0, 1   # oracle modes (oracle.SHEAR, oracle.KAPPA)


def path_stats(tpcf, args):
    """One batched call on the diagnostic build; prints the share of warp
    sub-chunks and lane-pairs per path of k_pairs."""
    import ctypes as C
    import torch
    tpcf._lib.LIB_PATH = os.path.join(ROOT, "2pcf_b200", "libtpcf_b200_stats.so")
    if not os.path.exists(tpcf._lib.LIB_PATH):
        raise SystemExit("--path-stats needs the diagnostic build: make -C 2pcf_b200/csrc stats")
    w = workload(args.scale)
    bins = tpcf.create_bins(*w["bins"])
    dev = lambda a: torch.from_numpy(a).cuda()
    L = [tpcf.LensCatalog(**{k: dev(l[k]) for k in ("x", "y", "val", "w", "z")}) for l in w["lens_bins"]]
    S = [tpcf.ShapeCatalog(**{k: dev(s[k]) for k in ("x", "y", "e1", "e2", "w", "z", "m")})
         for s in w["shape_bins"]]
    ctx = tpcf.Context(0)
    ctx.set_cell_size(bins.x_max / (args.cell_divisor or 64))
    lib = tpcf._lib.lib()
    st = (C.c_ulonglong * 15)()
    lib.tpcf_debug_mode_stats(st)
    base = np.array(st[:])
    outs = tpcf.batch_shear_2pcf(L, S, w["tasks"], bins, ctx=ctx)
    lib.tpcf_debug_mode_stats(st)
    v = np.array(st[:]) - base
    binned = sum(int(o.n_pairs.sum()) for o in outs)
    res = {"binned_pairs": binned}
    names = ("skip", "single_bin", "one_edge", "two_edges", "per_pair")
    for i, name in enumerate(names):
        res[name] = {"warp_chunks": float(v[i] / v[:5].sum()), "lane_pairs": float(v[5 + i] / v[5:10].sum())}
    res["computed_lane_pairs_per_binned_pair"] = float(v[6:10].sum() / binned)
    res["lane_class_of_active_lane_pairs"] = {("out_of_range" if i == 0 else name): float(v[10 + i] / v[10:15].sum())
                                              for i, name in enumerate(names)}
    print(json.dumps(res), flush=True)


def config_line(tpcf, args, rank):
    """`--config N` (1-4): that configuration's measurement as the one JSON line."""
    import torch
    stream = torch.cuda.current_stream()
    ctx = tpcf.Context(0)
    peak = ctx.measure_fp32_peak()
    ctx.close()
    with ClockSampler(0) as cs:
        t0 = time.time()
        r = config_timing(args.config, tpcf, stream, peak, steps=args.steps, warmup=args.warmup,
                          with_cpu=not args.no_cpu_baseline, cpu_seconds=args.cpu_seconds / 2)
        cs.window(t0, time.time())
    line = {"metric": METRIC, "value": r.pop("value"), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r.pop("ms_per_step"), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "accumulate": "f64", "data": "synthetic",
            "config": {"workload": r.pop("workload"), "l2": "no flush between steps"}}
    line.update(r)
    line["clocks"] = cs.summary()
    if rank == 0:
        print(json.dumps(line), flush=True)


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    w = workload(args.scale)
    nt = host_threads()
    per_step = max(2.0, min(20.0, 120.0 / max(1, args.steps)))
    cb = cpu_baseline(w, per_step, nt, steps=args.steps, warmup=args.warmup)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["seconds"] * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD_DESC, "scale": args.scale},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------------- ours --
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="object-count scale of the workload")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the batched+adjoint measurement")
    ap.add_argument("--path-stats", action="store_true",
                    help="diagnostic: load the counting build (make -C 2pcf_b200/csrc stats) and print the "
                         "pair kernel's path mix for one batched call instead of benchmarking")
    ap.add_argument("--region", type=float, default=0.0,
                    help="profiling: keep only objects with x, y < REGION arcmin (density unchanged)")
    ap.add_argument("--task", type=int, default=-1, help="profiling: run only this task of the 25")
    ap.add_argument("--geometry", default="plane", choices=["plane", "sphere"],
                    help="profiling: 'sphere' projects the catalogues onto a sky patch and times the spherical "
                         "pair kernel instead")
    ap.add_argument("--marks-only", action="store_true",
                    help="profiling: only the xi-from-marks and marks-bootstrap measurements, as one JSON line")
    ap.add_argument("--no-widened", action="store_true",
                    help="skip the spherical, marks, bootstrap, k-means and reader measurements")
    ap.add_argument("--cell-divisor", type=int, default=0,
                    help="fix the grid cell side at theta_max/D and the default tile shape instead of running "
                         "the autotuner (2pcf_b200.autotune) once before the warm-up")
    ap.add_argument("--config", type=int, default=5, choices=[1, 2, 3, 4, 5],
                    help="5 (default): the tomography headline; 1-4: only that configuration's line")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the measurements of configurations 1-4 that the default run adds")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    tpcf = importlib.import_module("2pcf_b200")
    if args.path_stats:
        return path_stats(tpcf, args)
    if args.config != 5:
        return config_line(tpcf, args, rank)
    if args.marks_only:
        res = marks_timing(tpcf, torch.cuda.current_stream(), 20)
        if rank == 0:
            print(json.dumps(res), flush=True)
        return 0

    w = workload(args.scale)
    if args.region > 0:
        for cat in w["lens_bins"] + w["shape_bins"]:
            keep = (cat["x"] < args.region) & (cat["y"] < args.region)
            for k in list(cat):
                cat[k] = np.ascontiguousarray(cat[k][keep])
    if args.task >= 0:
        w["tasks"] = [w["tasks"][args.task]]
    sphere = args.geometry == "sphere"
    if sphere:
        for cat in w["lens_bins"] + w["shape_bins"]:
            cat["x"], cat["y"] = sky_patch(cat["x"], cat["y"], w["box"])
        lo, hi, nb_ = w["bins"]
        w["bins"] = (lo / 60.0 * np.pi / 180.0, hi / 60.0 * np.pi / 180.0, nb_)
    bins = tpcf.create_bins(*w["bins"])
    n_patch = w["n_patch"]
    ctx = tpcf.Context(local)
    ctx.set_timing(True)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    # cell side and tile shape picked once by the autotuner (trial calls on a
    # density-preserving corner of the field, before the warm-up), or fixed
    if args.cell_divisor > 0:
        ctx.set_cell_size(bins.x_max / args.cell_divisor)
        tune = None
    else:
        at = importlib.import_module("2pcf_b200.autotune")
        tune = at.autotune(
            [tpcf.LensCatalog(**{k: l[k] for k in ("x", "y", "val", "w", "z")}) for l in w["lens_bins"]],
            [tpcf.ShapeCatalog(**{k: s_[k] for k in ("x", "y", "e1", "e2", "w", "z", "m")})
             for s_ in w["shape_bins"]],
            w["tasks"], bins, ctx, corner=0.4, spherical_coords=sphere)
    if world > 1:
        ctx.set_shard(rank, world)
    n_boot = w["n_boot"]

    def cats(to):
        L = [tpcf.LensCatalog(**{k: to(l[k]) for k in ("x", "y", "val", "w", "z")}) for l in w["lens_bins"]]
        S = [tpcf.ShapeCatalog(**{k: to(s[k]) for k in ("x", "y", "e1", "e2", "w", "z", "m")})
             for s in w["shape_bins"]]
        return L, S

    dev = lambda a: torch.from_numpy(a).cuda()
    pin = lambda a: torch.from_numpy(a).pin_memory()
    Ld, Sd = cats(dev)
    Lh, Sh = cats(pin)
    # k-means input: all lens positions with the reference's weights 0.01 + w/max(w)
    # (src/tpcf.f90:1104), one patch set shared by the 5 scalar bins
    ux = np.concatenate([l["x"] for l in w["lens_bins"]])
    uy = np.concatenate([l["y"] for l in w["lens_bins"]])
    uw = np.concatenate([l["w"] for l in w["lens_bins"]])
    uw = (0.01 + uw / uw.max()).astype(np.float32)
    U_d = [dev(a) for a in (ux, uy, uw)]
    U_h = [pin(a) for a in (ux, uy, uw)]
    offs = np.cumsum([0] + [len(l["x"]) for l in w["lens_bins"]])
    torch.cuda.synchronize()

    ctx_pair_ms = [0.0]

    def step(L, S, U):
        lab, _, _ = tpcf.partition_data(U[0], U[1], U[2], n_patch, ctx=ctx)
        P = [lab[offs[i]:offs[i + 1]] for i in range(len(L))]
        outs = tpcf.batch_shear_2pcf(L, S, w["tasks"], bins, lens_patches=P, n_patch=n_patch,
                                     spherical_coords=sphere, ctx=ctx)
        ctx_pair_ms[0] = ctx.stats()["pair_kernel_ms"]  # the pair kernel's own CUDA-event time
        ps = np.stack([o.patch_sums for o in outs])
        if world > 1:
            t = torch.from_numpy(ps).cuda()
            dist.all_reduce(t)
            ps = t.cpu().numpy()
        boot = tpcf.block_bootstrap(ps, n_boot, seed=1005, ctx=ctx)
        return int(ps[:, :, 5].sum()), boot

    def timed(L, S, U, n):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.kernel_launches
        pair_ms = 0.0
        pairs = 0
        e0.record(stream)
        for _ in range(n):
            pairs, _ = step(L, S, U)
            pair_ms += ctx_pair_ms[0]
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1) / n
        t = torch.tensor([ms], device="cuda")
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.item(), pairs, pair_ms / n, ctx.kernel_launches - l0

    with ClockSampler(local) as cs:  # started before the warm-up: its start-up stays outside the timing
        for _ in range(args.warmup):
            step(Ld, Sd, U_d)
        t0 = time.time()
        ms, pairs, pair_ms, launches = timed(Ld, Sd, U_d, args.steps)
        cs.window(t0, time.time())
    clocks = cs.summary()
    value = pairs / (ms * 1e-3) / 1e9

    # end to end through the public API with pinned host inputs
    step(Lh, Sh, U_h)
    ms_e2e, pairs_e2e, _, _ = timed(Lh, Sh, U_h, args.steps)
    h2d = sum(a.numel() * a.element_size() for c in (Lh + Sh) for a in vars(c).values()
              if hasattr(a, "numel")) + sum(a.numel() * 4 for a in U_h)
    d2h = (int(ux.size) * 4 + len(w["tasks"]) * bins.n_bin * (5 * 8 + 8 + 5 * 4 + n_patch * 6 * 8)
           + 2 * n_boot * len(w["tasks"]) * bins.n_bin * 8 + 2 * (len(w["tasks"]) * bins.n_bin) ** 2 * 8)

    peak = ctx.measure_fp32_peak()
    adjoint = None
    if world == 1 and not args.no_adjoint and not sphere:
        adjoint = adjoint_timing(w, ctx, bins, pairs, pair_ms, stream, peak)
    fpp = SPH_FLOP_PER_PAIR if sphere else FLOP_PER_PAIR
    achieved = pairs * fpp / (pair_ms * 1e-3) / 1e12
    # DRAM bytes of one pair-kernel launch of this exact workload at a captured
    # cell side; other configurations were not captured
    traffic = None
    if not sphere and args.scale == 1.0 and args.region <= 0 and args.task < 0:
        for d, byt in K_PAIRS_DRAM_BYTES.items():
            if abs(ctx.cell_size - bins.x_max / d) < 1e-6:
                traffic = byt

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "accumulate": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD_DESC, "scale": args.scale, "region": args.region, "task": args.task,
                   "global_batch": int(pairs),
                   "parallelism": f"work items sharded over {world} rank(s)" if world > 1 else "single GPU",
                   "l2": "inputs (280 MB of catalogues) larger than L2 (126 MB); no flush",
                   "cell_size": ctx.cell_size,
                   "tile_shape": {"threads_per_block": ctx.tile_shape[0] or 128, "tile_chunks": ctx.tile_shape[1] or 2},
                   "autotune_ms_per_gpair": None if tune is None else {
                       "cell": {f"theta_max/{d}": round(v, 3) for d, v in tune["cell"].items()},
                       "tile": {g: round(v, 3) for g, v in tune["tile"].items()}, "choice": tune["choice"]},
                   "step": "k-means (100 patches, all 2.4 M lens positions) + grid build + one 25-task "
                           "pair launch + per-patch sums + 1000-resample bootstrap with the joint "
                           "500x500 covariance"},
        "e2e": {"value": pairs_e2e / (ms_e2e * 1e-3) / 1e9, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic, "kernel": "k_pairs_sph" if sphere else "k_pairs",
                     "flop_per_pair": fpp, "kernel_ms": pair_ms,
                     "peak_source": "measured in this run: FFMA loop (tpcf_measure_fp32_peak); "
                                    "MEASURED_PEAKS.json has no FP32 figure"},
        "gpu_launches": int(launches),
        "batched_adjoint": adjoint,
        "clocks": clocks,
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline and not sphere:
        cb = cpu_baseline(w, args.cpu_seconds, host_threads())
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        # the same restatement on one host thread (a shorter bounded sample)
        c1 = cpu_baseline(w, min(args.cpu_seconds, 5.0), 1)
        line["cpu_baseline"]["single_thread"] = {k: c1[k] for k in ("value", "unit", "cores", "sample")}
    if world == 1 and not args.no_widened and args.region <= 0 and args.task < 0 and not sphere:
        line["widened"] = widened_timing(tpcf, w, peak, stream, host_threads(), with_cpu=not args.no_cpu_baseline)
    if world == 1 and not args.no_configs and args.region <= 0 and args.task < 0 and not sphere:
        line["configs"] = {str(k): config_timing(k, tpcf, stream, peak, with_cpu=not args.no_cpu_baseline)
                           for k in (1, 2, 3, 4)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
