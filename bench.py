#!/usr/bin/env python
"""Benchmark of the SGT engine: frequency slices per second.

Workload (default, psv2048): the P-SV engine on a synthetic 1-D Earth (solid
inner core, fluid outer core, 6 mantle/crust zones; seeded quadratic
profiles), tlen 3276.8 s, 2048 frequencies (fmax 0.625 Hz, cutoffs up to
about 7000), source 300 km deep, 201 receiver radii 1000-6350 km, 1441
epicentral distances (0.125 deg).  A step is one batch of frequency slices
(20 by default, --per-step) spread across the band, each fully processed
(all orders up to the reference's cutoff, all m, all sources, TSGT + RSGT +
SYNN on the full (r, theta) grid).  psv1024 (the FP64 configuration's
band: 1024 frequencies, 721 distances), sh256, the catalogue consumer, its
per-point kernel formulas (kernels) and the batched models x depths request
are the other workloads.

  python bench.py [--gpus N --steps K --warmup W] [--workload psv2048|psv1024|sh256|catalogue|kernels|batch]
                  [--precision mixed|mixed_bf16|fp64] [--per-step F]
  python bench.py --impl reference ...   # CPU restatement of the reference

The headline path is the mixed-precision one (split fp16 l-sum on the
tensor cores, depth cut-off of the band; learned first order ranges with
--lmax); the plain FP64 GPU path runs the same steps for the speedup, and
the library's own accuracy report (an FP64 context attached to the mixed
one) gives the per-component relative L2 on a sample of frequencies that
includes the top of the band.

One JSON line is printed by rank 0.  Under torchrun (N > 1) every rank
processes its own frequencies (weak scaling, no collective on the data
path); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "dsm-kernel_b200"))
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402

METRIC = "SGT freq-slices/s at rel-L2<=1e-6 vs FP64; speedup over plain FP64 GPU path"
UNIT = "freq-slices/s"


WORKLOADS = {
    # P-SV on the GPU (the FP64 configuration; default)
    "psv1024": dict(mode="psv", tlen=3276.8, imax=1024, thdelta=0.25, rdelta=26.75, rmin=1000.0,
                    rmax=6350.0, r0=6071.0, thetas=721),
    # its mixed-precision form at twice the band (lmax ~5000-7000, 1441 distances)
    "psv2048": dict(mode="psv", tlen=3276.8, imax=2048, thdelta=0.125, rdelta=26.75, rmin=1000.0,
                    rmax=6350.0, r0=6071.0, thetas=1441),
    # SH (the reference's CPU configuration)
    "sh256": dict(mode="sh", tlen=1638.4, imax=256, thdelta=0.5, rdelta=28.5, rmin=3500.0,
                  rmax=6321.5, r0=6271.0, thetas=361),
}


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of a
# kernel on a workload, from an ncu capture of that kernel; the line reports
# where each figure came from next to it, and null where none was taken.
TRAFFIC = {
    ("catalogue", "cat_interp"): (0.672e9, "ncu capture of one launch (catalogue workload)"),
    ("catalogue", "cat_omega"): (0.598e9, "ncu capture of one launch (catalogue workload)"),
}
# Per-unit DRAM bytes of a kernel whose full-size launch is too large for an
# ncu capture with several metrics: measured on a small case of the same
# workload and scaled to a launch by the units it processes (reads by the
# orders contracted, writes by the frequencies whose output it writes).
TRAFFIC_PER_UNIT = {
    ("psv2048", "lsum_tc"): (0.5074e9 / 4281, 0.378e9 / 2,
                             "ncu capture of a two-frequency launch of this workload (4281 orders: 0.507 GB read, "
                             "0.378 GB written), scaled to the launch by orders (reads) and frequencies (writes)"),
}


def traffic(name, kernel, orders=None, freqs=None):
    v = TRAFFIC.get((name, kernel))
    if v:
        return v[0], v[1]
    u = TRAFFIC_PER_UNIT.get((name, kernel))
    if u and orders is not None and freqs is not None:
        return u[0] * orders + u[1] * freqs, u[2]
    return None, "not captured for this workload"


def workload(name: str):
    """Job (parameter file, DSM.config, model) and description of a workload."""
    import dsmsgt
    from dsmsgt import synth
    name = {"psv": "psv2048", "sh": "sh256"}.get(name, name)
    w = WORKLOADS[name]
    model = synth.psv_earth_model(0) if w["mode"] == "psv" else synth.sh_mantle_model(0)
    job = dsmsgt.Job(
        synth.param_file(tlen=w["tlen"], rmin=w["rmin"], rmax=w["rmax"], rdelta=w["rdelta"], r0=w["r0"],
                         thmin=0.0, thmax=180.0, thdelta=w["thdelta"], imin=0, imax=w["imax"]),
        synth.dsm_config(), model)
    nrec = int(round((w["rmax"] - w["rmin"]) / w["rdelta"])) + 1
    if w["mode"] == "psv":
        what = "SGTpsv synthetic Earth (IC solid, OC fluid, 6 mantle/crust zones, seed 0)"
    else:
        what = "SGTsh synthetic mantle (5 solid zones, seed 0)"
    desc = {"workload": what, "name": name, "tlen_s": w["tlen"], "np": w["imax"],
            "source_depth_km": round(6371.0 - w["r0"]), "receivers": nrec, "thetas": w["thetas"]}
    return job, desc


def workload_mode(name: str) -> str:
    return WORKLOADS[{"psv": "psv2048", "sh": "sh256"}.get(name, name)]["mode"]


def workload_imax(name: str) -> int:
    return WORKLOADS[{"psv": "psv2048", "sh": "sh256"}.get(name, name)]["imax"]


def per_component_rel_l2(a, b):
    """Relative L2 of each output component (last axis) over frequencies,
    radii and distances; components that vanish identically for the path
    (round-off only) are measured against the whole array's norm."""
    tot = np.sqrt(np.sum(np.abs(b) ** 2))
    out = []
    for c in range(a.shape[-1]):
        nb = np.sqrt(np.sum(np.abs(b[..., c]) ** 2))
        d = np.sqrt(np.sum(np.abs(a[..., c] - b[..., c]) ** 2))
        out.append(float(d / (nb if nb >= 1e-10 * tot else tot)) if tot > 0 else float(d))
    return out


def load_lmax_params(name: str):
    """Trained parameter block of the learned cutoff for a workload (written
    by dsmsgt.lmax_data for that workload's band and grid), or None."""
    name = {"psv": "psv2048", "sh": "sh256"}.get(name, name)
    path = os.path.join(REPO, "dsm-kernel_b200", "dsmsgt", f"lmax_{name}.f32")
    if not os.path.exists(path):
        return None
    p = np.fromfile(path, dtype=np.float32)
    return p if p.size == 34713 else None


def step_freqs(step: int, per_step: int, imax: int, rank: int = 0, world: int = 1) -> list[int]:
    """Frequencies of one step: per_step indices spread evenly over the
    frequencies this rank owns (the reference's zig-zag split of 1..imax),
    shifted per step so that steps differ."""
    from dsmsgt.shard import owned_freqs
    own = owned_freqs(1, imax, rank, world)
    off = (step * 37) % max(1, len(own) // per_step)
    return [own[(j * len(own) // per_step + off) % len(own)] for j in range(per_step)]


class ClockSampler:
    """Samples the SM clock, power and clock-event reasons of the bench's GPU
    during the timed region.  The GPU is found by its PCI bus id (CUDA and
    NVML number devices differently under CUDA_VISIBLE_DEVICES).  NVML is
    read every 10 ms from a thread (reads only: no setting is changed);
    without NVML, nvidia-smi is polled every 0.2 s."""
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []   # (sm MHz, max sm MHz, watts, set of active reason names)
        self.source = None
        self._stop = threading.Event()
        self._t = None
        try:
            import torch
            p = torch.cuda.get_device_properties(device)
            self.bus = f"{p.pci_domain_id:08X}:{p.pci_bus_id:02X}:{p.pci_device_id:02X}.0"
        except Exception:
            self.bus = None

    def _nvml(self):
        import pynvml
        pynvml.nvmlInit()
        h = pynvml.nvmlDeviceGetHandleByPciBusId(self.bus) if self.bus else \
            pynvml.nvmlDeviceGetHandleByIndex(self.device)
        masks = [pynvml.nvmlClocksEventReasonHwSlowdown, pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                 pynvml.nvmlClocksEventReasonSwThermalSlowdown, pynvml.nvmlClocksEventReasonSwPowerCap]
        mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

        def read():
            sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
            w = pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0
            bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
            return sm, mx, w, {n for n, m in zip(self.NAMES, masks) if bits & m}
        read()
        return read, pynvml.nvmlShutdown

    def _smi(self):
        ident = self.bus if self.bus else str(self.device)

        def read():
            out = subprocess.run(["nvidia-smi", f"--id={ident}", f"--query-gpu={self.Q}",
                                  "--format=csv,noheader,nounits"], capture_output=True,
                                 text=True, timeout=5).stdout.strip()
            f = [x.strip() for x in out.split(",")]
            if len(f) < 7:
                raise RuntimeError(out)
            num = lambda s: float(s) if s.replace(".", "").isdigit() else float("nan")
            return (num(f[0]), num(f[1]), num(f[2]),
                    {n for n, s in zip(self.NAMES, f[3:7]) if s.lower().startswith("active")})
        return read, lambda: None

    def start(self):
        try:
            read, close = self._nvml()
            self.source, period = "nvml", 0.01
        except Exception:
            read, close = self._smi()
            self.source, period = "nvidia-smi", 0.2

        def run():
            while not self._stop.is_set():
                try:
                    self.rows.append(read())
                except Exception:
                    pass
                self._stop.wait(period)
            try:
                close()
            except Exception:
                pass
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        mhz = [r[0] for r in self.rows if r[0] == r[0]]
        mx = [r[1] for r in self.rows if r[1] == r[1]]
        watts = [r[2] for r in self.rows if r[2] == r[2]]
        reasons = set().union(*[r[3] for r in self.rows]) if self.rows else set()
        return {"sm_mhz": float(np.median(mhz)) if mhz else None,
                "sm_max_mhz": max(mx) if mx else None,
                "sm_mhz_min": min(mhz) if mhz else None,
                "power_w_median": round(float(np.median(watts)), 1) if watts else None,
                "reasons": sorted(reasons), "samples": len(self.rows),
                "source": self.source, "pci_bus_id": self.bus}


CPU_THETAS = 8  # interior epicentral distances of a CPU sample


def cpu_sample(name: str, freq: int, threads: int):
    """Times the oracle (the FP64 CPU restatement of the reference's frequency
    loop, its own set-up, no product code) on one frequency of the workload:
    every order up to the cutoff, every receiver, all sources and outputs, on
    CPU_THETAS interior epicentral distances spread over 0-180 deg, one
    frequency spread over `threads` host threads.  The oracle times the parts
    proportional to the number of distances (vector harmonics, SYNN, the
    receiver x theta loop: the same work for every interior distance)
    separately, so the time of the full slice is the measured rest plus that
    part scaled to the workload's distances.  Returns (estimated seconds per
    full slice, measured seconds, measured theta seconds, llog)."""
    import dsmsgt
    from oracle import driver_setup, oracle as orc
    job, desc = workload(name)
    w = WORKLOADS[desc["name"]]
    if w["mode"] != "psv":
        raise ValueError("the CPU sample covers the P-SV workloads")
    d = 180.0 / CPU_THETAS
    text = job.param_text.replace(f"0.0 180.0 {w['thdelta']!r}\n", f"{d / 2!r} {180.0 - d / 2!r} {d!r}\n")
    s = driver_setup.psv_setup(dsmsgt.Job(text, job.conf_text, job.model_text))
    assert s.theta_n == CPU_THETAS, s.theta_n
    _, _, _, llog, t_theta, t_total = orc.run_threads(s, [freq], threads)
    full = float(t_total[0] - t_theta[0] + t_theta[0] * desc["thetas"] / CPU_THETAS)
    return full, float(t_total[0]), float(t_theta[0]), int(llog[0])


def cpu_sample_freq(k: int, imax: int, nspread: int = 20) -> int:
    """Frequency of CPU sample k: a fixed spread of nspread indices over the
    band (the same set whatever the step count), visited in turn."""
    j = k % nspread
    return 1 + int((j + 0.5) * imax / nspread)


CAT_METRIC = "catalogue points/s (6 windowed time series per point from 30 SGT components)"
CAT_UNIT = "points/s"
# one receiver radius of the mixed-precision catalogue (imax 2048, 1441
# distances at 0.125 deg) read the way KernelMaker reads it for a kernel grid
CAT_WORKLOAD = dict(name="catalogue", tlen=3276.8, fmin=0, fmax=2048, theta_n=1441, theta_delta=0.125,
                    sampling_hz=2.0, window_s=[400.0, 1000.0], ipdistance=10.0, c_red_reci=0.0,
                    points=1681, distances_deg=[30.0, 90.0], outputs=6,
                    record_sets="P-SV TSGT (20 components) + SH TSGT (10, into 7 and 12-20), complex64")


def catalogue_params():
    import dsmsgt
    w = CAT_WORKLOAD
    np1, shz, s0, s1 = dsmsgt.cat_np1(w["tlen"], w["fmax"], w["sampling_hz"], *w["window_s"])
    return dict(num=20, theta_n=w["theta_n"], theta_min=0.0, theta_delta=w["theta_delta"], fmin=w["fmin"],
                fmax=w["fmax"], np1=np1, tlen=w["tlen"], omegai=float(np.log(100.0) / w["tlen"]),
                ipdistance=w["ipdistance"], c_red_reci=w["c_red_reci"], iwin_start=s0, iwin_end=s1)


def catalogue_inputs(seed: int):
    """Seeded points (sorted distances) and per-point combination matrices."""
    rng = np.random.default_rng(seed)
    w = CAT_WORKLOAD
    dist = np.sort(rng.uniform(*w["distances_deg"], w["points"]))
    coef = rng.standard_normal((w["points"], w["outputs"], 20))
    return dist, coef


def catalogue_cpu(p, recs_host, dist, coef, npts: int):
    """The oracle (numpy FP64, one thread) on one radius: rdsgtomega over the
    full records once, then clsgt + combination + transform per point on a
    sample of points; scaled to the workload's points."""
    from oracle import catalogue as cat
    t0 = time.perf_counter()
    theta = p["theta_min"] + np.arange(p["theta_n"]) * p["theta_delta"]
    sets = [(recs_host[0], np.arange(20), np.ones(20)),
            (recs_host[1], cat.kind_dst(cat.TSGT_SH, 10), np.ones(10))]
    om = cat.omega_sgt(sets, 20, p["fmin"], p["fmax"], theta, p["tlen"], p["c_red_reci"])
    t_omega = time.perf_counter() - t0
    t0 = time.perf_counter()
    for k in range(npts):
        f = cat.clsgt(float(dist[k]), om, p["fmin"], p["theta_min"], p["theta_delta"], p["ipdistance"],
                      p["tlen"], p["c_red_reci"])
        cat.vector_fft_double(coef[k] @ f.T, p["fmin"], p["fmax"], p["np1"], p["omegai"], p["tlen"],
                              p["iwin_start"], p["iwin_end"])
    t_pt = (time.perf_counter() - t0) / npts
    t_step = t_omega + t_pt * len(dist)
    return len(dist) / t_step, {"rdsgtomega_s": t_omega, "per_point_s": t_pt}


def catalogue_bench(args):
    """Catalogue consumer: one step = one receiver radius (two record sets
    registered, series at every point)."""
    w = CAT_WORKLOAD
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    nf, nt = w["fmax"] - w["fmin"] + 1, w["theta_n"]

    def host_records(seed):
        rng = np.random.default_rng(seed)
        out = []
        for nc in (20, 10):
            a = np.empty((nf, nt, nc), np.complex64)
            a.real = rng.standard_normal((nf, nt, nc), dtype=np.float32)
            a.imag = rng.standard_normal((nf, nt, nc), dtype=np.float32)
            out.append(a)
        return out

    if args.impl == "reference":
        if rank != 0:
            return
        p = catalogue_params()
        dist, coef = catalogue_inputs(0)
        recs = host_records(1)
        for _ in range(args.warmup):
            catalogue_cpu(p, recs, dist, coef, 1)
        tot, samples = 0.0, []
        for _ in range(args.steps):
            v, t = catalogue_cpu(p, recs, dist, coef, 8)
            tot += len(dist) / v
            samples.append(t)
        value = args.steps * len(dist) / tot
        cpu = {"value": value, "unit": CAT_UNIT, "cores": 1, "kind": "port",
               "sample": "rdsgtomega over the full records once per step, clsgt + combination + "
                         "transform on 8 points per step scaled to 1681 points"}
        print(json.dumps({"impl": "reference", "metric": CAT_METRIC, "value": value, "unit": CAT_UNIT,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": {"workload": "catalogue", **w}, "cpu_baseline": cpu,
                          "e2e": {"value": value, "unit": CAT_UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    import dsmsgt
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    p = catalogue_params()
    dist, coef = catalogue_inputs(rank)
    # two radii, alternating; host copies in pinned memory (the e2e leg copies them in every step)
    pinned = [[torch.from_numpy(a).pin_memory() for a in host_records(10 * rank + k)] for k in range(2)]
    hrec = [[t_.numpy() for t_ in r] for r in pinned]
    drec = [[t_.to(f"cuda:{dev}") for t_ in r] for r in pinned]
    dst_sh = np.array([6] + list(range(11, 20)), np.int32)
    c = dsmsgt.Catalogue(p, device=dev)
    nwin = p["iwin_end"] - p["iwin_start"] + 1
    out = torch.empty((len(dist), w["outputs"], nwin), dtype=torch.float64, device=f"cuda:{dev}")

    def step(k, host):
        c.clear()
        r = hrec[k % 2] if host else drec[k % 2]
        c.add(r[0])
        c.add(r[1], dst_sh)
        return c.series(dist, coef) if host else c.series(dist, coef, out=out)

    for k in range(args.warmup):
        step(k, False)
    c.set_profiling(True)
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    ms, launches, kst = 0.0, 0, {}
    for k in range(args.steps):
        step(k, False)
        st = c.stats()
        ms += st.ms_total
        launches += st.launches
        for name, (t, n, b, f) in st.kernels().items():
            a = kst.setdefault(name, [0.0, 0, 0.0, 0.0])
            a[0] += t; a[1] += n; a[2] += b; a[3] += f
    torch.cuda.synchronize()
    clk = clocks.stop()
    # end to end: host records (numpy views of pinned memory) copied in, series copied out
    for k in range(2):
        step(k, True)
    t_e2e = 0.0
    for k in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step(k, True)
        t_e2e += time.perf_counter() - t0
    c.close()
    t = ms / 1e3
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    fp64 = max(dsmsgt.fp64_peak(dev), dsmsgt.fp64_peak(dev, mma=True))
    rooflines = {}
    for name, (tk, nk, bk, fk) in kst.items():
        if fk > 0:
            ach = fk / (tk / 1e3) / 1e12
            rooflines[name] = {"kernel": name, "bound": "fp64", "achieved": ach, "peak": fp64,
                               "unit": "TFLOP/s (algorithmic)", "frac": ach / fp64,
                               "traffic": traffic("catalogue", name)[0],
                               "traffic_source": traffic("catalogue", name)[1],
                               "peak_source": "measured (FP64 FMA and tensor-core probes, this run; the larger)",
                               "avg_launch_ms": tk / max(nk, 1)}
        else:
            ach = bk / (tk / 1e3) / 1e9
            peak = peaks.get("hbm_gbs", 6650.0)
            rooflines[name] = {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                               "frac": ach / peak, "traffic": traffic("catalogue", name)[0],
                               "traffic_source": traffic("catalogue", name)[1],
                               "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                               "avg_launch_ms": tk / max(nk, 1)}
    roof = rooflines[max(kst.items(), key=lambda kv: kv[1][0])[0]]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, tt = catalogue_cpu(p, hrec[0], dist, coef, 8)
        cpu = {"value": v, "unit": CAT_UNIT, "cores": 1, "kind": "port",
               "sample": "oracle: rdsgtomega over the full records once, clsgt + combination + transform "
                         f"on 8 points scaled to {len(dist)} points; measured: {json.dumps(tt)}"}
    if rank == 0:
        rec_bytes = sum(a.nbytes for a in hrec[0])
        print(json.dumps({
            "metric": CAT_METRIC, "value": args.steps * len(dist) * world / t, "unit": CAT_UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded complex64 records, seeded distances and combination matrices)",
            "config": {"workload": "catalogue", **w, "np1": p["np1"], "window_samples": nwin,
                       "l2": "inputs larger than L2 (708 MB of records per step, two radii alternating)"},
            "e2e": {"value": args.steps * len(dist) / t_e2e, "unit": CAT_UNIT,
                    "h2d_bytes_per_step": int(rec_bytes + dist.nbytes + coef.nbytes),
                    "d2h_bytes_per_step": int(len(dist) * w["outputs"] * nwin * 8)},
            "gpu_launches": int(launches), "roofline": roof, "stage_rooflines": rooflines,
            "kernel_share": {k: round(v[0] / max(ms, 1e-9), 4) for k, v in kst.items()},
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kst.items()},
            "cpu_baseline": cpu, "clocks": clk}))


KER_METRIC = "kernel points/s (isotropic P and S kernels: 3 products, transforms, Butterworth filter, sums)"
KER_UNIT = "points/s"


def kernels_inputs(seed: int, p, npt: int, nr: int):
    rng = np.random.default_rng(seed)
    nf = p["fmax"] - p["fmin"] + 1
    nwin = p["iwin_end"] - p["iwin_start"] + 1
    fs = 2 * p["np1"] / p["tlen"]
    h = [(rng.standard_normal((npt, 6, nf)) + 1j * rng.standard_normal((npt, 6, nf))) for _ in range(2)]
    kp = dict(types=3, nfilter=0, fclp=[0.005], fchp=[0.05], npoles=4, sampling_hz=fs,
              nt1=[p["iwin_start"] + nwin // 8], nt2=[p["iwin_end"] - nwin // 8],
              coeff=rng.standard_normal((nwin, nr, 8, 1)),
              jacobian=rng.standard_normal((nf, nr)) + 1j * rng.standard_normal((nf, nr)))
    ir = rng.integers(0, nr, npt).astype(np.int32)
    return h[0], h[1], kp, ir


def kernels_bench(args):
    """Per-point kernel formulas: one step = the isotropic P and S kernels
    (types 1, 3, 4, 5, 7, 8; one broad-band filter, the reference's nfilter
    = 0, 4 Butterworth sections) of the catalogue workload's 1681 points,
    from h3 / h4 spectra resident on the device."""
    w = CAT_WORKLOAD
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    p = catalogue_params()
    npt, nr = w["points"], 4
    nwin = p["iwin_end"] - p["iwin_start"] + 1
    nf = p["fmax"] - p["fmin"] + 1
    cfg = {"workload": "kernels", "points": npt, "np1": p["np1"], "window_samples": nwin,
           "frequencies": nf, "radii": nr, "filters": 1, "npoles": 4,
           "l2": "inputs larger than L2 (h3 and h4 spectra: 661 MB per step)"}

    def cpu(h3, h4, kp, ir, nsample):
        from oracle import catalogue as cat
        q = dict(kp, nr=nr, nktype=8)
        t0 = time.perf_counter()
        cat.iso_kernels(p, q, ir[:nsample], h3[:nsample], h4[:nsample])
        return nsample / (time.perf_counter() - t0)

    if args.impl == "reference":
        if rank != 0:
            return
        h3, h4, kp, ir = kernels_inputs(0, p, 64, nr)
        cpu(h3, h4, kp, ir, 4)
        vals = [cpu(h3, h4, kp, ir, 64) for _ in range(args.steps)]
        value = len(vals) / sum(1.0 / v for v in vals)
        print(json.dumps({"impl": "reference", "metric": KER_METRIC, "value": value, "unit": KER_UNIT,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1e3 * 64 / value, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
                          "cpu_baseline": {"value": value, "unit": KER_UNIT, "cores": 1, "kind": "port",
                                           "sample": "oracle on 64 points per step (numpy, one thread); "
                                                     "ms_per_step is that sample's time"},
                          "e2e": {"value": value, "unit": KER_UNIT, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    import dsmsgt
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    h3, h4, kp, ir = kernels_inputs(rank, p, npt, nr)
    d3 = torch.from_numpy(h3).to(f"cuda:{dev}")
    d4 = torch.from_numpy(h4).to(f"cuda:{dev}")
    c = dsmsgt.Catalogue(p, device=dev)
    c.set_kernel_params(kp["types"], kp["nfilter"], kp["fclp"], kp["fchp"], kp["npoles"], kp["sampling_hz"],
                        kp["nt1"], kp["nt2"], kp["coeff"], kp["jacobian"])
    ker = torch.zeros((npt, 1, 9), dtype=torch.float64, device=f"cuda:{dev}")
    irr = np.ascontiguousarray(ir, np.int32)
    L = dsmsgt.lib()

    def step():
        rc = L.dsm_cat_kernels(c.h, npt, dsmsgt._ptr(irr, dsmsgt._ip), d3.data_ptr(), d4.data_ptr(), 1,
                               ker.data_ptr(), None, 1)
        assert rc == 0, L.dsm_cat_last_error(c.h).decode()

    for _ in range(args.warmup):
        step()
    c.set_profiling(True)
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ms, kst = 0.0, {}
    for _ in range(args.steps):
        step()
        st = c.stats()
        ms += st.ms_total
        for name, (tk, nk, bk, _) in st.kernels().items():
            a_ = kst.setdefault(name, [0.0, 0, 0.0])
            a_[0] += tk; a_[1] += nk; a_[2] += bk
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t0
    clk = clocks.stop()
    c.set_profiling(False)
    t = ms / 1e3
    # end to end: spectra from pinned host memory, kernels back to the host
    p3 = torch.from_numpy(h3).pin_memory().numpy()
    p4 = torch.from_numpy(h4).pin_memory().numpy()
    c.kernels(ir, p3, p4)
    t_e2e = 0.0
    for _ in range(args.steps):
        t1 = time.perf_counter()
        c.kernels(ir, p3, p4)
        t_e2e += time.perf_counter() - t1
    c.close()
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    # per stage: algorithmic bytes (the library's count) over the stage's
    # event time; the line's roofline is the longest stage's
    peak = peaks.get("hbm_gbs", 6650.0)
    psrc = "measured" if "hbm_gbs" in peaks else "fallback"
    stages = {}
    for name, (tk, nk, bk) in kst.items():
        ach_k = bk / (tk / 1e3) / 1e9
        stages[name] = {"kernel": name, "bound": "hbm" if name != "ker_filter" else "latency (sequential recursion)",
                        "achieved": ach_k, "peak": peak, "unit": "GB/s", "frac": ach_k / peak,
                        "avg_launch_ms": tk / max(nk, 1), "launches": nk, "alg_bytes_per_step": bk / args.steps,
                        "peak_source": psrc}
    top = max(kst.items(), key=lambda kv: kv[1][0])[0]
    alg = sum(v[2] for v in kst.values())
    ach = alg / t / 1e9
    cpu_b = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v = cpu(h3, h4, kp, ir, 64)
        cpu_b = {"value": v, "unit": KER_UNIT, "cores": 1, "kind": "port",
                 "sample": "oracle on 64 of the 1681 points (numpy, one thread)"}
    if rank == 0:
        print(json.dumps({
            "metric": KER_METRIC, "value": args.steps * npt * world / t, "unit": KER_UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded spectra, coefficients and jacobian)", "config": cfg,
            "timing": "CUDA events of the library (profiling on) over the device work of each call; "
                      f"host clock around the same calls: {1e3 * t_wall / args.steps:.3f} ms per step",
            "e2e": {"value": args.steps * npt / t_e2e, "unit": KER_UNIT,
                    "h2d_bytes_per_step": int(h3.nbytes + h4.nbytes + irr.nbytes),
                    "d2h_bytes_per_step": int(npt * 9 * 8)},
            "gpu_launches": int(sum(v[1] for k_, v in kst.items() if k_ != "ker_fft")),
            "roofline": dict(stages[top], traffic=None),
            "stage_rooflines": stages,
            "call_roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                              "scope": "whole call (products, cuFFT, filter and sums)", "peak_source": psrc},
            "kernel_share": {k_: round(v[0] / max(ms, 1e-9), 4) for k_, v in kst.items()},
            "cpu_baseline": cpu_b, "clocks": clk}))


# Batched uneven-size form, scaled to fit a few minutes and the memory of
# one GPU: several seeded models and source depths of P-SV and SH in one
# request (all contexts resident at once; an 8-depth P-SV context's field
# matrices reach 8192 orders, about 38 GB at 4 frequencies per step).  P-SV
# depths of a model share one context (one factorisation per (omega, l));
# SH contexts hold one depth each.
BATCH = dict(tlen=3276.8, imax=1024, models=2, psv_depths_km=[10, 108, 207, 305, 404, 502, 601, 700],
             sh_depths_km=[100, 400],
             psv=dict(thdelta=0.25, rdelta=26.75, rmin=1000.0, rmax=6350.0),
             sh=dict(thdelta=0.5, rdelta=28.5, rmin=3500.0, rmax=6321.5))


def batch_setups(model: int, mode: str, depths_km):
    import dsmsgt
    from dsmsgt import synth
    g = BATCH[mode]
    text = synth.psv_earth_model(model) if mode == "psv" else synth.sh_mantle_model(model)
    out = []
    for d in depths_km:
        job = dsmsgt.Job(synth.param_file(tlen=BATCH["tlen"], rmin=g["rmin"], rmax=g["rmax"], rdelta=g["rdelta"],
                                          r0=6371.0 - d, thmin=0.0, thmax=180.0, thdelta=g["thdelta"], imin=0,
                                          imax=BATCH["imax"]), synth.dsm_config(), text)
        out.append(dsmsgt.Setup(job, mode))
    return out


def batch_bench(args):
    """Several models x source depths, P-SV and SH, per step: per_step
    frequencies of every context.  Timed twice over the same steps: the
    contexts one after another with the default tile shapes, and all of them
    in one dsm_run_request (each context on its own host thread and streams)
    after dsm_autotune chose each context's tiles.  The unit is a
    source-frequency slice (one frequency of one source depth, every order
    to the cutoff, all outputs on the full grid)."""
    import torch
    import dsmsgt
    prec = {"fp64": dsmsgt.DSM_PREC_FP64, "mixed": dsmsgt.DSM_PREC_MIXED,
            "mixed_bf16": dsmsgt.DSM_PREC_MIXED_BF16}[args.precision]
    F = args.per_step
    imax = BATCH["imax"]
    psv = [batch_setups(m, "psv", BATCH["psv_depths_km"]) for m in range(BATCH["models"])]
    sh = [batch_setups(m, "sh", BATCH["sh_depths_km"]) for m in range(BATCH["models"])]
    ctxs = ([dsmsgt.MultiSourceContext(ss, precision=prec, freq_batch=F) for ss in psv] +
            [dsmsgt.Context(s, precision=prec, freq_batch=F) for ss in sh for s in ss])
    nsrc = [len(c.setups) if isinstance(c, dsmsgt.MultiSourceContext) else 1 for c in ctxs]
    per_step = F * sum(nsrc)

    def freqs(step, k):  # each context its own spread of the band
        return step_freqs(step * 7 + k, F, imax)

    def sequential(step):
        for k, c in enumerate(ctxs):
            dsmsgt.run_request([c], [freqs(step, k)], outputs=False)

    def together(step):
        dsmsgt.run_request(ctxs, [freqs(step, k) for k in range(len(ctxs))], outputs=False)

    def timed(fn):
        for w in range(args.warmup):
            fn(1000 + w)
        torch.cuda.synchronize()
        clocks = ClockSampler(0)
        clocks.start()
        t0 = time.perf_counter()
        for k in range(args.steps):
            fn(k)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        return t, clocks.stop()

    t_seq, clk_seq = timed(sequential)
    tunings = []
    for k, c in enumerate(ctxs):
        t, _ = c.autotune(freqs(2000, k), reps=1)
        tunings.append(t)
    t_req, clk = timed(together)
    free, total = torch.cuda.mem_get_info()
    launches = sum(c.stats().launches for c in ctxs)
    for c in ctxs:
        c.close()

    # accuracy of the mixed path on the batch: one model's P-SV depths and
    # one SH context, mixed against FP64 on a low and the top frequency
    rel = None
    if prec != dsmsgt.DSM_PREC_FP64:
        worst = {"tsgt": 0.0, "rsgt": 0.0, "synn": 0.0}
        fr = [3, imax]
        for ss in (psv[-1][::3],):
            a = dsmsgt.MultiSourceContext(ss, precision=prec, freq_batch=2)
            b = dsmsgt.MultiSourceContext(ss, precision=dsmsgt.DSM_PREC_FP64, freq_batch=2)
            for ga, gb in zip(a.run(fr), b.run(fr)):
                for key, x, y in zip(("tsgt", "rsgt", "synn"), ga[:3], gb[:3]):
                    worst[key] = max(worst[key], max(per_component_rel_l2(x, y)))
            a.close()
            b.close()
        a = dsmsgt.Context(sh[-1][0], precision=prec, freq_batch=2)
        b = dsmsgt.Context(sh[-1][0], precision=dsmsgt.DSM_PREC_FP64, freq_batch=2)
        for key, x, y in zip(("tsgt", "rsgt", "synn"), a.run(fr)[:3], b.run(fr)[:3]):
            worst[key] = max(worst[key], max(per_component_rel_l2(x, y)))
        a.close()
        b.close()
        rel = dict(worst, frequencies=fr, sample="last model: P-SV depths 10, 305, 601 km and SH 100 km")

    slices = args.steps * per_step
    line = {"metric": "SGT source-frequency slices/s, batched models x depths (P-SV + SH)",
            "value": slices / t_req, "unit": "source-freq-slices/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_req / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if prec == dsmsgt.DSM_PREC_FP64 else "fp16x2 pieces, f32 accumulate (l-sum); f64 solves",
            "data": "synthetic (seeded 1-D polynomial models, reference file formats)",
            "config": {"workload": "batched models x depths", "tlen_s": BATCH["tlen"], "np": imax,
                       "models": BATCH["models"], "psv_depths_km": BATCH["psv_depths_km"],
                       "sh_depths_km": BATCH["sh_depths_km"], "contexts": len(ctxs),
                       "sources": sum(nsrc), "freqs_per_context_per_step": F, "precision": args.precision,
                       "learned_lmax": False, "psv_grid": BATCH["psv"], "sh_grid": BATCH["sh"],
                       "l2": "inputs larger than L2", "device_memory_used_gb": round((total - free) / 1e9, 1)},
            "timing": "host wall clock around the requests, device synchronised on both sides "
                      "(outputs stay on the device)",
            "sequential": {"value": slices / t_seq, "ms_per_step": 1e3 * t_seq / args.steps,
                           "tiles": "default", "clocks": clk_seq},
            "speedup_request_vs_sequential": t_seq / t_req,
            "tunings": tunings, "gpu_launches": int(launches), "clocks": clk,
            "rel_l2_vs_fp64": rel}
    print(json.dumps(line))


def reference_arm(args):
    """The reference's CPU implementation of the path (the oracle: the FP64
    restatement of the Fortran frequency loop, with its own set-up), timed on
    the host cores on a bounded sample per step: one frequency of a fixed
    spread over the band (cpu_sample)."""
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    imax = workload_imax(args.mode)
    _, desc = workload(args.mode)
    for w in range(args.warmup):  # untimed: the lowest frequencies (page cache, thread start)
        cpu_sample(args.mode, 1 + w, threads)
    est, wall, samples = 0.0, 0.0, []
    for k in range(args.steps):
        f = cpu_sample_freq(k, imax)
        full, t, th, ll = cpu_sample(args.mode, f, threads)
        est += full
        wall += t
        samples.append({"freq": f, "llog": ll, "measured_s": round(t, 3), "theta_part_s": round(th, 3),
                        "full_slice_s": round(full, 2)})
    value = args.steps / est
    cpu = {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": (f"one frequency per step from a fixed spread of 20 over 1..{imax}, every order to the "
                      f"cutoff, all {desc['receivers']} receivers and outputs, {CPU_THETAS} interior epicentral "
                      f"distances; the theta-proportional part (timed by the oracle) scaled to {desc['thetas']}"),
           "extrapolated": f"theta loop x {desc['thetas']}/{CPU_THETAS}; solves and set-up per order measured in full",
           "setup": "oracle's own (numpy restatement of the reference's set-up; no product library)",
           "steps": samples}
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic", "config": desc, "cpu_baseline": cpu,
                      "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", "--mode", dest="mode", default="psv2048",
                    choices=["psv1024", "psv2048", "sh256", "psv", "sh", "catalogue", "kernels", "batch"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed_bf16"])
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64 comparison run")
    # The plain first ranges pad 2.0 % of the orders on the 2048-frequency
    # benchmark model, the trained block 2.8 % (its held-out models: 14.5 %
    # plain, 3.0 % learned), so the default run uses the plain ranges
    ap.add_argument("--lmax", dest="lmax", action="store_true",
                    help="first order ranges from the trained cutoff block of the workload")
    ap.add_argument("--per-step", type=int, default=None,
                    help="frequency slices per step (default 20; 4 per context for --workload batch)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="default tile shapes instead of the library's tuner")
    args = ap.parse_args()
    if args.per_step is None:
        args.per_step = 4 if args.mode == "batch" else 20
    if args.mode == "catalogue":
        catalogue_bench(args)
        return
    if args.mode == "kernels":
        kernels_bench(args)
        return
    if args.mode == "batch":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched form has no reference run "
                              "(one model and depth per reference job)"}))
        elif int(os.environ.get("RANK", "0")) == 0:
            batch_bench(args)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    imax = workload_imax(args.mode)
    mode = workload_mode(args.mode)

    if args.impl == "reference":
        if rank == 0:
            reference_arm(args)
        return

    import torch
    import dsmsgt
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = local
    job, desc = workload(args.mode)
    setup = dsmsgt.Setup(job, mode)
    lmax_params = load_lmax_params(args.mode) if args.lmax else None

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(t):
        if world > 1:
            tt = torch.tensor([t], device=f"cuda:{dev}", dtype=torch.float64)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            t = float(tt.item())
        return t

    def measure(prec, use_lmax):
        """Device and end-to-end throughput of one precision mode over the
        same steps; per-kernel CUDA-event times; solve statistics."""
        ctx = dsmsgt.Context(setup, precision=prec, device=dev, freq_batch=args.per_step,
                             use_lmax_predictor=1 if use_lmax else 0)
        if use_lmax:
            ctx.set_lmax_model(lmax_params)
        # tile shapes chosen by the library's tuner on a step outside the
        # timed ones (untimed), for each precision mode alike
        tuning = None
        if args.autotune:
            tuning, _ = ctx.autotune(step_freqs(2000, args.per_step, imax, rank, world), reps=1)
        for w in range(args.warmup):  # untimed
            ctx.run_device(step_freqs(1000 + w, args.per_step, imax, rank, world))
        ctx.set_profiling(True)
        clocks = ClockSampler(dev)
        clocks.start()
        kstats, ms_dev, launches, llogs = {}, 0.0, 0, []
        phases = {"solve": 0.0, "lsum": 0.0}
        exec_flops = 0.0
        sol = {"systems": 0, "orders_used": 0, "orders_padded": 0, "solve_rounds": 0, "freqs_extended": 0}
        barrier()
        for k in range(args.steps):
            llogs.append(ctx.run_device(step_freqs(k, args.per_step, imax, rank, world)).tolist())
            st = ctx.stats()
            ms_dev += st.ms_total
            phases["solve"] += st.ms_solve
            phases["lsum"] += st.ms_lsum
            exec_flops += st.lsum_flops_exec
            for key in sol:
                sol[key] += getattr(st, key)
            launches += st.launches - sum(v[1] for n_, v in st.kernels().items() if n_.startswith("lsum_dgemm"))
            for name, (ms, n, b, f) in st.kernels().items():
                acc = kstats.setdefault(name, [0.0, 0, 0.0, 0.0])
                acc[0] += ms; acc[1] += n; acc[2] += b; acc[3] += f
        barrier()
        clk = clocks.stop()
        ctx.set_profiling(False)
        t_dev = max_over_ranks(ms_dev / 1e3)
        # end to end through the C-ABI (dsm_run_freqs), host wall clock: the
        # frequency list goes in, complex64 catalogue records come back to
        # pinned host memory every step; the set-up is resident per context
        nt, nr, ns = setup.num
        per_t = nt * setup.r_n * setup.theta_n
        per_r = nr * setup.r_n * setup.theta_n
        per_s = ns * setup.theta_n
        F = args.per_step
        ht = torch.empty(2 * per_t * F, dtype=torch.float32, pin_memory=True)
        hr = torch.empty(2 * per_r * F, dtype=torch.float32, pin_memory=True)
        hy = torch.empty(2 * per_s * F, dtype=torch.float32, pin_memory=True)
        ll = np.zeros(F, np.int32)
        ctx.run_host32(step_freqs(0, F, imax, rank, world), ht.data_ptr(), hr.data_ptr(), hy.data_ptr(), ll)
        barrier()
        t0 = time.perf_counter()
        for k in range(args.steps):
            ctx.run_host32(step_freqs(k, F, imax, rank, world), ht.data_ptr(), hr.data_ptr(), hy.data_ptr(), ll)
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        barrier()
        ctx.close()
        slices = args.steps * args.per_step * world
        return {"value": slices / t_dev, "t": t_dev, "kstats": kstats, "launches": launches, "tuning": tuning,
                "llogs": llogs, "clocks": clk, "solve": sol,
                "phase_ms_per_step": {k: v / args.steps for k, v in phases.items()},
                "exec_flops": exec_flops,
                "e2e": {"value": slices / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 4 * F,
                        "d2h_bytes_per_step": 8 * (per_t + per_r + per_s) * F + 4 * F,
                        "timing": "host wall clock around dsm_run_freqs (perf_counter), records to pinned memory"}}

    headline_prec = {"fp64": dsmsgt.DSM_PREC_FP64, "mixed": dsmsgt.DSM_PREC_MIXED,
                     "mixed_bf16": dsmsgt.DSM_PREC_MIXED_BF16}[args.precision]
    mixed = headline_prec != dsmsgt.DSM_PREC_FP64
    use_lmax = mixed and lmax_params is not None
    run = measure(headline_prec, use_lmax)
    plain = measure(dsmsgt.DSM_PREC_FP64, False) if mixed and not args.no_fp64 else None

    # accuracy of the headline path against the FP64 GPU path, from the
    # library's own report: an FP64 context attached to the mixed one
    # recomputes every fourth frequency of the first step and the top of the
    # band (outside the timed region)
    rel = None
    if mixed and rank == 0:
        fr = sorted(set(step_freqs(0, args.per_step, imax)) | {imax})
        c64 = dsmsgt.Context(setup, precision=dsmsgt.DSM_PREC_FP64, device=dev, freq_batch=4)
        cm = dsmsgt.Context(setup, precision=headline_prec, device=dev, freq_batch=len(fr))
        cm.set_fp64_check(c64, 1)
        cm.run_device(fr)
        acc = cm.accuracy()
        cm.set_fp64_check(None)
        cm.close()
        c64.close()
        rel = {"frequencies": fr, "llog_equal": acc["llog_equal"], "tsgt": acc["tsgt_max"],
               "rsgt": acc["rsgt_max"], "synn": acc["synn_max"], "source": "dsm_get_accuracy"}

    # roofline of the dominant kernel of this library (CUDA events on the
    # library's stream over the timed region)
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as fh:
            peaks = json.load(fh)
    except Exception:
        pass
    kstats = run["kstats"]
    own = {k: v for k, v in kstats.items() if not k.startswith("lsum_dgemm")}
    dom = max(own.items(), key=lambda kv: kv[1][0]) if own else None
    roof = None
    if dom:
        name, (ms, n, b, f) = dom
        sol = run["solve"]
        tr, tr_src = traffic(desc["name"], name, orders=sol["orders_used"] / max(n, 1),
                             freqs=args.steps * args.per_step / max(n, 1))
        if f > 0:
            # algorithmic flops (one real product per row, column and order up
            # to the cutoff); the split path runs three fp16 piece products
            # per algorithmic product, so its ceiling is a third of the peak
            ach = f / (ms / 1e3) / 1e12
            peak = peaks.get("bf16_tflops", 1590.0)
            roof = {"kernel": name, "bound": "tensor", "achieved": ach, "peak": peak,
                    "unit": "TFLOP/s", "frac": ach / peak, "traffic": tr, "traffic_source": tr_src,
                    "peak_source": "measured (bf16 burst)" if "bf16_tflops" in peaks else "fallback",
                    "avg_launch_ms": ms / max(n, 1), "piece_products": 3,
                    "frac_of_piece_ceiling": 3.0 * ach / peak}
            if run.get("exec_flops", 0.0) > 0:
                # the row tiles stop at their rows' last nonzero order (the
                # depth cut zeroes deep receivers' high orders): executed
                # products, three fp16 pieces each, against the same peak
                ache = run["exec_flops"] / (ms / 1e3) / 1e12
                roof.update({"executed_fraction_of_algorithmic": run["exec_flops"] / f,
                             "achieved_executed": ache, "frac_executed_of_piece_ceiling": 3.0 * ache / peak})
        else:
            ach = b / (ms / 1e3) / 1e9
            peak = peaks.get("hbm_gbs", 6650.0)
            roof = {"kernel": name, "bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                    "frac": ach / peak, "traffic": tr, "traffic_source": tr_src,
                    "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                    "avg_launch_ms": ms / max(n, 1)}
    share = {k: round(v[0] / max(run["t"] * 1e3, 1e-9), 4) for k, v in kstats.items()}
    # HBM-bound band kernels: algorithmic bytes over their event time
    hbm = {}
    for k in ("psv_factor", "psv_substitution", "psv_factor_long", "psv_substitution_long"):
        if k in kstats and kstats[k][0] > 0:
            ach = kstats[k][2] / (kstats[k][0] / 1e3) / 1e9
            peak = peaks.get("hbm_gbs", 6650.0)
            hbm[k] = {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                      "alg_bytes_per_step": kstats[k][2] / args.steps, "ms_per_step": kstats[k][0] / args.steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and mode == "psv":
        threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        f = cpu_sample_freq(0, imax)
        full, t, th, _ = cpu_sample(args.mode, f, threads)
        cpu = {"value": 1.0 / full, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": (f"frequency {f}, every order to the cutoff, all receivers and outputs, {CPU_THETAS} "
                          f"interior distances (measured {t:.1f} s, theta part {th:.1f} s), theta part scaled "
                          f"to {desc['thetas']} distances; oracle with its own set-up"),
               "extrapolated": f"theta loop x {desc['thetas']}/{CPU_THETAS}"}

    if rank == 0:
        sol = run["solve"]
        line = {"metric": METRIC, "value": run["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * run["t"] / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if not mixed else ("fp16x2 pieces, f32 accumulate (l-sum); f64 solves"
                                                 if args.precision == "mixed" else
                                                 "bf16x3 pieces, f32 accumulate (l-sum); f64 solves"),
                "data": "synthetic (seeded 1-D polynomial model, reference file formats)",
                "config": dict(desc, precision=args.precision, slices_per_step=args.per_step,
                               learned_lmax=bool(use_lmax),
                               depth_cutoff=(1e-20 if mixed and mode == "psv" else 0.0),
                               parallelism=f"dp{world} (frequencies per rank)",
                               l2="inputs larger than L2 (field matrices of several GB per step)"),
                "e2e": run["e2e"], "gpu_launches": int(run["launches"]), "tuning": run["tuning"],
                "roofline": roof, "hbm_kernels": hbm, "kernel_share": share,
                "phase_ms_per_step": run["phase_ms_per_step"],
                "cpu_baseline": cpu, "clocks": run["clocks"],
                "solve": dict(sol, slices=args.steps * args.per_step,
                              padded_fraction=sol["orders_padded"] / max(sol["orders_used"], 1),
                              miss_rate=sol["freqs_extended"] / max(args.steps * args.per_step, 1)),
                "llog_first_step": run["llogs"][0]}
        if plain:
            line["fp64"] = {"value": plain["value"], "ms_per_step": 1e3 * plain["t"] / args.steps,
                            "tuning": plain["tuning"],
                            "e2e": plain["e2e"]["value"], "solve": plain["solve"], "clocks": plain["clocks"],
                            "kernel_share": {k: round(v[0] / max(plain["t"] * 1e3, 1e-9), 4)
                                             for k, v in plain["kstats"].items()}}
            line["speedup_vs_fp64"] = run["value"] / plain["value"]
            line["speedup_vs_fp64_e2e"] = run["e2e"]["value"] / plain["e2e"]["value"]
        if rel:
            line["rel_l2_vs_fp64"] = rel
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
