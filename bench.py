"""Benchmark of the structure-factor + detector-chain path.

Workload (one step): the 50,000-atom precision-stress particle (C 62 % N 17 %
O 20 % S 1 %, uniform in a 12 nm ball, 1.2 A minimum separation, seeded) on a
1024 x 1024 detector of 75 um pixels at 0.1 m, wavelength 0.15 nm, compensated
FP32 structure factor followed by the full detector chain (Thomson, solid
angle, photons, Poisson, electrons, readout noise 10 e-, ADC with a clamp at
65535).  Inputs are device-resident for `value`; `e2e` runs the reference-
facing simulate_shot call with host buffers.  Under torchrun every rank
simulates its own orientation of the particle (weak scaling, no data-path
collective); the timing is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom·pixel terms/s at ≤1e-5 rel |F|² err vs FP64; backward/forward time ratio"
UNIT = "terms/s"
WORKLOAD = "precision_50k"
MUFU_PER_SM_CLK = 16          # sin/cos (MUFU) results per SM per clock, nominal
FMA_PER_SM_CLK = 128          # FP32 FMA lanes per SM per clock, nominal
OPS_PER_TERM_MUFU = 2         # canonical term: 2 MUFU (sin, cos)
OPS_PER_TERM_FMA = 5          # canonical term: 3 FMA (q.r) + 2 FMA (accumulate)
L2_FLUSH_BYTES = 256 << 20


def workload_desc():
    return ("precision_50k: 50,000 atoms (C 62% N 17% O 20% S 1%, 12 nm ball), 1024x1024 pixels of 75 um at 0.1 m, "
            "lambda 0.15 nm, FP32 structure factor (FP64 phase, FP32 sin/cos) + detector chain (readout 10 e-, clamp 65535)")


# ----------------------------------------------------------------- CPU reference

def _ref_worker(args):
    """spsim's own CPU path on one pixel slab (runs in a spawned process)."""
    Z, pos, hkl, vector = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O

    t = time.perf_counter()
    O.ref_pattern(Z, pos, hkl, vector=vector)
    return time.perf_counter() - t


def _ref_kind():
    from oracle import oracle as O

    return "reference" if O.ref_available() else "port"


def _cpu_sample(Z, pos, hkl_all, pool, nproc, target_s, vector=True):
    """Time spsim's CPU structure factor on an evenly spread pixel sample sized to
    about target_s of wall time over nproc processes; returns (terms/s, desc)."""
    from oracle import oracle as O

    n_atoms = int(np.count_nonzero(Z))
    if O.ref_available():
        t = time.perf_counter()
        O.ref_pattern(Z, pos, hkl_all[:64], vector=vector)
        per_pix = (time.perf_counter() - t) / 64
    else:
        per_pix = n_atoms * 30e-9
    npix = int(min(len(hkl_all), max(nproc, target_s * nproc / max(per_pix, 1e-9))))
    idx = np.linspace(0, len(hkl_all) - 1, npix).astype(np.int64)
    sample = hkl_all[idx]
    slabs = np.array_split(sample, nproc)
    if O.ref_available():
        t = time.perf_counter()
        pool.map(_ref_worker, [(Z, pos, s, vector) for s in slabs])
        wall = time.perf_counter() - t
    else:  # the oracle port, FP64, threaded
        t = time.perf_counter()
        O.structure_factor(Z, pos.astype(np.float64), sample.astype(np.float64), nthreads=nproc)
        wall = time.perf_counter() - t
    path = "vector_compute_pattern_on_list" if vector else "compute_pattern_on_list"
    desc = "%d evenly spaced pixels of the 1024x1024 detector x %d atoms, %s, %d processes over contiguous " \
           "slabs (src/mpi.c:30-48)" % (npix, n_atoms, path, nproc)
    return npix * n_atoms / wall, desc, wall


def _make_workload(rank=0):
    from spsim_b200 import synth

    w = synth.WORKLOADS[WORKLOAD]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    return w, Z, pos


def _hkl_host(w):
    from oracle import oracle as O

    d = w["det"]
    return O.hkl_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"]).astype(
        np.float32)


def run_reference(args):
    """--impl reference: spsim's own CPU path on this box's host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import multiprocessing as mp

    nproc = os.cpu_count() or 1
    ctx = mp.get_context("spawn")
    w, Z, pos = _make_workload()
    hkl = _hkl_host(w)
    with ctx.Pool(nproc) as pool:
        vals, walls = [], []
        for i in range(args.warmup + args.steps):
            v, desc, wall = _cpu_sample(Z, pos, hkl, pool, nproc, target_s=2.0)
            if i >= args.warmup:
                vals.append(v)
                walls.append(wall)
    value = float(statistics.median(vals))
    terms = float(w["natoms"]) * w["det"]["nx"] * w["det"]["ny"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        # a step is one bounded pixel sample of the workload (terms/s is intensive)
        "ms_per_step": float(statistics.median(walls)) * 1e3,
        "ms_per_full_pattern_extrapolated": terms / value * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_desc(), "precision": "reference float path (SSE sincos_ps)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nproc, "kind": _ref_kind(), "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------- GPU

class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()
        return False

    def summary(self):
        rows = []
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


_PROBE = {}
PROBE_SRC = os.path.join(ROOT, "pipe_probe.cu")
PROBE_EXE = os.path.join(ROOT, "_build", "pipe_probe")


def _build_probe():
    """Compile pipe_probe.cu for sm_100a into _build/ (once; a few seconds)."""
    if os.path.exists(PROBE_EXE) and os.path.getmtime(PROBE_EXE) >= os.path.getmtime(PROBE_SRC):
        return True
    os.makedirs(os.path.dirname(PROBE_EXE), exist_ok=True)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    try:
        r = subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-I", ROOT, "-o", PROBE_EXE,
                            PROBE_SRC], capture_output=True, text=True, timeout=300)
    except (OSError, subprocess.TimeoutExpired):
        return False
    return r.returncode == 0


def measured_pipe_peaks():
    """FP32-FMA lane-ops/s and MUFU ops/s measured on this GPU by the pipe probe
    (pipe_probe.cu), or None when it cannot be built or run."""
    if "v" not in _PROBE:
        _PROBE["v"] = None
        exe = PROBE_EXE
        if _build_probe():
            try:
                out = subprocess.run([exe], capture_output=True, text=True, timeout=120).stdout
                for line in out.splitlines():
                    if line.startswith("{"):
                        _PROBE["v"] = json.loads(line)
            except (OSError, subprocess.TimeoutExpired, ValueError):
                pass
    return _PROBE["v"]


# Per-term instruction mix of each kernel form (lane operations per atom.pixel
# term, counted from the kernel source): FP32 = FP32 FMA/MUL/ADD, DFMA = FP64
# FMA/ADD, IMAD = integer multiply-add, XU = MUFU and FP64->FP32 conversions,
# I2F = int32->FP32 conversions (not a bound: the f32_fast sweep runs two MUFU
# and one I2F per term faster than the probe's MUFU rate allows for three XU
# operations, so I2F issues elsewhere).  "+word": the fixed-point phase word;
# "+narrow": the neighbour pairs' second pixels on the NARROW polynomial.
MIX = {
    # half the terms FP64-anchored, half by FP32 step
    "sf_dpair_kernel": {"fp32": 15, "dfma": 3, "imad": 0.5, "xu": 0.875},
    "sf_dpair_kernel+word": {"fp32": 15.5, "dfma": 1.5, "imad": 0.5, "alu": 0.5, "xu": 0.375, "i2f": 0.5},
    # second pixels on the NARROW polynomial: one FMA fewer per second-pixel term
    "sf_dpair_kernel+word+narrow": {"fp32": 15.0, "dfma": 1.5, "imad": 0.5, "alu": 0.5, "xu": 0.375, "i2f": 0.5},
    # a quarter of the terms FP64-anchored (13 FP32: scale, DHALF, sums); the
    # other three step from the anchor in one 3-FMA chain (16 FP32 with NARROW,
    # 17 with WIDER); the two-pixel step always WIDER
    "sf_dquad_kernel+word/f32": {"fp32": 16.0, "dfma": 0.75, "imad": 0.25, "alu": 0.25, "xu": 0.375, "i2f": 0.25},
    "sf_dquad_kernel+word+narrow/f32": {"fp32": 15.5, "dfma": 0.75, "imad": 0.25, "alu": 0.25, "xu": 0.375,
                                        "i2f": 0.25},
    # f32_fast: pixel 4m on a polynomial, pixels 4m+2 and 4m+3 on MUFU (6 FP32:
    # step, scale to radians, sums; 2 MUFU each); XU also takes the atom's
    # FP64 -> FP32 conversions (3 per 8 terms)
    "sf_dquad_kernel+word/f32_fast": {"fp32": 10.5, "dfma": 0.75, "imad": 0.25, "alu": 0.25, "xu": 1.375,
                                      "i2f": 0.25},
    "sf_dquad_kernel+word+narrow/f32_fast": {"fp32": 10.25, "dfma": 0.75, "imad": 0.25, "alu": 0.25, "xu": 1.375,
                                             "i2f": 0.25},
    # FP64 phase + reduction, DHALF poly
    "sf_dphase_kernel": {"fp32": 12, "dfma": 6, "imad": 1, "xu": 1},
    "sf_dphase_kernel+word/f32": {"fp32": 13, "dfma": 3, "imad": 1, "alu": 1, "i2f": 1},
    "sf_dphase_kernel+word/f32_fast": {"fp32": 4, "dfma": 3, "xu": 2, "i2f": 1},
    "sf_f32x2_kernel/f32": {"fp32": 27, "alu": 2},                   # compensated phase, HALF poly
    "sf_f32x2_kernel/f32_fast": {"fp32": 16, "xu": 2},               # compensated phase, MUFU sin/cos
}


def _kernel_key():
    """MIX key of the structure-factor kernel the last forward ran."""
    from spsim_b200 import core
    return (core.kernel_name() + ("+word" if core.last_phase_word() else "")
            + ("+narrow" if core.last_pair_narrow() else ""))


def balanced_bound(kernel, prec, probe):
    """Terms/s the kernel's own instruction mix allows on the measured pipe
    rates.  FP32, FP64 and integer multiply-add issue through pipes that the
    probe shows to be additive (packed FP32 beside FP64 FMA or FP64 MMA runs at
    the sum of their times), so their times add; the XU pipe (MUFU,
    conversions) runs beside them, so the bound is the larger of the two."""
    if not probe or not probe.get("fma_lane_ops_per_s"):
        return None
    mix = MIX.get("%s/%s" % (kernel, prec)) or MIX.get(kernel)
    if not mix:
        return None
    rate = {"fp32": probe["fma_lane_ops_per_s"], "dfma": probe.get("dfma_lane_ops_per_s"),
            "imad": probe.get("imad_lane_ops_per_s"), "alu": probe.get("alu_lane_ops_per_s"),
            "xu": probe.get("mufu_ops_per_s")}
    t_issue = 0.0
    for k in ("fp32", "dfma", "imad", "alu"):
        if mix.get(k):
            if not rate[k]:
                return None
            t_issue += mix[k] / rate[k]
    t_xu = mix.get("xu", 0) / rate["xu"] if mix.get("xu") else 0.0
    return {"terms_per_s": 1.0 / max(t_issue, t_xu), "mix_per_term": mix,
            "model": "1 / max(sum_p ops_p / rate_p over FP32, FP64, IMAD, ALU; XU ops / XU rate), rates from "
                     "pipe_probe.cu"}


def _peaks(props):
    probe = measured_pipe_peaks()
    if probe and probe.get("fma_lane_ops_per_s") and probe.get("mufu_ops_per_s"):
        p_fma, p_mufu = probe["fma_lane_ops_per_s"], probe["mufu_ops_per_s"]
        src = "measured by pipe_probe.cu at %s MHz (%d SMs)" % (probe.get("clock_mhz"), probe.get("sms"))
        return min(p_fma / OPS_PER_TERM_FMA, p_mufu / OPS_PER_TERM_MUFU), p_mufu, p_fma, probe.get("clock_mhz"), src
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    src = "nominal"
    sm_max = 1965.0
    if os.path.exists(path):
        try:
            mp = json.load(open(path))
            sm_max = float(mp.get("sm_max_mhz", sm_max))
            src = "MEASURED_PEAKS.json sm_max_mhz"
        except (ValueError, OSError):
            pass
    sms = props.multi_processor_count
    p_mufu = sms * MUFU_PER_SM_CLK * sm_max * 1e6
    p_fma = sms * FMA_PER_SM_CLK * sm_max * 1e6
    return min(p_fma / OPS_PER_TERM_FMA, p_mufu / OPS_PER_TERM_MUFU), p_mufu, p_fma, sm_max, src


TRAFFIC_PROFILE = os.path.join(ROOT, "profiles", "sf_dquad_precision50k_traffic.md")


def _traffic_per_launch():
    """DRAM bytes (read + write) of one structure-factor launch on this workload,
    from the committed ncu summary (its "dram bytes per launch:" line)."""
    try:
        for line in open(TRAFFIC_PROFILE):
            if line.lower().startswith("dram bytes per launch:"):
                return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError, IndexError):
        return None
    return None


def run_b200(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pool = None
    nproc = os.cpu_count() or 1
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import multiprocessing as mp

        pool = mp.get_context("spawn").Pool(nproc)  # before the first CUDA call

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    from spsim_b200 import core, synth

    w, Z, pos = _make_workload()
    d = w["det"]
    prec = args.precision
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    rot = synth.haar_rotations(world, 77)[rank] if world > 1 else None
    npix = d["nx"] * d["ny"]
    terms = float(np.count_nonzero(Z)) * npix
    chain = core.chain_params(nx=d["nx"], ny=d["ny"], width=d["width"], height=d["height"], distance=d["distance"],
                              pixel_width=d["width"] / d["nx"], pixel_height=d["height"] / d["ny"],
                              wavelength=d["wavelength"], beam_intensity=1e30, quantum_efficiency=1.0,
                              electron_hole_production_energy=5.8e-19, readout_noise=w["readout_noise"],
                              linear_full_well=2e5, maximum_value=w["full_well_clamp"], clamp_to_maximum=1,
                              exposure_time=1e-3, dark_current=0.0, seed=1234 + rank)
    F = torch.empty(npix, dtype=torch.complex64, device="cuda")
    I = torch.empty(npix, dtype=torch.float32, device="cuda")
    outs = ["photon_count", "real_output", "noiseless_output"]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step(pattern, prec=prec):
        chain.pattern_index = pattern
        core.forward(mol, qs, rot=rot, precision=prec, F=F, I=I)
        return core.detector_chain(chain, I, outputs=outs)

    def timed(prec, steps, warmup):
        for i in range(warmup):
            step(i, prec)
        torch.cuda.synchronize()
        core.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        with core.timing() as kt, ClockSampler(local) as clocks:
            for i, (a, b) in enumerate(evs):
                flush.zero_()  # L2 flush between timed steps, outside the events
                a.record()
                step(warmup + i, prec)
                b.record()
            torch.cuda.synchronize()
            kt.read()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        core.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs)
        if dist:
            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        sf = kt.ms[-steps:] if kt.ms else []
        return ms, (statistics.mean(sf) if sf else None), clocks

    elapsed_ms, sf_avg, clocks = timed(prec, args.steps, args.warmup)
    value = world * args.steps * terms / (elapsed_ms * 1e-3)
    kname = _kernel_key()

    line = None
    if rank == 0:
        props = torch.cuda.get_device_properties(local)
        R, p_mufu, p_fma, sm_max, src = _peaks(props)
        achieved = terms / (sf_avg * 1e-3) if sf_avg else None
        balanced = balanced_bound(kname, prec, measured_pipe_peaks())
        if balanced and achieved:
            balanced["frac"] = achieved / balanced["terms_per_s"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if prec != "fp64" else "f64",
            "data": "synthetic (seeded molecule; no dataset)",
            "config": {"workload": workload_desc(), "precision": prec,
                       "parallelism": "one orientation per rank" if world > 1 else "single GPU",
                       "l2": "flushed between timed steps (256 MiB write outside the timed events)"},
            "roofline": {
                "bound": "sfu", "achieved": achieved, "peak": R, "unit": UNIT,
                "frac": achieved / R if achieved else None, "traffic": _traffic_per_launch(),
                "kernel": kname,
                "kernel_ms": sf_avg,
                "balanced": balanced,
                "peak_source": "R = min(P_FMA/5, P_MUFU/2) terms/s; P_FMA = %.4g FMA lane-ops/s, P_MUFU = %.4g "
                               "ops/s, %s (MEASURED_PEAKS.json has no FP32-FMA or MUFU figure)" % (p_fma, p_mufu, src),
                "peak_nominal": props.multi_processor_count * MUFU_PER_SM_CLK * 1965e6 / OPS_PER_TERM_MUFU,
            },
            "clocks": clocks.summary(),
            "gpu_launches": 3 * args.steps,
        }
    # the other precisions on the same workload, and accuracy against the FP64
    # GPU kernel: single-GPU extras (their timing takes no collective steps the
    # other ranks would have to match)
    extra = _modes(args, core, mol, qs, rot, terms, timed, prec) if world == 1 and not args.no_modes else None
    if rank == 0 and extra:
        line.update(extra)
    # end to end through the reference-facing simulate_shot (host buffers), on every rank
    if not args.no_e2e:
        e2e = _e2e(args, w, Z, pos, terms, world, dist)
        if rank == 0:
            line["e2e"] = e2e
    if rank == 0 and pool is not None:
        v, desc, _ = _cpu_sample(Z, pos, _hkl_host(w), pool, nproc, target_s=12.0)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nproc, "kind": _ref_kind(), "sample": desc}
        pool.close()
    if rank == 0:
        if line.get("fp64_plain"):
            f = line["fp64_plain"]
            f["f32_speedup"] = line["roofline"]["achieved"] / f["kernel_terms_per_s"] if line["roofline"]["achieved"] else None
            if line.get("f32_fast", {}).get("kernel_terms_per_s"):
                f["f32_fast_speedup"] = line["f32_fast"]["kernel_terms_per_s"] / f["kernel_terms_per_s"]
        # the batched workloads at their stated sizes (single-GPU extras: the
        # other ranks of a multi-GPU run would wait on them at the final barrier)
        batched = {}
        if world == 1 and not args.no_batched:
            batched["orientations_20k"] = batched_orientations(prec, line["roofline"]["peak"])
            batched["uneven_64"] = batched_uneven(prec, line["roofline"]["peak"])
            fp64 = line.get("fp64_plain", {}).get("kernel_terms_per_s")
            if fp64:
                # the batched forwards against the plain per-pattern FP64 kernel
                o = batched["orientations_20k"]
                o["vs_fp64_plain"] = o["terms_per_s"] / fp64
                if "f32_fast" in o:
                    o["f32_fast"]["vs_fp64_plain"] = o["f32_fast"]["terms_per_s"] / fp64
        if not args.no_adjoint:
            batched["adjoint_5k"] = batched_adjoint(prec)
        if batched:
            line["batched"] = batched
        line["backward_forward_ratio"] = batched["adjoint_5k"]["backward_forward_ratio"] if "adjoint_5k" in batched \
            else None
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _modes(args, core, mol, qs, rot, terms, timed, prec):
    """f32_fast throughput, the plain FP64 kernel on every 8th pixel, and the
    relative |F|^2 errors of both FP32 modes against that FP64 kernel (itself
    within 2e-7 of the FP64 oracle: tests/test_gpu_sf.py) on every 64th row."""
    import torch

    out = {}
    R = None
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    R = _peaks(props)[0]
    if prec != "f32_fast":
        ms, sf_ms, _ = timed("f32_fast", max(2, args.steps // 2), 1)
        kname = _kernel_key()
        bal = balanced_bound(kname, "f32_fast", measured_pipe_peaks())
        if bal and sf_ms:
            bal["frac"] = terms / (sf_ms * 1e-3) / bal["terms_per_s"]
        out["f32_fast"] = {"value": terms * max(2, args.steps // 2) / (ms * 1e-3), "unit": UNIT,
                           "kernel": kname,
                           "kernel_terms_per_s": terms / (sf_ms * 1e-3) if sf_ms else None,
                           "frac_of_R": terms / (sf_ms * 1e-3) / R if sf_ms else None,
                           "balanced": bal}
    q = qs.q()
    sub_rows = core.QSet.from_list(q.reshape(1024, 1024, 3)[::64].reshape(-1, 3))
    sub8 = core.QSet.from_list(q[::8])
    with core.timing() as t:
        for _ in range(3):
            core.forward(mol, sub8, rot=rot, precision="fp64")
        torch.cuda.synchronize()
    fp64_ms = statistics.median(t.ms[1:])
    fp64_rate = terms / 8 / (fp64_ms * 1e-3)
    _, I64 = core.forward(mol, sub_rows, rot=rot, precision="fp64")
    I64 = I64.double().cpu().numpy()
    acc = {}
    for p in ("f32", "f32_fast"):
        _, Ip = core.forward(mol, sub_rows, rot=rot, precision=p)
        Ip = Ip.double().cpu().numpy()
        den = np.maximum(I64, 1e-3 * I64.mean())
        acc[p] = {"floored_max_rel": float(np.max(np.abs(Ip - I64) / den)),
                  "l2_rel": float(np.linalg.norm(Ip - I64) / np.linalg.norm(I64)),
                  "p99_rel": float(np.percentile(np.abs(Ip - I64) / np.maximum(I64, 1e-30), 99))}
    torch.cuda.synchronize()
    out["accuracy"] = {"reference": "plain FP64 GPU kernel", "pixels": "every 64th detector row (16,384)",
                       "floor": "1e-3 x mean intensity", **acc}
    out["nufft"] = _nufft_mode(core, mol, qs, rot, terms, sub_rows, I64)
    out["fp64_plain"] = {"kernel_terms_per_s": fp64_rate, "sample": "every 8th pixel",
                         "f32_speedup": None, "f32_fast_speedup": None}
    return out


def _nufft_mode(core, mol, qs, rot, terms, sub_rows, I64, eps=1e-8, steps=5):
    """The same structure factor by the type-3 NUFFT (spsim_b200_forward_nufft,
    the reference's use_nfft_for_sf path): device-resident time per pattern
    (CUDA events around the call, L2 flushed between calls), the equivalent
    atom.pixel terms/s, and its |F|^2 error on the accuracy rows."""
    import torch

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    F = torch.empty(qs.npix, dtype=torch.complex64, device="cuda")
    I = torch.empty(qs.npix, dtype=torch.float32, device="cuda")
    for _ in range(3):
        core.forward_nufft(mol, qs, rot=rot, eps=eps, F=F, I=I)
    torch.cuda.synchronize()
    core.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, b in evs:
        flush.zero_()
        a.record()
        core.forward_nufft(mol, qs, rot=rot, eps=eps, F=F, I=I)
        b.record()
    torch.cuda.synchronize()
    core.synchronize()
    ms = statistics.median(a.elapsed_time(b) for a, b in evs)
    w1, w2, n2 = core.last_nufft_grid()
    _, In = core.forward_nufft(mol, sub_rows, rot=rot, eps=eps)
    In = In.double().cpu().numpy()
    den = np.maximum(I64, 1e-3 * I64.mean())
    return {"ms_per_pattern": ms, "equivalent_terms_per_s": terms / (ms * 1e-3), "eps": eps,
            "kernel_widths": [w1, w2], "fft_grid": list(n2),
            "accuracy": {"floored_max_rel": float(np.max(np.abs(In - I64) / den)),
                         "l2_rel": float(np.linalg.norm(In - I64) / np.linalg.norm(I64))},
            "note": "type-3 NUFFT per element (spread; pruned x, y, z FFT passes with the deconvolution and the "
                    "FP32 packing fused; interpolate; FP64 spreading and FFT, "
                    "FP32 interpolation grid), a different algorithm from the direct sum the headline value times"}


def _e2e(args, w, Z, pos, terms, world, dist=None):
    """simulate_shot (src/spsim.c:281) with host buffers: geometry, structure factor
    and the detector chain, every host<->device copy inside the timed region.
    Under torchrun every rank runs it on its own GPU at the same time (barrier
    before, the slowest rank's time after)."""
    import torch

    from spsim_b200 import spsim as S

    d = w["det"]
    opts = S.set_defaults()
    o = opts.contents
    det, exp = o.detector.contents, o.experiment.contents
    det.nx, det.ny, det.nz = d["nx"], d["ny"], 1
    det.width, det.height, det.distance = d["width"], d["height"], d["distance"]
    det.pixel_width = det.pixel_height = d["width"] / d["nx"]
    det.quantum_efficiency, det.electron_hole_production_energy = 1.0, 5.8e-19
    det.readout_noise, det.linear_full_well, det.maximum_value = w["readout_noise"], 2e5, w["full_well_clamp"]
    exp.wavelength, exp.beam_intensity, exp.exposure_time = d["wavelength"], 1e30, 1e-3
    o.verbosity_level = 0
    o.random_seed = 99
    # two copies of the molecule, the second shifted by 1e-13 m, alternate from
    # step to step: the library keeps the last molecule while the caller's atom
    # arrays are unchanged, so alternating makes every step upload its atoms
    mols = [S.get_molecule_from_atoms(Z, pos), S.get_molecule_from_atoms(Z, pos + 1e-13)]
    n = d["nx"] * d["ny"]
    nsteps = max(2, min(args.steps, 5))
    for i in range(2):
        S.free_stuff(S.simulate_shot(mols[i % 2], opts), opts)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t = time.perf_counter()
    for i in range(nsteps):
        S.free_stuff(S.simulate_shot(mols[i % 2], opts), opts)
    wall = (time.perf_counter() - t) / nsteps
    if dist:
        tw = torch.tensor([wall], dtype=torch.float64, device="cuda")
        dist.all_reduce(tw, op=dist.ReduceOp.MAX)
        wall = float(tw.item())
    for m in mols:
        S.free_mol(m)
    # bytes per step up: the new molecule's positions (12 B per atom), its
    # permutation and base weights (8 B per padded atom; the device builds the
    # atom records from them), tiles and form-factor coefficients, and the
    # plan's pattern descriptor (232 B) and work items (16 B per 1,024-pixel
    # tile); down: HKL list, F, |F|^2 and the seven chain arrays
    counts = np.bincount(np.asarray(Z, np.int64), minlength=100)[1:]
    n_pad = int(sum((c + 7) // 8 * 8 for c in counts if c))
    n_tiles = int(sum((c + 7) // 8 * 8 // 128 + (1 if ((c + 7) // 8 * 8) % 128 else 0) for c in counts if c))
    n_elem = int(np.count_nonzero(counts))
    n_items = (n + 1023) // 1024
    return {"value": world * terms / wall, "unit": UNIT,
            "h2d_bytes_per_step": 12 * len(Z) + 8 * n_pad + 16 * n_tiles + 36 * n_elem + 232 + 16 * n_items,
            "d2h_bytes_per_step": 12 * n + 8 * n + 4 * n + 7 * 4 * n,
            "call": "simulate_shot (reference-facing C ABI, host buffers, a new molecule upload every step)",
            "steps": nsteps, "note": "reference semantics: no ADC clamp (extension) in this call"}


PROFILE_VARIANTS = {"f32": (128, 8, 4), "f32_fast": (128, 8, 4)}  # the untuned defaults on the 1024^2 workload


def profile_case(precisions):
    """One forward per precision on the 20,000-atom / 256^2 case (~1.3e9 terms),
    each with the kernel variant the benchmark workload runs by default: a
    short, small-memory command for ncu captures.  "adjoint" instead runs one
    FP32 forward and one adjoint of the refinement shape (5,000 atoms, 512^2
    pixels, 2 orientations, ~2.6e9 terms each)."""
    import torch

    from spsim_b200 import core, synth

    if "nufft" in precisions or "nufft_small" in precisions:
        # the NUFFT structure factor: the 50,000-atom / 1024^2 workload, or the
        # 20,000-atom / 256^2 case; two calls (the first sizes the grids)
        w = synth.WORKLOADS["precision_50k" if "nufft" in precisions else "orientations_20k"]
        Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
        d = w["det"]
        mol = core.Molecule(Z, pos)
        qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
        for _ in range(2):
            core.forward_nufft(mol, qs)
        torch.cuda.synchronize()
        core.synchronize()
        print("profile case ok", core.last_nufft_grid())
        return 0
    if "adjoint" in precisions:
        w = synth.WORKLOADS["adjoint_5k"]
        Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
        d = w["det"]
        mol = core.Molecule(Z, pos, occ=np.ones(len(Z), np.float32))
        qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
        R = synth.haar_rotations(2, w["rot_seed"])
        F, I = core.forward_batch([mol] * 2, [qs] * 2, rots=R, precision="f32")
        core.adjoint(mol, qs, torch.cat(F), torch.rand(2 * qs.npix, device="cuda"), rots=R, precision="f32")
        torch.cuda.synchronize()
        core.synchronize()
        print("profile case ok")
        return 0
    w = synth.WORKLOADS["orientations_20k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    for p in precisions:
        core.set_variant(*PROFILE_VARIANTS[p])
        core.forward(mol, qs, precision=p)
    core.set_variant(-1)
    torch.cuda.synchronize()
    core.synchronize()
    print("profile case ok")
    return 0


def sweep():
    """Kernel-variant sweep on the benchmark workload (structure-factor kernel time)."""
    import torch

    from spsim_b200 import core, synth

    w, Z, pos = _make_workload()
    d = w["det"]
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    terms = float(len(Z)) * d["nx"] * d["ny"]
    R = _peaks(torch.cuda.get_device_properties(0))[0]
    F = torch.empty(qs.npix, dtype=torch.complex64, device="cuda")
    I = torch.empty(qs.npix, device="cuda")
    for prec in ("f32", "f32_fast"):
        for v in [(128, 2, 0), (128, 4, 0), (256, 4, 0), (128, 2, 1), (128, 4, 1), (256, 4, 1), (128, 6, 1),
                  (128, 2, 2), (128, 4, 2), (256, 4, 2), (128, 6, 2), (128, 8, 2), (128, 4, 3), (128, 8, 3),
                  (128, 12, 3), (256, 4, 3), (128, 8, 4), (128, 16, 4), (256, 8, 4)]:
            core.set_variant(*v)
            for _ in range(2):
                core.forward(mol, qs, precision=prec, F=F, I=I)
            torch.cuda.synchronize()
            with core.timing() as t:
                for _ in range(4):
                    core.forward(mol, qs, precision=prec, F=F, I=I)
                torch.cuda.synchronize()
            ms = statistics.median(t.ms)
            print(json.dumps({"precision": prec, "threads": v[0], "pixels_per_thread": v[1], "form": v[2],
                              "ran": list(core.last_variant()), "kernel": _kernel_key(),
                              "ms": ms, "terms_per_s": terms / ms * 1e3, "frac_of_R": terms / ms * 1e3 / R}),
                  flush=True)
    core.set_variant(-1)
    return 0


def _event_timer(stream):
    """ev_time(fn, reps): fn() once untimed, then the median of `reps` runs,
    each bracketed by CUDA events on `stream` (the launching stream)."""
    import torch

    def ev_time(fn, reps=3):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b))
        return statistics.median(ts)

    return ev_time


def batched_orientations(prec, R0, n_orient=None, reps=2, nufft=True):
    """orientations_20k: 20,000 atoms, 256^2 pixels of 150 um at 0.2 m, 0.2 nm,
    n_orient Haar rotations (4,096 by default) in one persistent launch
    (graph-replayed on a side stream), against a loop of single-pattern calls
    (64 timed, scaled to n_orient), and the same orientations by the NUFFT batch."""
    import torch

    from spsim_b200 import core, synth

    w = synth.WORKLOADS["orientations_20k"]
    n_orient = n_orient or w["n_orient"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    mol = core.Molecule(Z, pos)
    qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    R = synth.haar_rotations(n_orient, w["rot_seed"])
    terms = float(len(Z)) * qs.npix * n_orient
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    ev_time = _event_timer(stream)
    Iall = torch.empty(n_orient, qs.npix, device="cuda")
    I = list(Iall.unbind(0))
    with torch.cuda.stream(stream):
        t_batch = ev_time(lambda: core.forward_batch(mol, qs, rots=R, precision=prec, I=I, want_F=False,
                                                     stream=stream), reps=reps)
        kname = _kernel_key()
        nloop = min(n_orient, 64)
        Iloop = torch.empty(qs.npix, device="cuda")
        t_loop = ev_time(lambda: [core.forward(mol, qs, rot=R[i], precision=prec, I=Iloop, want_F=False,
                                               stream=stream) for i in range(nloop)], reps=2) * n_orient / nloop
    def first4_error(Ib):
        # floored max relative |F|^2 error of patterns 0..3 against the FP64 kernel
        errs = []
        with torch.cuda.stream(stream):
            for i in range(4):
                _, I64 = core.forward(mol, qs, rot=R[i], precision="fp64", stream=stream)
                I64 = I64.double()
                errs.append(float(((Ib[i].double() - I64).abs() /
                                   torch.clamp(I64, min=1e-3 * float(I64.mean()))).max()))
            stream.synchronize()
        return max(errs)

    out = {"workload": "orientations_20k: 20,000 atoms, 256^2 pixels of 150 um at 0.2 m, 0.2 nm, %d Haar rotations "
                       "in one batched forward (graph-replayed)" % n_orient,
           "precision": prec, "orientations": n_orient, "kernel": kname, "batch_ms": t_batch,
           "terms_per_s": terms / t_batch * 1e3, "frac_of_R": terms / t_batch * 1e3 / R0,
           "loop_of_single_calls_ms": t_loop, "batch_speedup": t_loop / t_batch,
           "floored_max_rel_vs_fp64_first4": first4_error(Iall)}
    if prec == "f32":
        # the same batch in the fast mode (pixels 4m+2, 4m+3 of each neighbour
        # quad on MUFU sin/cos), with its error on the same patterns
        with torch.cuda.stream(stream):
            t_fast = ev_time(lambda: core.forward_batch(mol, qs, rots=R, precision="f32_fast", I=I, want_F=False,
                                                        stream=stream), reps=reps)
        out["f32_fast"] = {"batch_ms": t_fast, "terms_per_s": terms / t_fast * 1e3,
                           "frac_of_R": terms / t_fast * 1e3 / R0,
                           "floored_max_rel_vs_fp64_first4": first4_error(Iall),
                           "note": "measured here; the fast mode's MUFU bias can reach ~1.7e-5 on random "
                                   "high-|q| neighbour quads, so SPSIM_PREC_F32 is the mode held to 1e-5 everywhere"}
    del Iall, I
    if nufft:
        with torch.cuda.stream(stream):
            Fn, In = core.forward_nufft_batch(mol, qs, R, stream=stream, want_F=False)
            t_nufft = ev_time(lambda: core.forward_nufft_batch(mol, qs, R, I=In, want_F=False, stream=stream),
                              reps=reps)
            errs = []
            for i in range(4):
                _, I64 = core.forward(mol, qs, rot=R[i], precision="fp64", stream=stream)
                I64 = I64.double()
                errs.append(float(((In[i].double() - I64).abs() /
                                   torch.clamp(I64, min=1e-3 * float(I64.mean()))).max()))
            stream.synchronize()
        w1, w2, n2 = core.last_nufft_grid()
        out["nufft_batch"] = {"ms": t_nufft, "equivalent_terms_per_s": terms / t_nufft * 1e3,
                              "speedup_vs_direct_batch": t_batch / t_nufft, "kernel_widths": [w1, w2],
                              "fft_grid": list(n2), "floored_max_rel_vs_fp64_first4": max(errs),
                              "note": "type-3 NUFFT, one grid for every rotation: a different algorithm from the "
                                      "direct sum"}
        del In
    return out


def batched_uneven(prec, R0, reps=3):
    """uneven_64: 64 molecules of 500..100,000 atoms on their own 128^2..1024^2
    detectors and wavelengths, in one batched forward; the batch autotuner
    picks the tile shape first (its choice and the untuned default's time are
    reported)."""
    import torch

    from spsim_b200 import core, synth

    mols, qsets, cost = [], [], 0.0
    for m in synth.uneven_batch():
        Zm, pm = synth.random_molecule(m["natoms"], m["radius"], m["seed"])
        dm = m["det"]
        mols.append(core.Molecule(Zm, pm))
        qsets.append(core.QSet.from_detector(dm["nx"], dm["ny"], dm["width"], dm["height"], dm["distance"],
                                             dm["wavelength"]))
        cost += float(len(Zm)) * qsets[-1].npix
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    ev_time = _event_timer(stream)
    with torch.cuda.stream(stream):
        F, I = core.forward_batch(mols, qsets, precision=prec, want_F=False, stream=stream)
        t_d = ev_time(lambda: core.forward_batch(mols, qsets, precision=prec, I=I, want_F=False, stream=stream),
                      reps=reps)
        try:
            tuned = core.autotune_batch(mols, qsets, precision=prec, stream=stream)
            t_u = ev_time(lambda: core.forward_batch(mols, qsets, precision=prec, I=I, want_F=False, stream=stream),
                          reps=reps)
        finally:
            core.clear_tuning()
    return {"workload": "uneven_64: 64 molecules, 500..100,000 atoms (log-uniform), 128^2..1024^2 detectors, "
                        "lambda 0.1..0.3 nm, one batched forward after autotuning",
            "precision": prec, "terms": cost, "batch_ms": t_u, "terms_per_s": cost / t_u * 1e3,
            "frac_of_R": cost / t_u * 1e3 / R0,
            "autotuned_variant": {"threads": tuned[0], "pixels_per_thread": tuned[1], "form": tuned[2]},
            "untuned_default_ms": t_d}


def batched_adjoint(prec, reps=3):
    """adjoint_5k: 5,000 atoms, 512^2 pixels of 75 um at 0.15 m, 0.25 nm, 256
    orientations, per-atom occupancies and B factors: the batched forward and
    the adjoint (dL/dpos, dL/docc, dL/dB for a given dL/dI), each timed with
    CUDA events; their ratio is the metric's backward/forward time ratio."""
    import torch

    from spsim_b200 import core, synth

    w = synth.WORKLOADS["adjoint_5k"]
    Z, pos = synth.random_molecule(w["natoms"], w["radius"], w["seed"])
    d = w["det"]
    rng = np.random.Generator(np.random.PCG64(w["seed"]))
    mol = core.Molecule(Z, pos, occ=rng.uniform(0.5, 1.0, len(Z)).astype(np.float32),
                        bfac=rng.uniform(0.0, 30.0, len(Z)).astype(np.float32))
    qs = core.QSet.from_detector(d["nx"], d["ny"], d["width"], d["height"], d["distance"], d["wavelength"])
    R = synth.haar_rotations(w["n_orient"], w["rot_seed"])
    terms = float(len(Z)) * qs.npix * len(R)
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())
    ev_time = _event_timer(stream)
    with torch.cuda.stream(stream):
        Fall = torch.empty(len(R), qs.npix, dtype=torch.complex64, device="cuda")
        Iall = torch.empty(len(R), qs.npix, device="cuda")
        F, I = list(Fall.unbind(0)), list(Iall.unbind(0))
        G = torch.rand(len(R) * qs.npix, device="cuda")
        t_f = ev_time(lambda: core.forward_batch(mol, qs, rots=R, precision=prec, F=F, I=I, stream=stream), reps=reps)
        t_b = ev_time(lambda: core.adjoint(mol, qs, Fall.reshape(-1), G, rots=R, precision=prec, stream=stream),
                      reps=reps)
    return {"workload": "adjoint_5k: 5,000 atoms, 512^2 pixels, 256 orientations, per-atom occupancies and B "
                        "factors: batched forward and adjoint",
            "precision": prec, "orientations": len(R), "forward_ms": t_f, "adjoint_ms": t_b,
            "backward_forward_ratio": t_b / t_f, "forward_terms_per_s": terms / t_f * 1e3,
            "adjoint_terms_per_s": terms / t_b * 1e3}


def workloads(prec, n_orient=None):
    """The batched workloads, one JSON line each (batched_orientations,
    batched_uneven, batched_adjoint)."""
    import torch

    R0 = _peaks(torch.cuda.get_device_properties(0))[0]
    print(json.dumps(batched_orientations(prec, R0, n_orient)), flush=True)
    print(json.dumps(batched_uneven(prec, R0)), flush=True)
    print(json.dumps(batched_adjoint(prec)), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="f32", choices=["f32", "f32_fast", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched orientation and uneven workloads")
    ap.add_argument("--no-modes", action="store_true", help="skip the f32_fast / fp64 / accuracy extras")
    ap.add_argument("--profile-case", default=None,
                    help="comma-separated precisions: one forward each on the 20,000-atom x 256^2 case, or "
                         "\"adjoint\": one forward and one adjoint of the 5,000-atom refinement shape, "
                         "\"nufft\" / \"nufft_small\": two NUFFT forwards of the 50,000-atom / 1024^2 workload or "
                         "the 20,000-atom / 256^2 case (for ncu)")
    ap.add_argument("--sweep", action="store_true", help="time every compiled FP32 kernel variant")
    ap.add_argument("--workloads", action="store_true", help="time the batched workloads (orientations, uneven, "
                                                              "adjoint)")
    args = ap.parse_args()
    if args.workloads:
        return workloads(args.precision)
    if args.profile_case:
        return profile_case(args.profile_case.split(","))
    if args.sweep:
        return sweep()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
