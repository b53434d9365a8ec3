"""Benchmark of the B200 dual-resolution GP-HMC sampler.

Workload (default, "batched64"): 64 independent HMC chains on the seeded
synthetic 32^3 @ 1 mm volume (RBF 0.806/0.132/1, 64^3 embedding, ellipsoid mask
~60 %, noise 0.5 / 0.3, kriging radius 6.9 mm), leapfrog 25, burnin 500,
nsave 500, thin 3.  A step is one HMC iteration of every chain (one
MultiResParameters::update + HMCParameters::update per chain).  Metric: HMC
gradient evaluations per second (sum over chains of L + 1 per iteration).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload batched64|single_c1|single_c2|served|served_c1|served_c3] [--no-ess]

Served workloads ("served": the C4 size/parameter distribution; "served_c1":
one-chain fits of 32^3 images; "served_c3": fits of the batched size, 64
chains on each request's own 32^3 image): --steps jobs arrive as a Poisson
process (20 jobs/s) at
a continuous-batching server; after --warmup untimed jobs, the line reports
fits completed per second, gradient evaluations per second over the makespan,
and p50/p99 job latency (submission to result on the host).

Under torchrun each rank runs its own 64-chain set on its GPU (chains are
independent: no collective on the data path, weak scaling); the timed region
is bracketed by barriers and the max over ranks is reported.

--impl reference times the reference algorithm on the host CPU: the oracle's
FP32 restatement of MultiResParameters<float>::update (the `dualgpmf`
build: four FFTs per leapfrog step, OpenMP), all host threads, one chain and
one iteration per step (a bounded sample of the same workload).  The
reference itself cannot be built in this image (Eigen, FFTW3, Boost and NLopt
are absent), so the restatement stands in for it.
"""
from __future__ import annotations

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

METRIC = "HMC gradient evals/sec"
UNIT = "grad_evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched64", choices=sorted(WORKLOADS))
    ap.add_argument("--rate", type=float, default=-1.0, help="served workloads: arrivals per second")
    ap.add_argument("--no-ess", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="host time of each timed part of the CPU baseline (one chain; independent chains)")
    ap.add_argument("--no-served", action="store_true", help="skip the short served stream in the batched line")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--profile-kernel", type=int, default=-1,
                    help="set up, run --warmup iterations, then launch kernel K of the leapfrog step 4 times "
                         "(for ncu: its launches are the last ones of that kernel name)")
    return ap.parse_args()


# ------------------------------------------------------------------ distributed plumbing
class Dist:
    def __init__(self, backend):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            if backend == "nccl":
                import torch
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.pg = dist
        self.backend = backend

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x):
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x):
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ------------------------------------------------------------------ workloads
WORKLOADS = {
    "batched64": dict(chains=64, vol="c1", burnin=500, nsave=500, thin=3, leapfrog=25),
    "single_c1": dict(chains=1, vol="c1", burnin=200, nsave=200, thin=1, leapfrog=25),
    "single_c2": dict(chains=1, vol="c2", burnin=200, nsave=200, thin=1, leapfrog=25),
    "tiny": dict(chains=2, vol="small", burnin=10, nsave=10, thin=1, leapfrog=5),  # test-sized
    # the largest class of the uneven batch (80x80x64 latent, 256x256x128 embedding: the x-line path), 4 chains
    "xline256": dict(chains=4, vol="x256", burnin=300, nsave=300, thin=3, leapfrog=25),
    # served streams: a step is one job; jobs arrive as a Poisson process
    "served": dict(chains=1, vol="c4", burnin=300, nsave=300, thin=3, leapfrog=25, rate=20.0),
    "served_c1": dict(chains=1, vol="c1", burnin=300, nsave=300, thin=3, leapfrog=25, rate=20.0),
    # jobs of the batched size: 64 chains on each request's own 32^3 image (one fit of the batched configuration)
    "served_c3": dict(chains=64, vol="c1", burnin=300, nsave=300, thin=3, leapfrog=25, rate=20.0),
    "served_tiny": dict(chains=1, vol="small", burnin=20, nsave=20, thin=1, leapfrog=5, rate=50.0),  # test-sized
    # config 4: 32 volumes of the uneven size/parameter distribution fitted together (all submitted at once)
    "uneven32": dict(chains=1, vol="c4", burnin=300, nsave=300, thin=3, leapfrog=25, rate=float("inf"), jobs=32),
}


def make_volume(name):
    from dualres_b200 import synth
    if name == "small":
        return synth.small_volume()
    if name == "c4":
        return synth.config_c4_volume(0)
    if name == "x256":
        return synth.make_volume((80, 80, 64), 1.0, (1.0, 0.35, 1.4), 0.6, 0.4, 6.9, "ellipsoid", 0.60, 5, name="x256")
    return synth.config_c1() if name == "c1" else synth.config_c2()


def config_of(w, extra=None):
    vol = WORKLOADS[w]["vol"]
    desc = {"c1": ("32x32x32 @ 1mm", "64^3", [0.806, 0.132, 1.0], 6.9),
            "c2": ("64x64x48 @ 1.5mm", "128^3", [1.0, 0.4, 1.5], 6.9),
            "small": ("10x9x7 @ 1mm", "32x16x16", [0.8, 0.3, 1.0], 3.2),
            "x256": ("80x80x64 @ 1mm", "256x256x128", [1.0, 0.35, 1.4], 6.9),
            "c4": ("uniform over 32^3, 48x48x40, 64x64x48, 80x80x64 @ 1mm", "64^3 .. 256x256x128",
                   "RBF v=1, b~U[0.1,0.6], e~U[1,2]", 6.9)}[vol]
    cfg = {"workload": w, **{k: v for k, v in WORKLOADS[w].items()},
           "latent_grid": desc[0], "embedding": desc[1], "covariance": desc[2],
           "neighborhood_mm": desc[3], "parallelism": "independent chains per GPU (no collective)"}
    if extra:
        cfg.update(extra)
    return cfg


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()  # the first sample arrives once nvidia-smi is up: start timing after it
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        try:  # one more sample at the end of the timed region
            out = subprocess.run(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                  "-i", str(self.gpu)], capture_output=True, text=True, timeout=10).stdout
            self.lines.extend(ln.strip() for ln in out.splitlines())
        except Exception:
            pass
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ ESS
def ess_geyer(x):
    """ESS of one chain (Geyer initial monotone sequence over the FFT autocorrelation); x: (n, V)."""
    n = x.shape[0]
    x = x - x.mean(axis=0)
    f = np.fft.rfft(x, n=2 * n, axis=0)
    ac = np.fft.irfft(f * np.conj(f), axis=0)[:n] / n
    var = ac[0]
    ok = var > 0
    rho = np.where(ok, ac / np.where(ok, var, 1.0), 0.0)
    m = (n - 1) // 2
    pairs = rho[0:2 * m:2] + rho[1:2 * m:2]           # Gamma_k = rho_2k + rho_2k+1
    pos = pairs > 0
    first_neg = np.where(pos.all(axis=0), m, np.argmin(pos, axis=0))
    keep = np.arange(m)[:, None] < first_neg[None, :]   # initial positive sequence
    # initial monotone sequence: running minimum over the kept pairs; pairs past the truncation count zero
    pairs = np.minimum.accumulate(np.where(keep, pairs, np.inf), axis=0)
    pairs = np.where(keep, pairs, 0.0)
    tau = -1.0 + 2.0 * pairs.sum(axis=0)
    tau = np.maximum(tau, 1.0 / np.log10(max(n, 10)))
    return np.where(ok, n / tau, 0.0)


# ------------------------------------------------------------------ our arm
def run_ours(args, dist):
    import dualres_b200 as d
    wl = WORKLOADS[args.workload]
    C = wl["chains"]
    hmc = d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"], leapfrog=wl["leapfrog"],
                          seed=args.seed + 7919 * dist.rank)
    vol = make_volume(wl["vol"])
    d.lib()
    import ctypes
    dev = dist.local  # one process per GPU: the library works on this rank's device

    # ---- process warm-up (untimed): CUDA context, module loading, per-device tables
    from dualres_b200 import synth as _synth
    _wd = d.MultiResData.from_volume(_synth.small_volume(), device=dev)
    _wc = d.MultiResParameters(_wd, d.HMCParameters(burnin=2, nsave=1, thin=1, leapfrog=2, seed=1), 1)
    _wc.update(1)
    _wc.close()
    _wd.close()

    # ---- end to end through the C ABI with host buffers: volume + chains + K iterations,
    # each followed by a device->host read of every chain's statistics; then the summary.
    dist.barrier()
    t0 = time.perf_counter()
    data = d.MultiResData.from_volume(vol, device=dev)
    t_vol = time.perf_counter()
    chains = d.MultiResParameters(data, hmc, C)
    t_cs = time.perf_counter()
    stats = None
    for _ in range(args.warmup + args.steps):
        chains.update(1)
        stats = chains.stats()
    summ = chains.summary(-1)
    t_e2e = time.perf_counter() - t0
    e2e_parts = {"volume": round(t_vol - t0, 4), "chain_set_incl_tuning": round(t_cs - t_vol, 4),
                 "iterations_and_reads": round(t0 + t_e2e - t_cs, 4)}
    grads_e2e = sum(s["grad_evals"] for s in stats)
    img_bytes = sum(a.nbytes for a in (vol.highres, vol.stdres))
    stat_bytes = C * ctypes.sizeof(d.api.ChainStats)
    t_e2e = dist.max(t_e2e)
    grads_e2e = dist.sum(grads_e2e)

    # ---- device-timed steps on the warm chain set
    chains.update(args.warmup)
    st0 = chains.stats()
    launches0 = d.kernel_launches()
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    dist.barrier()
    clk.start()
    ms = chains.update_timed(args.steps)
    clocks = clk.stop()
    launches = d.kernel_launches() - launches0
    st1 = chains.stats()
    grads = sum(b["grad_evals"] - a["grad_evals"] for a, b in zip(st0, st1))
    t_max = dist.max(ms / 1e3)
    grads_all = dist.sum(grads)
    value = grads_all / t_max

    extra = {}
    # ---- the plain GPU form (B2): the reference algorithm ported plainly to the GPU (four FFTs per step), one chain
    try:
        r_plain, ms_plain = plain_gpu_rate(data, wl["leapfrog"], 10, device=dev)
        extra["plain_gpu_single_chain"] = {
            "value": r_plain, "unit": UNIT, "ms_per_iteration": ms_plain,
            "batched_over_plain": (grads / (ms / 1e3)) / r_plain,
            "what": "reference algorithm on the GPU: torch.fft (cuFFT) 3D transforms, 4 per leapfrog step, sparse CSR "
                    "kriging products, host accept each iteration (bench.py PlainGPU)"}
    except Exception as e:  # the comparator must not break the benchmark line
        extra["plain_gpu_single_chain"] = {"error": str(e)[:200]}
    # ---- the plain single-chain GPU form on the same volume (same kernels, one chain)
    if C > 1:
        one = d.MultiResParameters(data, d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"],
                                                         leapfrog=wl["leapfrog"], seed=args.seed + 3), 1)
        one.update(args.warmup)
        a = one.stats()[0]["grad_evals"]
        one_ms = one.update_timed(args.steps)
        g1 = one.stats()[0]["grad_evals"] - a
        r1 = g1 / (one_ms / 1e3)
        extra["single_chain_gpu"] = {"value": r1, "unit": UNIT, "ms_per_step": one_ms / args.steps,
                                     "batched_over_single": (grads / (ms / 1e3)) / r1}
        one.close()

    # ---- ESS/s of voxelwise posterior means on the full configured job (fresh chain set)
    if not args.no_ess and dist.rank == 0:
        hmc2 = d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"], leapfrog=wl["leapfrog"],
                               seed=args.seed + 1, store_samples=True)
        job = d.MultiResParameters(data, hmc2, C)
        total_iters = wl["burnin"] + wl["thin"] * wl["nsave"]
        job_ms = job.update_timed(total_iters)
        st = job.stats()
        rng = np.random.default_rng(0)
        vox = np.sort(rng.choice(data.n_output, size=min(2000, data.n_output), replace=False))
        ess = np.zeros(len(vox))
        for c in range(C):
            s = job.samples(c)[:, vox].astype(np.float64)
            ess += ess_geyer(s)
        extra["ess"] = {"median": float(np.median(ess)), "min": float(np.min(ess)), "voxels": int(len(vox)),
                        "job_seconds": job_ms / 1e3, "iterations": total_iters,
                        "mh_rate": float(np.mean([x["mh_rate"] for x in st])),
                        "eps": float(np.mean([x["eps"] for x in st]))}
        extra["ess_per_sec"] = {"median": float(np.median(ess)) / (job_ms / 1e3),
                                "min": float(np.min(ess)) / (job_ms / 1e3)}
        extra["job_grad_evals_per_sec"] = sum(x["grad_evals"] for x in st) / (job_ms / 1e3)
        job.close()

    # ---- a short served stream of fits of the same volume class (continuous batching through dr_server_*)
    if not args.no_served and dist.world == 1 and C > 1:
        try:
            srv = served_sample("served_c1", 12, 2, args.seed + 11, dev)
            srv["over_plain_gpu"] = srv["value"] / extra["plain_gpu_single_chain"]["value"] \
                if "value" in extra.get("plain_gpu_single_chain", {}) else None
            extra["served_c1"] = srv
        except Exception as e:  # an extra must not break the benchmark line
            extra["served_c1"] = {"error": str(e)[:200]}
        try:  # three fits of the batched size (64 chains each) arriving together; tuning is cached from above
            srv = served_sample("served_c3", 3, 0, args.seed + 13, dev)
            srv["over_plain_gpu"] = srv["value"] / extra["plain_gpu_single_chain"]["value"] \
                if "value" in extra.get("plain_gpu_single_chain", {}) else None
            extra["served_c3"] = srv
        except Exception as e:  # an extra must not break the benchmark line
            extra["served_c3"] = {"error": str(e)[:200]}

    # ---- roofline of the dominant kernel (timed live with CUDA events on the library stream)
    per_iter = {}
    L = wl["leapfrog"]
    launches_per_iter = [L + 1, L, L, L + 1, L + 1, L + 1, L + 1]
    peak = peaks()
    for k in range(7):
        kms, kbytes = d.api.time_kernel(chains, k, step=1, reps=20)
        per_iter[k] = (kms * launches_per_iter[k], kms, kbytes)
    dom = max(per_iter, key=lambda k: per_iter[k][0])
    _, kms, kbytes = per_iter[dom]
    achieved = kbytes / (kms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": d.api.KERNEL_NAMES[dom], "achieved": achieved, "peak": peak[0],
                "unit": "GB/s", "frac": achieved / peak[0], "peak_source": peak[1],
                "algorithmic_bytes_per_launch": kbytes, "launch_ms": kms,
                "traffic": traffic_from_profile(), "kernels": {
                    d.api.KERNEL_NAMES[k]: {"ms_per_launch": v[1], "ms_per_iteration": v[0],
                                            "GBps_algorithmic": v[2] / (v[1] / 1e3) / 1e9}
                    for k, v in per_iter.items()}}
    info = data.info
    try:  # the same rate in the reference's byte model (four FFTs per step); the spectral formulation moves less
        b_ref = reference_bytes_per_step(int(info.N), int(info.kriging_nnz), C, int(info.n_highres),
                                         int(info.n_stdres))
        gbs_ref = b_ref * grads / (ms / 1e3) / 1e9   # one gradient evaluation per leapfrog step, this GPU
        roofline["reference_formulation"] = {"bytes_per_chain_step": b_ref, "equivalent_GBps": gbs_ref,
                                             "frac_of_peak": gbs_ref / peak[0]}
    except Exception as e:  # an accounting extra must not break the benchmark line
        roofline["reference_formulation"] = {"error": str(e)[:200]}
    cfg = config_of(args.workload, {
        "global_batch": C * dist.world, "l2": "working set larger than L2 (state 0.5 GB per GPU)",
        "n_highres": info.n_highres, "n_stdres": info.n_stdres, "kriging_nnz": int(info.kriging_nnz),
        "setup_seconds": info.setup_seconds, "kriging_seconds": info.kriging_seconds,
        "chain_set_config": chains.config()})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded GP draw)",
        "config": cfg,
        "e2e": {"value": grads_e2e / t_e2e, "unit": UNIT, "seconds": t_e2e,
                "h2d_bytes_per_step": int(img_bytes / (args.warmup + args.steps)),
                "d2h_bytes_per_step": int(stat_bytes),
                "includes": "in a warm process: volume upload + kriging + FP64 spectrum + chain-set tuning and init "
                            "+ every iteration (dr_step + d2h chain statistics) + summary d2h",
                "seconds_by_part": e2e_parts},
        "roofline": roofline, "gpu_launches": int(launches), "clocks": clocks,
        "grad_evals_per_step": grads_all / args.steps, **extra,
    }
    chains.close()
    data.close()
    return line



# ------------------------------------------------------------------ plain single-chain GPU baseline
class PlainGPU:
    """The reference's single-chain algorithm ported to the GPU the plain way (the B2 arm): mu and p kept in real
    space, four full 3D FFTs per leapfrog step (cuFFT through torch.fft), the kriging products as sparse CSR
    matrix-vector products, the accept decision read back every iteration.  It follows the restated algorithm of
    MultiResParameters::update (include/dualres/MultiResParameters.h:337-376, 674-727, 784-859) on the volume the
    library prepared (its indices, data, kriging matrix and FP64 eigenvalues).  A comparator for the benchmark,
    not part of the library."""

    def __init__(self, data, device="cuda:0"):
        import warnings

        import torch
        warnings.filterwarnings("ignore", message=".*[Ss]parse.*")
        self.t = torch
        self.dev = device
        lam = torch.tensor(data.lambda_re(), dtype=torch.float32, device=device)
        self.live = lam > 0
        self.inv_lam = torch.where(self.live, 1.0 / lam, torch.zeros_like(lam))
        self.N = lam.numel()
        self.shape = tuple(lam.shape)
        d_idx, _ = data.indices()
        self.D = torch.tensor(d_idx.astype(np.int64), device=device)
        yh, ys = data.data()
        self.Yh = torch.tensor(yh, device=device)
        self.Ys = torch.tensor(ys, device=device)
        self.dual = len(ys) > 0
        if self.dual:
            rp, col, val = data.W()
            W = torch.sparse_csr_tensor(torch.tensor(rp.astype(np.int64)), torch.tensor(col.astype(np.int64)),
                                        torch.tensor(val), size=(len(ys), len(yh)))
            self.W = W.to(device)
            self.WT = W.to_sparse_coo().t().coalesce().to_sparse_csr().to(device)

    def dft_plus(self, x):   # unnormalised inverse transform (FFTW sign +)
        return self.t.fft.ifftn(x, norm="forward")

    def dft_minus(self, x):  # unnormalised forward transform (FFTW sign -)
        return self.t.fft.fftn(x, norm="backward")

    def residuals(self, mu):
        muD = mu.real.reshape(-1)[self.D]
        rh = self.Yh - muD
        rs = self.Ys - (self.W @ muD.unsqueeze(1)).squeeze(1) if self.dual else None
        return rh, rs

    def gradient(self, mu, sh, ss):
        t = self.t
        u = self.dft_plus(mu)
        g = self.dft_minus(t.where(self.live, u * (-self.inv_lam / self.N), t.zeros_like(u)))
        rh, rs = self.residuals(mu)
        dg = sh * rh + (ss * (self.WT @ rs.unsqueeze(1)).squeeze(1) if self.dual else 0.0)
        gr = t.zeros(self.N, dtype=t.float32, device=self.dev)
        gr.index_add_(0, self.D, dg)
        return g + gr.reshape(self.shape)

    def log_post(self, mu, sh, ss):
        t = self.t
        u = self.dft_plus(mu)
        lp = -0.5 / self.N * t.sum(t.where(self.live, (u.real ** 2 + u.imag ** 2) * self.inv_lam,
                                            t.zeros_like(self.inv_lam)), dtype=t.float64)
        rh, rs = self.residuals(mu)
        ll = -0.5 * sh * t.sum(rh.double() ** 2)
        if self.dual:
            ll = ll - 0.5 * ss * t.sum(rs.double() ** 2)
        return lp + ll, rh, rs

    def iteration(self, mu, sh, ss, eps, L, gen):
        t = self.t
        lam_m = t.where(self.live, self.inv_lam + sh, t.zeros_like(self.inv_lam))
        inv_lam_m = t.where(self.live, 1.0 / t.where(self.live, lam_m, t.ones_like(lam_m)), t.zeros_like(lam_m))
        z = t.complex(t.randn(self.shape, generator=gen, device=self.dev), t.randn(self.shape, generator=gen, device=self.dev))
        e0 = -0.5 * t.sum((z.real ** 2 + z.imag ** 2).double())
        p = self.dft_minus(t.where(self.live, t.sqrt(lam_m) * self.dft_plus(z) / self.N, t.zeros_like(z)))
        h0, _, _ = self.log_post(mu, sh, ss)
        mu1 = mu
        p = p + 0.5 * eps * self.gradient(mu1, sh, ss)
        for s in range(1, L + 1):
            mu1 = mu1 + self.dft_minus(t.where(self.live, self.dft_plus(p) * (eps * inv_lam_m / self.N), t.zeros_like(p)))
            p = p + (0.5 if s == L else 1.0) * eps * self.gradient(mu1, sh, ss)
        q = self.dft_plus(p)
        kin = -0.5 / self.N * t.sum(t.where(self.live, (q.real ** 2 + q.imag ** 2) * inv_lam_m,
                                           t.zeros_like(inv_lam_m)), dtype=t.float64)
        h1, rh, rs = self.log_post(mu1, sh, ss)
        log_r = float(h1 + kin - (e0 + h0))
        accept = np.log(float(t.rand((), generator=gen, device=self.dev))) < log_r
        if accept:
            mu = mu1
        rh, rs = self.residuals(mu)
        sh = float(t.distributions.Gamma(len(self.Yh) / 2 + 1, 0.5 * t.sum(rh ** 2)).sample())
        if self.dual:
            ss = float(t.distributions.Gamma(len(self.Ys) / 2 + 1, 0.5 * t.sum(rs ** 2)).sample())
        return mu, sh, ss


def plain_gpu_rate(data, L, iters, seed=3, device=0):
    """Gradient evaluations per second of PlainGPU on one chain (CUDA events, after 2 warm-up iterations)."""
    import torch
    dev = f"cuda:{device}"
    pg = PlainGPU(data, dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    yh, _ = data.data()
    mr = torch.zeros(pg.N, dtype=torch.float32, device=dev)
    mr[pg.D] = torch.tensor(yh, device=dev)
    mu = torch.complex(mr.reshape(pg.shape), torch.zeros_like(mr).reshape(pg.shape))
    sh, ss, eps = 2.0, 5.0, 0.02
    for _ in range(2):
        mu, sh, ss = pg.iteration(mu, sh, ss, eps, L, gen)
    with torch.cuda.device(device):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(iters):
            mu, sh, ss = pg.iteration(mu, sh, ss, eps, L, gen)
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    return iters * (L + 1) / (ms / 1e3), ms / iters


# ------------------------------------------------------------------ served stream
def served_volume(wl, i, seed):
    from dualres_b200 import synth
    if wl["vol"] == "c4":
        return synth.config_c4_volume(i, seed=seed)
    if wl["vol"] == "small":
        return synth.small_volume(seed=seed + i)
    return synth.config_c1(seed=seed + i)  # each request its own image (same geometry class)


def run_served(args, dist):
    import dualres_b200 as d
    wl = WORKLOADS[args.workload]
    rate = args.rate if args.rate > 0 else wl["rate"]
    if "jobs" in wl:
        args.steps = wl["jobs"]
    hmc = lambda i: d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"],  # noqa: E731
                                    leapfrog=wl["leapfrog"], seed=args.seed + 7919 * dist.rank + i)
    t0 = time.perf_counter()
    vols = [served_volume(wl, i, args.seed + dist.rank * 100003) for i in range(args.warmup + args.steps)]
    gen_s = time.perf_counter() - t0
    rng = np.random.default_rng(args.seed + dist.rank)
    gaps = rng.exponential(1.0 / rate, size=args.steps) if np.isfinite(rate) else np.zeros(args.steps)
    sv = d.Server(device=dist.local, iterations_per_round=8, host_threads=4)
    # warm-up jobs (untimed): library tables, pools, first graphs
    for i in range(args.warmup):
        sv.submit_volume(vols[i], hmc(i), wl["chains"])
    sv.drain(3600)
    st0 = sv.stats()
    clk = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
    dist.barrier()
    clk.start()
    t_start = time.perf_counter()
    ids = []
    t_next = t_start
    for k in range(args.steps):
        t_next += gaps[k]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        ids.append(sv.submit_volume(vols[args.warmup + k], hmc(args.warmup + k), wl["chains"]))
    sv.drain(3600)
    makespan = time.perf_counter() - t_start
    clocks = clk.stop()
    st1 = sv.stats()
    res = [sv.result(j) for j in ids]
    lat = np.array([r.latency_s for r in res])
    queue = np.array([r.queue_s for r in res])
    grads = sum(r.grad_evals for r in res)
    sizes = [v.highres.shape for v in vols[args.warmup:]]
    makespan = dist.max(makespan)
    grads_all = dist.sum(grads)
    jobs_all = dist.sum(len(ids))
    img_bytes = sum(v.highres.nbytes + (v.stdres.nbytes if v.stdres is not None else 0) for v in vols[args.warmup:])
    out_bytes = sum(3 * 4 * len(r.mean) for r in res)
    line = {
        "metric": "served HMC gradient evals/sec", "value": grads_all / makespan, "unit": UNIT,
        "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": makespan * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded GP draws)",
        "config": config_of(args.workload, {"arrival_rate_per_s": rate, "jobs": args.steps,
                                            "grids": [list(s[::-1]) for s in sizes],
                                            "l2": "every job's state is its own; total resident state above L2",
                                            "volume_generation_seconds": gen_s}),
        "jobs_per_s": jobs_all / makespan,
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max()), "mean": float(lat.mean())},
        "queue_s": {"p50": float(np.percentile(queue, 50)), "p99": float(np.percentile(queue, 99))},
        "mh_rate": {"median": float(np.median([r.mh_rate for r in res]))},
        "server": {"peak_running": int(st1.peak_running), "peak_device_bytes": int(st1.peak_device_bytes),
                   "failed": int(st1.failed - st0.failed)},
        "e2e": {"value": grads_all / makespan, "unit": UNIT,
                "h2d_bytes_per_step": int(img_bytes / args.steps), "d2h_bytes_per_step": int(out_bytes / args.steps),
                "includes": "arrival process + host set-up (masks, kriging) + device set-up + sampling + result d2h"},
        "gpu_launches": int(st1.kernel_launches - st0.kernel_launches), "clocks": clocks,
    }
    sv.close()
    return line, vols[args.warmup:]


def served_cpu_baseline(job_vols, wl, target_s=12.0):
    """The CPU restatement on one served job's image (the smallest of the stream, which bounds the time of the FP64
    check), with the FP32 kernels' posterior-mean error against the FP64 oracle on that image: a served job runs the
    same kernels as a direct fit, with bit-identical results."""
    import dualres_b200 as d
    vol = min(job_vols, key=lambda v: v.highres.size)
    dv = d.MultiResData.from_volume(vol)
    rp, col, val = dv.W()
    n_embed = int(np.prod(dv.shape))
    dv.close()
    pm = (12, wl["leapfrog"]) if n_embed <= 64 ** 3 else (4, 10)
    line = cpu_baseline_line(vol, (rp, col, val.astype(np.float32)), wl["leapfrog"], target_s=target_s,
                             pm_iters=pm[0], pm_L=pm[1])
    line["sample"] = "one served job's image (grid %s, the smallest of the stream): %s" % (
        "x".join(str(x) for x in vol.highres.shape[::-1]), line["sample"])
    return line


def served_sample(workload, jobs, warmup_jobs, seed, device, rate=None):
    """A short served stream for the default benchmark line: `jobs` fits of `workload` arriving as a Poisson process,
    after `warmup_jobs` untimed ones; gradient evaluations per second over the makespan, fits per second, latency."""
    import dualres_b200 as d
    wl = WORKLOADS[workload]
    rate = wl["rate"] if rate is None else rate
    hmc = lambda i: d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"],  # noqa: E731
                                    leapfrog=wl["leapfrog"], seed=seed + i)
    vols = [served_volume(wl, i, seed) for i in range(warmup_jobs + jobs)]
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, size=jobs)
    sv = d.Server(device=device, iterations_per_round=8, host_threads=4)
    for i in range(warmup_jobs):
        sv.submit_volume(vols[i], hmc(i), wl["chains"])
    sv.drain(3600)
    t_start = time.perf_counter()
    t_next, ids = t_start, []
    for k in range(jobs):
        t_next += gaps[k]
        dt = t_next - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        ids.append(sv.submit_volume(vols[warmup_jobs + k], hmc(warmup_jobs + k), wl["chains"]))
    sv.drain(3600)
    makespan = time.perf_counter() - t_start
    res = [sv.result(j) for j in ids]
    sv.close()
    lat = np.array([r.latency_s for r in res])
    grads = sum(r.grad_evals for r in res)
    return {"workload": workload, "jobs": jobs, "arrival_rate_per_s": rate, "value": grads / makespan, "unit": UNIT,
            "fits_per_s": jobs / makespan, "makespan_s": makespan,
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "what": "a dualgpmf fit per job (%d chain%s, burnin %d, nsave %d, thin %d, L %d) through dr_server_*; "
                    "gradient evaluations over the makespan from the first arrival to the last result"
                    % (wl["chains"], "" if wl["chains"] == 1 else "s", wl["burnin"], wl["nsave"], wl["thin"],
                       wl["leapfrog"])}


def reference_bytes_per_step(N, nnz, chains, n_h, n_s):
    """Algorithmic bytes of one leapfrog step of one chain in the reference's formulation (four full complex64 3D
    FFTs per step, real-space state): 104 N + 16 nnz / C + 12 n_h + 8 n_s, with the kriging matrix (values and
    columns, read for W x and W^T r) shared by the C chains of one volume."""
    return 104.0 * N + 16.0 * nnz / chains + 12.0 * n_h + 8.0 * n_s


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f).get("bytes_per_launch")
    except Exception:
        return None


# ------------------------------------------------------------------ CPU (oracle restatement)
def oracle_model(vol, W=None, precision="f"):
    from oracle import oracle as o
    prep = o.prepare(vol.highres)
    if W is None:
        W = o.kriging(prep["masked"], vol.qform_hr, vol.stdres, vol.qform_sr, vol.theta, vol.radius)
    ys = vol.stdres.ravel()[~(np.isnan(vol.stdres.ravel()) | (vol.stdres.ravel() == 0))]
    m = o.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, W, prep["O"], precision=precision)
    return m, prep


def cpu_rate(m, iters, L, threads, seed=5):
    from oracle import oracle as o
    o.set_threads(threads)
    rng = np.random.default_rng(seed)
    mu = (rng.standard_normal(m.shape) * 0.1).astype(np.complex64)
    m.set_mu(mu)
    m.set_sigma(2.0, 5.0)
    t0 = time.perf_counter()
    g = m.run_iterations(iters, L, 0.02, seed)
    dt = time.perf_counter() - t0
    return g / dt, dt, g


def cpu_throughput(vol, W, L, cores, target_s=10.0):
    """Gradient evaluations per second of `cores` independent single-threaded chains of the FP32 restatement run
    side by side (one host thread each; ctypes releases the GIL during the C calls), each for about target_s."""
    import threading
    from oracle import oracle as o
    models = [oracle_model(vol, W)[0] for _ in range(cores)]
    o.set_threads(1)
    _, dt1, _ = cpu_rate(models[0], 1, L, 1)
    iters = max(1, int(target_s / max(dt1, 1e-3)))
    grads = [0] * cores

    def work(i):
        o.set_threads(1)  # the OpenMP thread count is per host thread
        m = models[i]
        rng = np.random.default_rng(100 + i)
        m.set_mu((rng.standard_normal(m.shape) * 0.1).astype(np.complex64))
        m.set_sigma(2.0, 5.0)
        grads[i] = m.run_iterations(iters, L, 0.02, 1000 + i)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(cores)]
    t0 = time.perf_counter()
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    dt = time.perf_counter() - t0
    return {"value": sum(grads) / dt, "unit": UNIT, "cores": cores, "chains": cores,
            "sample": f"{cores} independent chains x {iters} HMC iterations (L={L}), one host thread each, "
                      f"{dt:.1f} s wall"}


def posterior_mean_vs_fp64(vol, iters=12, L=25, eps=0.05, seed=1):
    """The FP32 sampler kernels against the FP64 oracle on identical draws (one chain on `vol`, sigma fixed at
    4 / 11): per iteration the same 2N standard normals become the momentum (MultiResParameters.h:784-815) and the
    same uniform decides the accept (MultiResParameters.h:680-705); the device runs the trajectory through its own
    leapfrog kernels (dr_leapfrog_fixed), the oracle through its FP64 transition (four FFTs per step,
    MultiResParameters.h:674-727).  Returns the norm-wise relative error of the running mean and variance of Re mu
    over the output voxels after `iters` iterations, and how many accept decisions differed."""
    import dualres_b200 as d
    from oracle import oracle as o
    o.set_threads(os.cpu_count() or 1)
    data = d.MultiResData.from_volume(vol)
    ch = d.MultiResParameters(data, d.HMCParameters(burnin=2, nsave=2, thin=1, leapfrog=L, seed=seed), 1)
    prep = o.prepare(vol.highres)
    rp, col, val = data.W()
    _, ys = data.data()
    md = o.Model(prep["D"], prep["Yh"], vol.qform_hr, vol.theta, ys, (rp, col, val.astype(np.float64)), prep["O"],
                 precision="d")
    sh, ss = 4.0, 11.0
    md.set_sigma(sh, ss)
    E = md.E
    flat = lambda ijk: (ijk[:, 2] * E[0] * E[1] + ijk[:, 1] * E[0] + ijk[:, 0])  # noqa: E731
    mu = np.zeros(md.shape, np.complex64)
    mu.ravel()[flat(np.asarray(prep["D"]).reshape(-1, 3))] = prep["Yh"]
    md.set_mu(mu)
    ch.set_state(0, mu, (sh, ss))
    oi = flat(np.asarray(prep["O"]).reshape(-1, 3))
    rng = np.random.default_rng(seed)
    s64, q64, s32, q32 = (np.zeros(len(oi)) for _ in range(4))
    flips = acc = 0
    t0 = time.perf_counter()
    for _ in range(iters):
        z = rng.standard_normal(2 * md.N).astype(np.float32)
        u = float(rng.random())
        p, e0z = md.momentum(z)
        _, out, _ = md.transition(z, u, eps, L)
        muL, _, en = ch.leapfrog(0, mu, p.astype(np.complex64), eps, L)
        log_r = (en[3] + en[4] + en[5]) - (e0z + en[0] + en[1])
        a32 = bool(np.log(u) < log_r)
        mu = muL if a32 else mu
        flips += int(a32 != bool(out[1]))
        acc += int(out[1])
        x64, x32 = md.get_mu().ravel()[oi].real.astype(np.float64), mu.ravel()[oi].real.astype(np.float64)
        s64 += x64
        q64 += x64 * x64
        s32 += x32
        q32 += x32 * x32
    dt = time.perf_counter() - t0
    ch.close()
    data.close()
    m64, m32 = s64 / iters, s32 / iters
    v64, v32 = q64 / iters - m64 * m64, q32 / iters - m32 * m32
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    return {"rel_mean": rel(m32, m64), "rel_var": rel(v32, v64), "iterations": iters, "leapfrog": L, "eps": eps,
            "accept_flips": flips, "accept_rate": acc / iters, "seconds": dt,
            "what": "FP32 sampler kernels (dr_leapfrog_fixed) vs the FP64 oracle on identical draws, one chain on "
                    "this volume, sigma fixed; norm-wise relative error of the running posterior mean and variance "
                    "of Re mu over the output voxels"}


def cpu_baseline_line(vol, W, L, target_s=12.0, pm_iters=12, pm_L=25):
    threads = os.cpu_count() or 1
    m, _ = oracle_model(vol, W)
    r1, dt1, _ = cpu_rate(m, 1, L, threads)
    iters = max(1, int(target_s / max(dt1, 1e-3)))
    r, dt, g = cpu_rate(m, iters, L, threads)
    line = {"value": r, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{iters} HMC iterations (L={L}, {g} gradient evals) of one chain on the same volume, "
                      f"FP32 restatement of MultiResParameters<float>::update (4 FFTs per leapfrog step), "
                      f"{dt:.1f} s"}
    try:  # the same restatement as independent single-threaded chains, one per host thread
        line["throughput"] = cpu_throughput(vol, W, L, threads, target_s=target_s * 10.0 / 12.0)
    except Exception as e:  # an extra must not break the benchmark line
        line["throughput"] = {"error": str(e)[:200]}
    try:  # the oracle as the checker of the device's numerics on this volume
        line["posterior_mean_vs_fp64"] = posterior_mean_vs_fp64(vol, iters=pm_iters, L=pm_L)
    except Exception as e:  # an extra must not break the benchmark line
        line["posterior_mean_vs_fp64"] = {"error": str(e)[:200]}
    return line


def run_reference(args, dist):
    wl = WORKLOADS[args.workload]
    if dist.rank != 0:
        return None
    vol = make_volume(wl["vol"])
    threads = os.cpu_count() or 1
    t0 = time.perf_counter()
    m, _ = oracle_model(vol, None)
    setup = time.perf_counter() - t0
    from oracle import oracle as o
    o.set_threads(threads)
    L = wl["leapfrog"]
    rng = np.random.default_rng(1)
    m.set_mu((rng.standard_normal(m.shape) * 0.1).astype(np.complex64))
    m.set_sigma(2.0, 5.0)
    for _ in range(args.warmup):
        m.run_iterations(1, L, 0.02, 3)
    t0 = time.perf_counter()
    g = 0
    for i in range(args.steps):
        g += m.run_iterations(1, L, 0.02, 100 + i)
    dt = time.perf_counter() - t0
    value = g / dt
    return {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic (seeded GP draw)",
            "impl": "reference",
            "config": config_of(args.workload, {"setup_seconds": setup,
                                                "sample": "one chain, one HMC iteration per step"}),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{args.steps} HMC iterations (L={L}) of one chain on the same volume, "
                                       f"FP32 restatement of MultiResParameters<float>::update, {threads} threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def profile_kernel(args):
    """Set up the workload, run --warmup iterations, then launch kernel K four times inside an NVTX range
    named "profile" (ncu --nvtx --nvtx-include "profile/" captures exactly those launches)."""
    import torch

    import dualres_b200 as d
    # under ncu the serialised replays distort the tuner's timings; profile the default configuration, which is the
    # one the tuner picks for the benchmark workloads when it runs without a profiler (chain_set_config in the line)
    os.environ.setdefault("DRB_AUTOTUNE", "0")
    wl = WORKLOADS[args.workload]
    hmc = d.HMCParameters(burnin=wl["burnin"], nsave=wl["nsave"], thin=wl["thin"], leapfrog=wl["leapfrog"],
                          seed=args.seed)
    data = d.MultiResData.from_volume(make_volume(wl["vol"]))
    chains = d.MultiResParameters(data, hmc, wl["chains"])
    chains.update(max(args.warmup, 3))
    torch.cuda.nvtx.range_push("profile")
    ms, b = d.api.time_kernel(chains, args.profile_kernel, step=1, reps=3)
    torch.cuda.nvtx.range_pop()
    print(json.dumps({"kernel": d.api.KERNEL_NAMES[args.profile_kernel], "ms": ms, "algorithmic_bytes": b,
                      "chains": wl["chains"], "steps": [s["integrator_steps"] for s in chains.stats()][:4]}))


def main():
    args = parse()
    if args.profile_kernel >= 0:
        profile_kernel(args)
        return
    if args.impl == "reference":
        dist = Dist("gloo")
        line = run_reference(args, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
        dist.close()
        return
    dist = Dist("nccl")
    if "rate" in WORKLOADS[args.workload]:
        line, job_vols = run_served(args, dist)
        if dist.rank == 0:
            if dist.world == 1 and not args.no_cpu:
                try:
                    line["cpu_baseline"] = served_cpu_baseline(job_vols, WORKLOADS[args.workload], args.cpu_seconds)
                except Exception as e:  # an extra must not break the benchmark line
                    line["cpu_baseline"] = {"error": str(e)[:200]}
            print(json.dumps(line), flush=True)
        dist.close()
        return
    line = run_ours(args, dist)
    if dist.rank == 0:
        if dist.world == 1 and not args.no_cpu:
            vol = make_volume(WORKLOADS[args.workload]["vol"])
            import dualres_b200 as d
            dv = d.MultiResData.from_volume(vol)
            rp, col, val = dv.W()
            dv.close()
            line["cpu_baseline"] = cpu_baseline_line(vol, (rp, col, val.astype(np.float32)),
                                                     WORKLOADS[args.workload]["leapfrog"], target_s=args.cpu_seconds)
        print(json.dumps(line), flush=True)
    dist.close()


if __name__ == "__main__":
    main()
