"""Benchmark: seconds to 8 band-edge eigenpairs of a ~2.0M-atom InAs dot.

Workload (the headline): InAs lens (base
20 nm, height 5 nm) on a one-monolayer InAs wetting layer in a GaAs box of
72 x 72 x 48 cells (1,990,656 atoms), sp3d5s* with spin-orbit (20 orbitals
per atom, H of dimension 39,813,120), dangling bonds passivated (+30 eV),
atom positions displaced by a seeded Gaussian (sigma = 0.5% of the bond
length) as a strain stand-in.  One step = one full mixed-precision solve
through libtbgpu: topology + Slater-Koster assembly from the structure into
the single-precision store, Lanczos on complex-float vectors with double
alpha/beta, tridiagonal and convergence test (the reference's windowed test)
for the 4 highest hole and 4 lowest electron states, the eigenvector pass by
regeneration of 256-iteration segments from first-pass checkpoints four at a
time, and the double-precision Rayleigh-Ritz refinement.  Start vector
uniform in [-1, 1], seed 0.

``value`` times steps whose inputs are already in HBM; ``e2e`` times the same
solve through the host-pointer C ABI (geometry and start vector copied in,
eigenvectors copied out).  The same run times the plain FP64 GPU Lanczos
(the reference's method: double store and vectors, second run of the
recurrence for the eigenvectors) on the same dot once, and reports the ratio,
the per-state eigenvalue difference and the FP64 residual ||Hv - lambda v||
of each mixed eigenpair through the recomputed double-precision product (a
product independent of the stored blocks).  ``--workload dome1M`` is the
1,022,656-atom dome (58 x 58 x 38 cells), plain FP64, 8 electron + 8 hole
states.
``--impl reference`` times the reference's own first Lanczos pass
(eigenvaluesLanczos of eigen/src/lanczos.c, compiled from its source into
oracle/_ref by oracle/build_ref.sh, running on the oracle's plain-C
restatement of the FP64 stored H*x with OpenMP over the host cores; the
oracle alone where that library is absent) on a bounded sample of iterations
per step and scales it to a full plain FP64 solve (both passes).

The mixed solve's convergence test bounds the tridiagonal eigenvector's last
components by max(tolerance, 2^-24 x the Gershgorin bound of T) -- the
rounding level of the complex-float recurrence (``--mixed-accept``; 0 gives
the tolerance alone, as the FP64 solve uses): values are then refined in
FP64, and the line carries each state's difference from the FP64 solve and
both solves' FP64 residuals.
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

from nemo3d_b200 import materials, workloads  # noqa: E402

METRIC = "s to 8 band-edge eigenpairs at <=1e-6 eV vs plain FP64 GPU Lanczos; SpMV HBM GB/s"
# Algorithmic bytes per atom of one H*x with the reference's compact store
# (blocks once per bond, on-site diagonal + spin-orbit, int32 column per bond,
# x read once, y written once): FP64 1864 + 640, complex-float 936 + 320.
BYTES_PER_ATOM = {64: 2504, 32: 1256}
# DRAM bytes per atom of one H*x launch, measured with ncu (dram__bytes_read
# + dram__bytes_write, one launch, cold L2) on the 384,000-atom profile case
# and scaled by atoms: the float lane kernel 488.6 MB, the FP64 default
# kernel 3054 B/atom at full size.
NCU_TRAFFIC_PER_ATOM = {32: 1272, 64: 3054}
# one complex vector per atom (20 entries: FP64 320 B, complex float 160 B) and
# the stored blocks + on-site records + neighbour columns per atom (B_H)
VEC_PER_ATOM = {64: 320, 32: 160}
H_PER_ATOM = {64: 1864, 32: 936}

# band-edge windows of the dome: 4 highest hole and 4 lowest electron states
# (Erange_vb / Erange_cb of the reference's Lanczos deck)
SOLVE = dict(ConvCheckStartIter=200, ConvCheckSkipRate=50, imax=20000,
             requested1=4, requested2=4, emin1=1.032, emax1=1.06,
             emin2=1.44, emax2=1.475, tolerance=1e-7)
NVEC = 8
# the 1.02M-atom dome: 8 hole and 8 electron states
SOLVE_8X8 = dict(SOLVE, requested1=8, requested2=8, emin1=0.95, emax1=1.06, emin2=1.44,
                 emax2=1.56, imax=30000)
# the mixed-precision solver: float store and vectors, H*x variant 5 (lane
# per atom and spin), eigenvector pass 1 (regeneration, 4 columns,
# 256-iteration segments)
MIXED_VARIANT = 5
MIXED_VEC_PASS = (1, 4, 256)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_structure(cells=(72, 72, 48)):
    """The InAs dome in a GaAs box of the given cells (default: the 1,990,656-atom
    dot of the headline; (58, 58, 38): the 1,022,656-atom dot)."""
    return workloads.dome_in_box(cells=cells, base_nm=20.0, height_nm=5.0,
                                 sigma_frac=0.005, seed=1)


MATS = [materials.MATERIALS["GaAs_spds"], materials.MATERIALS["InAs_spds"]]


# ------------------------------------------------------------------------------
class _QuietStdout:
    """Sends the C library's stdout (the reference's progress prints) to
    /dev/null while a reference routine runs, keeping bench.py's stdout to
    its JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.null)
        os.close(self.saved)


class CpuReference:
    """The reference's CPU path for this workload: its own Lanczos driver
    (eigenvaluesLanczos of eigen/src/lanczos.c, compiled from the reference's
    source into oracle/_ref/libref_lanczos.so) on the oracle's FP64 stored
    Hamiltonian and H*x (a plain-C restatement of Hmult_stored; the
    reference's own product needs its XML-driven set-up).  Without the
    reference build, the oracle's restatement of the same driver."""

    def __init__(self, st):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        self.oracle = oracle
        self.cores = os.cpu_count() or 1
        oracle.lib().orc_set_threads(self.cores)
        t0 = time.perf_counter()
        self.H = oracle.OracleHamiltonian(st, 10, 2, MATS)
        self.t_build = time.perf_counter() - t0
        self.r0 = workloads.random_start(self.H.n, seed=0)
        self.kind = "reference" if oracle.ref_lanczos_available() else "port"

    def per_iteration(self, n_it, threads):
        """Seconds per iteration of n_it iterations of the first pass (no
        convergence checks) on `threads` host threads."""
        self.oracle.lib().orc_set_threads(threads)
        kw = dict(imax=n_it + 1, req=(1, 1), conv_start=10 ** 9)
        t = time.perf_counter()
        if self.kind == "reference":
            with _QuietStdout():
                self.oracle.ref_eigenvalues_lanczos(self.H, self.r0, **kw)
        else:
            self.H.lanczos(self.r0, **kw)
        return (time.perf_counter() - t) / n_it


def cpu_sample(st, its_total, budget_s=60.0, ref=None):
    """The reference's CPU path (CpuReference) on a bounded sample of the
    workload: the H build, then timed iterations on 1 thread (the
    reference's Lanczos is serial) and on all host threads; the 1-thread
    time per iteration scaled to a solve of ``its_total`` iterations (both
    passes of the plain FP64 method) is the value."""
    ref = ref or CpuReference(st)
    per1 = ref.per_iteration(1, 1)                      # calibration
    n1 = int(max(2, min(100, 0.3 * budget_s / max(per1, 1e-6))))
    per1 = ref.per_iteration(n1, 1)
    perN = ref.per_iteration(1, ref.cores)
    nN = int(max(2, min(200, 0.5 * budget_s / max(perN, 1e-6))))
    perN = ref.per_iteration(nN, ref.cores)
    est = ref.t_build + per1 * its_total
    what = ("the reference's eigenvaluesLanczos (eigen/src/lanczos.c, compiled from its source) "
            "on the oracle's restatement of the FP64 stored H*x" if ref.kind == "reference"
            else "the oracle's restatement of the reference's FP64 H*x and Lanczos driver")
    return dict(value=est, unit="s", cores=1, kind=ref.kind,
                sample=(f"{what}: H build {ref.t_build:.1f} s (timed, {ref.cores} threads); "
                        f"{n1} iterations timed on 1 thread ({per1 * 1e3:.0f} ms each) and {nN} on "
                        f"{ref.cores} threads ({perN * 1e3:.0f} ms each; {ref.t_build + perN * its_total:.0f} s "
                        f"for the solve), no convergence checks, on {ref.H.natoms} atoms; "
                        f"extrapolated to {its_total} iterations (first pass + eigenvector pass "
                        f"of the plain FP64 method)"),
                all_cores_value=ref.t_build + perN * its_total, all_cores=ref.cores)


# ------------------------------------------------------------------------------
def run_reference(args, rank, world):
    if rank != 0:
        return
    cells = (58, 58, 38) if args.workload == "dome1M" else (72, 72, 48)
    st = make_structure(cells)
    its = args.ref_iterations
    ref = CpuReference(st)
    # each step: a bounded sample (4 iterations on all host threads) of the
    # reference's Lanczos on this dot, scaled to the full solve
    vals, pers = [], []
    for i in range(args.warmup + args.steps):
        per = ref.per_iteration(4, ref.cores)
        if i >= args.warmup:
            pers.append(per)
            vals.append(ref.t_build + per * its)
    v = float(np.mean(vals))
    cb = dict(value=v, unit="s", cores=ref.cores, kind=ref.kind,
              sample=(f"per step: 4 iterations of the first pass (no convergence checks) of "
                      + ("the reference's eigenvaluesLanczos (eigen/src/lanczos.c, compiled from "
                         "its source) on the oracle's restatement of the FP64 stored H*x"
                         if ref.kind == "reference" else "the oracle's restatement")
                      + f" on {ref.H.natoms} atoms with {ref.cores} threads "
                      f"({np.mean(pers) * 1e3:.0f} ms each), plus the H build ({ref.t_build:.1f} s, "
                      f"timed once), scaled to {its} iterations (both passes of the plain FP64 method)"))
    line = {"metric": METRIC,
            "impl": "reference", "value": v, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"InAs dome {cells[0]}x{cells[1]}x{cells[2]} cells, "
                                   f"{st.nsites} atoms, sp3d5s*+SO, plain FP64 Lanczos "
                                   "(the reference's method)",
                       "states": "4 e + 4 h", "iterations": its},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------
def max_over_ranks(value, dist, device):
    """The largest of one float across the ranks (the job's time is that of
    its slowest replica); `dist` is torch.distributed or None for one rank."""
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def per_iteration(bits, natoms, stats, res):
    its = max(int(res["iterations"]), 1)
    ms = stats["solve_ms"] / its
    alg = (BYTES_PER_ATOM[bits] + VEC_PER_ATOM[bits]) * natoms
    moved = (H_PER_ATOM[bits] + 6 * VEC_PER_ATOM[bits]) * natoms
    pk = peaks()[0]["hbm_gbs"]
    return {"ms": ms, "algorithmic_gb": alg / 1e9, "moved_gb": moved / 1e9,
            "algorithmic_frac": alg / (ms * 1e-3) / 1e9 / pk,
            "moved_frac": moved / (ms * 1e-3) / 1e9 / pk}


def _match_states(a, b):
    """Per-state |a_i - b_j| pairing each value of a with the nearest of b."""
    b = np.asarray(b)
    return [float(np.abs(b - v).min()) if b.size else None for v in np.asarray(a)]


def run_ours(args, rank, world, local_rank):
    import torch
    from nemo3d_b200 import tbgpu
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    dome1m = args.workload == "dome1M"
    cells = (58, 58, 38) if dome1m else (72, 72, 48)
    solve_kw = SOLVE_8X8 if dome1m else SOLVE
    nvec = 16 if dome1m else NVEC
    mixed = not dome1m
    bits = 32 if mixed else 64
    st = make_structure(cells)
    types_d = torch.from_numpy(np.ascontiguousarray(st.types).reshape(-1)).cuda()
    dsp_d = torch.from_numpy(np.ascontiguousarray(st.dsp).reshape(-1)).cuda()
    stream = torch.cuda.Stream()
    probe = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, build=True)
    natoms, n = probe.natoms, probe.n
    probe.close()
    r0_h = workloads.random_start(n, seed=0)
    r0_d = torch.from_numpy(r0_h).cuda()
    V_d = torch.empty(nvec * 2 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    def solve(precision, V, profile=False):
        """One full solve from device-resident inputs: build + solve (+ refine)."""
        opts = dict(ham_bits=32, lanczos_bits=32) if precision == 32 else {}
        H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, build=False,
                              device_inputs=(types_d.data_ptr(), dsp_d.data_ptr()), **opts)
        H.set_stream(stream.cuda_stream)
        if precision == 32:
            H.set_spmv_variant(args.mixed_variant)
            H.set_eigenvector_pass(1, args.mixed_columns, MIXED_VEC_PASS[2])
            H.set_mixed_acceptance(args.mixed_accept)
        else:
            H.set_spmv_variant(args.spmv_variant)
        H.build()
        if profile:
            H.set_profiling(True)
        res = H.eigensolve_lanczos_dev(r0_d.data_ptr(), V.data_ptr(), nvec, **solve_kw)
        s = H.stats()
        if precision == 32:
            res["state_resid"], res["state_delta"] = H.state_errors()
        H.close()
        return res, s

    def barrier():
        if dist is not None:
            dist.barrier()

    stats_acc = []
    for _ in range(args.warmup):
        res, s = solve(bits, V_d)
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    smi_index = vis.split(",")[local_rank] if vis else str(local_rank)
    with ClockSampler(smi_index) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            res, s = solve(bits, V_d, profile=True)
            stats_acc.append(s)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, "cuda")

    # the plain FP64 GPU Lanczos on the same dot (the reference's method)
    fp64 = None
    if mixed and not args.no_fp64_baseline:
        Vf = torch.empty_like(V_d)
        # untimed solves first, as for the mixed steps: the solver's memory
        # pool then holds this method's buffers too
        for _ in range(args.fp64_warmup):
            solve(64, Vf)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        rf, sf = solve(64, Vf)
        f1.record(stream)
        torch.cuda.synchronize()
        fp64 = dict(res=rf, stats=sf, s=max_over_ranks(f0.elapsed_time(f1) / 1e3, dist, "cuda"),
                    V=Vf)

    # FP64 residual ||H v - lambda v|| of each returned eigenpair through the
    # recomputed double-precision product (independent of the stored blocks),
    # for this solve and for the plain FP64 one
    resid, resid64 = [], []
    if not args.no_residuals:
        Hr = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, build=False, recompute=True,
                               device_inputs=(types_d.data_ptr(), dsp_d.data_ptr()))
        Hr.build()
        y = torch.empty(2 * n, dtype=torch.float64, device="cuda")

        def residuals(values, V):
            out = []
            for e, lam in enumerate(values[:nvec]):
                v = V[e * 2 * n:(e + 1) * 2 * n]
                Hr.hx_dev(v.data_ptr(), y.data_ptr(), float(lam))
                torch.cuda.synchronize()
                out.append(float(torch.linalg.vector_norm(y).item() /
                                 torch.linalg.vector_norm(v).item()))
            return out

        resid = residuals(res["values"], V_d)
        if fp64 is not None:
            resid64 = residuals(fp64["res"]["values"], fp64["V"])
        Hr.close()
        del y
    if fp64 is not None:
        del fp64["V"]
        torch.cuda.empty_cache()

    # end to end through the host-pointer C ABI
    e2e_s = None
    h2d = d2h = 0
    if args.e2e_steps > 0:
        times = []
        for _ in range(args.e2e_steps):
            torch.cuda.synchronize()
            barrier()
            t0 = time.perf_counter()
            opts = dict(ham_bits=32, lanczos_bits=32) if mixed else {}
            H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, **opts)   # host geometry in
            if mixed:
                H.set_spmv_variant(args.mixed_variant)
                H.set_eigenvector_pass(1, args.mixed_columns, MIXED_VEC_PASS[2])
                H.set_mixed_acceptance(args.mixed_accept)
            else:
                H.set_spmv_variant(args.spmv_variant)
            out = H.eigensolve_lanczos(r0_h, vectors=nvec, **solve_kw)  # host r0 in, vectors out
            H.close()
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(float(np.mean(times)), dist, "cuda")
        h2d = st.types.nbytes + st.dsp.nbytes + r0_h.nbytes + 8 * 8 * 68
        d2h = len(out["vectors"]) * 16 * n + 8 * len(out["values"])

    if rank == 0:
        pk, pk_kind = peaks()
        last = stats_acc[-1]
        spmv_ms = last["spmv_ms"] / max(last["spmv_launches"], 1)
        achieved = BYTES_PER_ATOM[bits] * natoms / (spmv_ms * 1e-3) / 1e9
        its_total = int(res["iterations"] + (max(res["conv_iterations"])
                                              if len(res["conv_iterations"]) else 0))
        name = (f"InAs dome {cells[0]}x{cells[1]}x{cells[2]} cells, {natoms:,} atoms, sp3d5s*+SO, "
                + ("mixed-precision Lanczos (complex-float store and vectors, FP64 alpha/beta, "
                   "tridiagonal and Rayleigh-Ritz refinement), eigenvectors regenerated from "
                   "checkpoints" if mixed else "plain FP64 Lanczos, 8 e + 8 h"))
        cfg = {"workload": name, "natoms": natoms, "dimension": n,
               "states": "4 e + 4 h (8 eigenpairs)" if mixed else "8 e + 8 h (16 eigenpairs)",
               "parallelism": f"replicas x{world} (one dot per GPU)",
               "l2": "inputs larger than L2 (H 1.9-6.4 GB, vectors 318-636 MB each)",
               "eigenvalues": [round(float(v), 12) for v in res["values"]],
               "iterations_first_pass": int(res["iterations"]),
               "build_ms": last["build_ms"], "solve_ms": last["solve_ms"],
               "vectors_ms": last["vectors_ms"], "refine_ms": last["refine_ms"],
               "vec_segments": last["vec_segments"], "vec_mismatch": last["vec_mismatch"],
               "hx_avg_ms": spmv_ms,
               # one first-pass iteration: the algorithmic bytes (B_SpMV + one
               # vector read, the recurrence's minimum) and the bytes this
               # design moves (B_H + 6 vector passes: the product's x and y,
               # the update's three reads and one write), over the measured
               # time per iteration (first pass / iterations)
               "per_iteration": per_iteration(bits, natoms, last, res),
               "update_avg_ms": last["update_ms"] / max(last["spmv_launches"], 1),
               "host_check_ms": last["check_ms"], "host_wait_ms": last["wait_ms"],
               "residual_per_state_ev": resid, "tolerance": solve_kw["tolerance"]}
        if mixed:
            cfg["refine_residual_per_state_ev"] = [float(v) for v in res["state_resid"]]
            cfg["mixed_acceptance_floor"] = (
                args.mixed_accept if args.mixed_accept >= 0 else
                "2^-24 x Gershgorin bound of T (complex-float rounding level)")
        if fp64 is not None:
            cfg["fp64_plain"] = {
                "s": fp64["s"], "iterations_first_pass": int(fp64["res"]["iterations"]),
                "first_pass_ms": fp64["stats"]["solve_ms"],
                "vectors_ms": fp64["stats"]["vectors_ms"],
                "eigenvalues": [round(float(v), 12) for v in fp64["res"]["values"]],
                "residual_per_state_ev": resid64, "warmup": args.fp64_warmup}
            cfg["speedup_vs_fp64_plain"] = fp64["s"] / (ms / 1e3)
            cfg["error_per_state_ev_vs_fp64"] = _match_states(res["values"], fp64["res"]["values"])
        line = {
            "metric": METRIC,
            "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "c32+f64" if mixed else "f64",
            "data": "synthetic (seeded InAs dome in GaAs, Gaussian displacements)",
            "config": cfg,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps},
            "gpu_launches": int(sum(x["kernel_launches"] for x in stats_acc) // len(stats_acc) + 4),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"],
                         "unit": "GB/s", "frac": achieved / pk["hbm_gbs"],
                         "peak_source": pk_kind,
                         "traffic": NCU_TRAFFIC_PER_ATOM[bits] * natoms,
                         "kernel": "H*x with fused alpha (first pass), "
                                   + ("complex-float lane kernel" if mixed else "FP64"),
                         "algorithmic_bytes": BYTES_PER_ATOM[bits] * natoms,
                         "avg_launch_ms": spmv_ms},
            "clocks": clk.summary(),
        }
        if not args.no_cpu_baseline:
            fp_its = (int(fp64["res"]["iterations"]) * 2 if fp64 is not None else its_total)
            line["cpu_baseline"] = cpu_sample(st, fp_its, budget_s=args.cpu_budget)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_profile_case(args):
    """A smaller dot (40 x 40 x 30 cells, 384,000 atoms; H and vectors ~2 GB,
    larger than L2) running a few Lanczos iterations without convergence
    checks: the k_spmv / k_update launches that ncu captures (stored or
    recomputed blocks, FP64 or mixed precision), or a few Keating VFF
    iterations of the same structure."""
    import torch
    from nemo3d_b200 import tbgpu
    torch.cuda.set_device(0)
    if args.profile_full:  # the 1.02M-atom dot (for 1-pass captures)
        st = make_structure((58, 58, 38))
    else:
        st = workloads.dome_in_box(cells=(40, 40, 30), base_nm=14.0, height_nm=4.0,
                                   sigma_frac=0.005, seed=1)
    if args.profile_vff:  # a few Keating iterations (k_vff_vertex / k_vff_gather)
        st.dsp = None
        H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, build=False)
        _, e, its = H.vff_relax(max_iter=args.profile_iterations, tol=0.0)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "vff", "natoms": st.nsites, "iterations": its,
                          "energy": e}), flush=True)
        return
    if args.profile_mixed:  # the headline's solver configuration on this dot
        H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, ham_bits=32, lanczos_bits=32)
        H.set_spmv_variant(args.mixed_variant)
        H.set_eigenvector_pass(1, args.mixed_columns, MIXED_VEC_PASS[2])
        H.set_mixed_acceptance(args.mixed_accept)
        r0 = workloads.random_start(H.n, seed=0)
        res = H.eigensolve_lanczos(r0, vectors=2, requested1=1, requested2=1, emin1=0.4,
                                   emax1=1.25, emin2=1.25, emax2=2.2, tolerance=1e-7,
                                   imax=20000)
        torch.cuda.synchronize()
        print(json.dumps({"profile_case": "mixed", "natoms": H.natoms, "dimension": H.n,
                          "values": [float(v) for v in res["values"]],
                          "iterations": res["iterations"], "stats": H.stats()}), flush=True)
        return
    opts = {}
    if args.profile_storage == "recompute":
        opts["recompute"] = True
    elif args.profile_precision == 32:
        opts["ham_bits"] = 32
    if args.profile_precision == 32:
        opts["lanczos_bits"] = 32
    H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, **opts)
    H.set_spmv_variant(args.spmv_variant)
    r0 = workloads.random_start(H.n, seed=0)
    if args.profile_vectors:  # a converging solve with the eigenvector pass (k_accum)
        res = H.eigensolve_lanczos(r0, vectors=8, requested1=4, requested2=4, emin1=0.4,
                                   emax1=1.25, emin2=1.25, emax2=2.2, tolerance=1e-7,
                                   imax=20000)
    else:
        res = H.eigensolve_lanczos(r0, imax=args.profile_iterations + 1, requested1=1,
                                   requested2=1, ConvCheckStartIter=10 ** 9)
    torch.cuda.synchronize()
    print(json.dumps({"profile_case": True, "natoms": H.natoms, "dimension": H.n,
                      "iterations": res["iterations"], "stats": H.stats()}), flush=True)


def _event_time(fn, reps, stream_ctx):
    """Average device time (ms) of fn() over reps calls, CUDA events on the
    context's stream (bound to torch's current stream)."""
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def run_extra(args):
    """Measurements beside the headline (one JSON line each), on one GPU:
    kernels   H*x of the 1.02M-atom dome: FP64 store (warp-staged and two-cell unit
              kernels), float store with float
              vectors, recompute in FP64 and in float
    mixed2M   the same dome at 72 x 72 x 48 cells (1,990,656 atoms): plain FP64
              solve against the mixed-precision solve on the float store and on
              the recompute product, eigenvalue error per state
    batch256  256 In(x)Ga(1-x)As dots, 1k-50k atoms log-uniform, x uniform in
              [0.4, 1.0], sp3s*+SO, 4 conduction states each with vectors:
              batched FP64 and mixed solves, and 16 of the dots solved one at
              a time (scaled by atoms)
    vff1M     Keating relaxation of the 1.02M-atom dome (no Gaussian
              displacements), AllFree
    warm      learned warm start: plain solves of --warm-train randomized
              In(x)Ga(1-x)As lens dots (20 x 20 x 14 cells, 44,800 sites,
              sp3d5s*+SO, 4 h + 4 e levels with vectors) as training data,
              the network trained on them, then --warm-test held-out seeds
              solved cold and warm: iterations and wall time of each
    bdots     block dots G = X^H Y of two blocks of 8 vectors, on the tensor
              cores (tbgpu_block_dots_dev; error against torch's complex
              matrix product), and 40 block Lanczos steps (p = 8) of a GaAs cube of
              --bdots-cube^3 cells with the CUDA-core and the tensor-core dots"""
    import torch
    from nemo3d_b200 import tbgpu
    torch.cuda.set_device(0)
    w = args.workload
    if w == "bdots":
        st = workloads.gaas_cube(args.bdots_cube)
        g = tbgpu.Hamiltonian(st, "sp3d5s*_so", [materials.MATERIALS["GaAs_spds"]])
        n2, p = g.n, 8
        gen = torch.Generator(device="cuda").manual_seed(7)
        X = torch.randn(p, 2 * n2, dtype=torch.float64, device="cuda", generator=gen)
        Y = torch.randn(p, 2 * n2, dtype=torch.float64, device="cuda", generator=gen)
        for _ in range(3):
            G = g.block_dots_dev(p, X.data_ptr(), Y.data_ptr(), n2)
        torch.cuda.synchronize()
        reps = 20
        t0 = time.perf_counter()
        for _ in range(reps):
            G = g.block_dots_dev(p, X.data_ptr(), Y.data_ptr(), n2)
        dt = (time.perf_counter() - t0) / reps
        Xc = torch.view_as_complex(X.view(p, n2, 2))
        Yc = torch.view_as_complex(Y.view(p, n2, 2))
        ref = (Xc.conj() @ Yc.T).cpu().numpy()
        norms = torch.linalg.vector_norm(X, dim=1).cpu().numpy()
        err = float(np.abs(G - ref).max() / norms.max() ** 2)
        r0 = np.random.default_rng(1).uniform(-1, 1, size=(p, 2 * n2))
        kw = dict(imax=40, requested1=3, requested2=3, emin1=-1.5, emax1=0.5, emin2=1.0,
                  emax2=3.5, tolerance=1e-7, ConvCheckStartIter=1000, ConvCheckSkipRate=50)
        steps = {}
        for mode in (0, 1):
            g.set_block_dots(mode)
            g.eigensolve_blk_lanczos(r0, **dict(kw, imax=5))
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = g.eigensolve_blk_lanczos(r0, **kw)
            torch.cuda.synchronize()
            steps[mode] = dict(steps=int(res["iterations"]), s=time.perf_counter() - t0)
        g.close()
        print(json.dumps({"workload": "bdots", "natoms": st.nsites, "n2": n2, "p": p,
                          "block_dots_dev_wall_ms": dt * 1e3,
                          "max_error_rel_to_norm2": err,
                          "block_lanczos_cuda_core": steps[0],
                          "block_lanczos_tensor_core": steps[1]}), flush=True)
    elif w == "kernels":
        st1 = make_structure((58, 58, 38))
        st2 = make_structure((72, 72, 48))
        f32o = dict(ham_bits=32, lanczos_bits=32)
        for name, opts, f32, var, st in (
                ("fp64 store", {}, False, 0, st1),
                ("fp64 store, two-cell units (variant 3)", {}, False, 3, st1),
                ("fp64 store, every piece by cp.async (variant 4)", {}, False, 4, st1),
                ("fp64 store, lane per atom and spin (variant 5)", {}, False, 5, st1),
                ("fp64 store, pencil layout (variant 6)", {}, False, 6, st1),
                ("float store, float vectors", dict(ham_bits=32, lanczos_bits=32), True, 0, st1),
                ("float store, float vectors, lane per atom and spin (variant 5)",
                 dict(ham_bits=32, lanczos_bits=32), True, 5, st1),
                ("float store, float vectors, pencil layout (variant 6)",
                 dict(ham_bits=32, lanczos_bits=32), True, 6, st1),
                ("recompute fp64", dict(recompute=True), False, 0, st1),
                ("recompute float", dict(recompute=True, lanczos_bits=32), True, 0, st1),
                ("2M dot, float store, float vectors, lane per atom and spin (variant 5)",
                 f32o, True, 5, st2),
                ("2M dot, float store, float vectors, pencil layout (variant 6)", f32o, True, 6,
                 st2),
                ("2M dot, float store, float vectors, pencil layout, staged rows (variant 7)",
                 f32o, True, 7, st2)):
            H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, **opts)
            H.set_spmv_variant(var)
            stream = torch.cuda.Stream()
            H.set_stream(stream.cuda_stream)
            dt = torch.float32 if f32 else torch.float64
            x = torch.from_numpy(workloads.random_start(H.n, seed=0)).to(dt).cuda()
            y = torch.empty_like(x)
            torch.cuda.synchronize()
            with torch.cuda.stream(stream):
                f = (lambda: H.hx_dev_f32(x.data_ptr(), y.data_ptr())) if f32 else \
                    (lambda: H.hx_dev(x.data_ptr(), y.data_ptr()))
                ms = _event_time(f, 20, stream)
            # inside the Lanczos recurrence: the product with the fused alpha on
            # the solver's own vectors (the pencil layout for variant 6), CUDA
            # events around every launch of a 60-iteration run without checks
            r0 = torch.from_numpy(workloads.random_start(H.n, seed=0)).cuda()
            H.set_profiling(True)
            H.eigensolve_lanczos_dev(r0.data_ptr(), 0, 0, imax=61, requested1=1, requested2=1,
                                     ConvCheckStartIter=10 ** 9)
            stt = H.stats()
            ms_solve = stt["spmv_ms"] / max(stt["spmv_launches"], 1)
            bpa = 1256 if f32 else 2504
            print(json.dumps({"workload": "kernels", "metric": "H*x ms per launch", "variant": name,
                              "natoms": H.natoms, "value": ms, "unit": "ms",
                              "in_solve_ms": ms_solve,
                              "in_solve_frac_of_peak": bpa * H.natoms / (ms_solve * 1e-3) / 1e9
                              / peaks()[0]["hbm_gbs"]}), flush=True)
            H.close()
    elif w == "mixed2M":
        st = workloads.dome_in_box(cells=(72, 72, 48), base_nm=20.0, height_nm=5.0,
                                   sigma_frac=0.005, seed=1)
        ref = None
        f32 = dict(ham_bits=32, lanczos_bits=32)
        # (name, options, H*x variant, eigenvector pass (mode, columns,
        # segment) or None, tolerance)
        variants = [("fp64 (warp-staged kernel, second run for the vectors)", {}, 0, None, 1e-7),
                    ("fp64, pencil kernel", {}, 6, None, 1e-7),
                    ("fp64, pencil kernel, regenerated vectors P=2 L=256", {}, 6, (1, 2, 256),
                     1e-7),
                    ("mixed, float store, warp-staged kernel", f32, 0, None, 1e-7),
                    ("mixed, float store, lane kernel, regenerated vectors P=4 L=256", f32, 5,
                     (1, 4, 256), 1e-7),
                    ("mixed, float store, pencil kernel, regenerated vectors P=4 L=256", f32, 6,
                     (1, 4, 256), 1e-7),
                    ("mixed, float store, pencil kernel, regenerated vectors P=4 L=128", f32, 6,
                     (1, 4, 128), 1e-7)]
        if args.mixed_recompute:
            variants.append(("mixed, recompute", dict(recompute=True, lanczos_bits=32), 0, None,
                             1e-7))
        for name, opts, var, vpass, tol in variants:
            H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, **opts)
            H.set_spmv_variant(var)
            if vpass:
                H.set_eigenvector_pass(*vpass)
            r0 = torch.from_numpy(workloads.random_start(H.n, seed=0)).cuda()
            V = torch.empty((NVEC, 2 * H.n), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            t = time.time()
            res = H.eigensolve_lanczos_dev(r0.data_ptr(), V.data_ptr(), NVEC,
                                           **dict(SOLVE, tolerance=tol))
            torch.cuda.synchronize()
            wall = time.time() - t
            stt = H.stats()
            line = {"workload": "mixed2M", "metric": "s to 8 band-edge eigenpairs", "variant": name,
                    "natoms": H.natoms, "value": wall, "unit": "s",
                    "first_pass_ms": stt["solve_ms"], "vectors_ms": stt["vectors_ms"],
                    "refine_ms": stt["refine_ms"], "iterations": res["iterations"],
                    "vec_segments": stt["vec_segments"], "vec_mismatch": stt["vec_mismatch"],
                    "eigenvalues": [round(float(v), 12) for v in res["values"]]}
            if ref is None:
                ref = res["values"]
            elif len(ref) == len(res["values"]):
                line["error_per_state_ev"] = [float(abs(a - b)) for a, b in zip(ref, res["values"])]
            if "lanczos_bits" in opts:
                r, _ = H.state_errors()
                line["residual_per_state_ev"] = [float(v) for v in r]
            print(json.dumps(line), flush=True)
            H.close()
            del V, r0
            torch.cuda.empty_cache()
    elif w == "batch256":
        nd = 256
        rng = np.random.default_rng(2024)
        sizes = np.exp(rng.uniform(np.log(1000), np.log(50000), nd)).astype(int)
        xs = rng.uniform(0.4, 1.0, nd)
        dots = [workloads.alloy_dot(int(n), float(x), seed=i) for i, (n, x) in enumerate(zip(sizes, xs))]
        packed, cells = workloads.pack_dots(dots)
        mats = [materials.MATERIALS["GaAs_sps"], materials.MATERIALS["InAs_sps"]]
        kw = dict(ConvCheckStartIter=200, ConvCheckSkipRate=50, imax=12000, requested1=0,
                  requested2=4, tolerance=1e-7)
        win = dict(emin1=np.zeros(nd), emax1=np.zeros(nd), emin2=np.full(nd, 1.0),
                   emax2=np.full(nd, 2.6))
        for name, opts in (("fp64 batch", {}), ("mixed batch", dict(ham_bits=32, lanczos_bits=32))):
            H = tbgpu.Hamiltonian(packed, "sp3s*_so", mats, **opts)
            tuned = H.autotune_spmv(reps=5)  # untimed; the 5-orbital model has one kernel
            r0 = torch.from_numpy(workloads.random_start(H.n, seed=0)).cuda()
            torch.cuda.synchronize()
            t = time.time()
            res = H.eigensolve_lanczos_batched(r0, cells, vectors=4, **win, **kw)
            torch.cuda.synchronize()
            wall = time.time() - t
            stt = H.stats()
            print(json.dumps({"workload": "batch256", "metric": "s to 4 conduction states of 256 dots",
                              "variant": name, "natoms": H.natoms, "value": wall, "unit": "s",
                              "spmv_autotuned": {"variant": tuned[0], "ms": tuned[1]},
                              "first_pass_ms": stt["solve_ms"], "vectors_ms": stt["vectors_ms"],
                              "refine_ms": stt["refine_ms"],
                              "iterations_max": int(res["iterations"].max()),
                              "iterations_median": float(np.median(res["iterations"])),
                              "found_min": int(min(len(v) for v in res["values"]))}), flush=True)
            H.close()
        samp = list(range(0, nd, nd // 16))
        t = time.time()
        atoms = 0
        for i in samp:
            H = tbgpu.Hamiltonian(dots[i], "sp3s*_so", mats, ham_bits=32, lanczos_bits=32)
            H.eigensolve_lanczos(workloads.random_start(H.n, seed=i), emin1=0.0, emax1=0.0,
                                 emin2=1.0, emax2=2.6, vectors=4, **kw)
            atoms += H.natoms
            H.close()
        wall = time.time() - t
        print(json.dumps({"workload": "batch256", "metric": "s to 4 conduction states of 256 dots",
                          "variant": "dots one at a time (mixed; 16-dot sample scaled by atoms)",
                          "value": wall * sizes.sum() / atoms, "unit": "s",
                          "sample_s": wall, "sample_atoms": atoms}), flush=True)
    elif w == "vff1M":
        st = workloads.dome_in_box(cells=(58, 58, 38), base_nm=20.0, height_nm=5.0,
                                   sigma_frac=0.0, seed=1)
        H = tbgpu.Hamiltonian(st, "sp3d5s*_so", MATS, build=False)
        e0 = H.vff_energy()
        torch.cuda.synchronize()
        t = time.time()
        _, e, its = H.vff_relax(bc=0, max_iter=20000, tol=1e-9)
        torch.cuda.synchronize()
        wall = time.time() - t
        print(json.dumps({"workload": "vff1M", "metric": "s to relax (Keating, macopt)",
                          "natoms": st.nsites, "value": wall, "unit": "s", "iterations": its,
                          "energy_start": e0, "energy_end": e}), flush=True)
    elif w == "warm":
        from nemo3d_b200 import warmstart as ws
        G, cells = 16, (20, 20, 14)
        t = time.time()
        train = [ws.solve_sample(workloads.random_lens(s, cells), G)
                 for s in range(args.warm_train)]
        train = [x for x in train if x is not None]
        t_data = time.time() - t
        net = ws.WarmStartNet(G=G, seed=0)
        torch.cuda.synchronize()
        t = time.time()
        hist = net.fit(train, epochs=args.warm_epochs, batch=8)
        torch.cuda.synchronize()
        t_fit = time.time() - t
        # one untimed solve first, so that neither arm pays the first-call costs
        H = tbgpu.Hamiltonian(workloads.random_lens(99_999, cells), ws.MODEL, ws._mats())
        ws.warm_solve(H, net)
        H.close()
        rows = []
        for s in range(args.warm_test):
            st = workloads.random_lens(100_000 + s, cells)
            H = tbgpu.Hamiltonian(st, ws.MODEL, ws._mats())
            out = {}
            for name, model in (("cold", None), ("warm", net)):
                torch.cuda.synchronize()
                t0 = time.time()
                res = ws.warm_solve(H, model)
                out[name] = (res, time.time() - t0)
            c, wv = out["cold"][0], out["warm"][0]
            ok = c["edges"] is not None and wv["edges"] is not None
            rows.append(dict(
                iters_cold=c["iterations"], iters_warm=wv["iterations"],
                wall_cold=out["cold"][1], wall_warm=out["warm"][1], warm_used=wv["warm"],
                dE=float(np.abs(c["edges"] - wv["edges"]).max()) if ok else None,
                sigma_err=abs(wv["sigma"] - 0.5 * (c["edges"][3] + c["edges"][4]))
                if c["edges"] is not None else None,
                edges_cold=None if c["edges"] is None else [float(e) for e in c["edges"]],
                edges_warm=None if wv["edges"] is None else [float(e) for e in wv["edges"]]))
            H.close()
        # the bound on any start vector: the cold solve's own band-edge
        # eigenvectors (random phases) plus a random part of relative weight
        # eps, on the first held-out dots
        ideal = []
        for s in range(min(4, args.warm_test)):
            st = workloads.random_lens(100_000 + s, cells)
            H = tbgpu.Hamiltonian(st, ws.MODEL, ws._mats())
            c = ws.warm_solve(H, None, vectors=ws.MAXVEC)
            idx = ws.band_edges(c["values"], ws.SIGMA0)
            if idx is None or idx[-1] >= len(c["vectors"]):
                H.close()
                continue
            rng = np.random.default_rng(s)
            u = workloads.random_start(H.n, seed=0)
            uc = u[0::2] + 1j * u[1::2]
            for eps in (1.0, 0.1):
                v = sum(c["vectors"][i] * np.exp(2j * np.pi * rng.random()) for i in idx)
                v = v / np.linalg.norm(v) + eps * uc / np.linalg.norm(uc)
                r0 = np.empty(2 * H.n)
                r0[0::2], r0[1::2] = v.real, v.imag
                res = H.eigensolve_lanczos(r0, **ws.solve_kw(ws.SIGMA0))
                e = ws.band_edges(res["values"], ws.SIGMA0)
                ideal.append(dict(dot=s, eps=eps, iters_cold=c["iterations"],
                                  iters_ideal=res["iterations"],
                                  same_levels=e is not None and bool(np.abs(
                                      np.asarray(res["values"])[e] - np.asarray(c["values"])[idx]
                                  ).max() < 1e-6)))
            H.close()
        ic = np.array([r["iters_cold"] for r in rows], float)
        iw = np.array([r["iters_warm"] for r in rows], float)
        print(json.dumps({
            "workload": "warm", "metric": "Lanczos iterations to 4 h + 4 e levels, warm / cold",
            "value": float(iw.sum() / ic.sum()), "unit": "ratio",
            "iterations_cold_mean": float(ic.mean()), "iterations_warm_mean": float(iw.mean()),
            "wall_cold_mean_s": float(np.mean([r["wall_cold"] for r in rows])),
            "wall_warm_mean_s": float(np.mean([r["wall_warm"] for r in rows])),
            "iterations_cold_median": float(np.median(ic)),
            "iterations_warm_median": float(np.median(iw)),
            "warm_used": int(sum(r["warm_used"] for r in rows)), "test_dots": len(rows),
            "max_dE_eV": max([r["dE"] for r in rows if r["dE"] is not None], default=None),
            "sigma_err_mean_eV": float(np.mean([r["sigma_err"] for r in rows
                                                if r["sigma_err"] is not None])),
            "train_dots": len(train), "train_iterations_mean": float(np.mean(
                [x["iterations"] for x in train])), "data_s": t_data, "fit_s": t_fit,
            "loss_first": hist[0], "loss_last": hist[-1], "grid": G, "cells": list(cells),
            "ideal_start": ideal,
            "per_dot": rows}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=60.0,
                    help="seconds of timed CPU-baseline iterations (1 thread and all threads)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64-baseline", action="store_true",
                    help="skip the plain FP64 solve of the same dot")
    ap.add_argument("--fp64-warmup", type=int, default=1,
                    help="untimed plain FP64 solves before the timed one")
    ap.add_argument("--no-residuals", action="store_true",
                    help="skip the FP64 residuals of the returned eigenpairs")
    ap.add_argument("--profile-case", action="store_true",
                    help="small-case run of the solver kernels for ncu captures")
    ap.add_argument("--profile-iterations", type=int, default=6)
    ap.add_argument("--profile-full", action="store_true",
                    help="with --profile-case: use the full-size workload")
    ap.add_argument("--profile-storage", default="store", choices=["store", "recompute"],
                    help="with --profile-case: stored blocks or blocks recomputed in H*x")
    ap.add_argument("--profile-precision", type=int, default=64, choices=[64, 32],
                    help="with --profile-case: FP64 or the mixed-precision Lanczos")
    ap.add_argument("--profile-mixed", action="store_true",
                    help="with --profile-case: the headline's mixed solve (kernel, "
                         "regenerating pass, acceptance floor) for 1 hole + 1 electron state")
    ap.add_argument("--profile-vectors", action="store_true",
                    help="with --profile-case: a converging solve with the eigenvector pass")
    ap.add_argument("--profile-vff", action="store_true",
                    help="with --profile-case: a few Keating VFF iterations instead")
    ap.add_argument("--spmv-variant", type=int, default=0, choices=[0, 1, 2, 3, 4, 5, 6],
                    help="H*x kernel of the solve (tbgpu_set_spmv_variant)")
    ap.add_argument("--mixed-variant", type=int, default=MIXED_VARIANT, choices=[5, 6, 7],
                    help="H*x kernel of the mixed solve (its columns must compute as one-column "
                         "launches for the regenerating pass: 5, 6 or 7)")
    ap.add_argument("--mixed-columns", type=int, default=MIXED_VEC_PASS[1], choices=[1, 2, 3, 4],
                    help="eigenvector pass of the mixed solve: segments regenerated per launch")
    ap.add_argument("--mixed-accept", type=float, default=-1.0,
                    help="mixed solve: floor of the convergence test's bound on the last "
                         "components of a tridiagonal eigenvector (0: the tolerance; "
                         "negative, the default: 2^-24 x the Gershgorin bound of T, the "
                         "complex-float rounding level)")
    ap.add_argument("--mixed-recompute", action="store_true",
                    help="--workload mixed2M: also the mixed solve on the recompute product")
    ap.add_argument("--warm-train", type=int, default=64,
                    help="--workload warm: training dots")
    ap.add_argument("--warm-test", type=int, default=16, help="--workload warm: held-out dots")
    ap.add_argument("--warm-epochs", type=int, default=300, help="--workload warm: epochs")
    ap.add_argument("--workload", default="dot2M",
                    choices=["dot2M", "dome1M", "kernels", "mixed2M", "batch256", "vff1M", "warm",
                             "bdots"],
                    help="dot2M: the headline bench (mixed precision, 1,990,656 atoms); "
                         "dome1M: plain FP64, 8 e + 8 h on 1,022,656 atoms; the others: "
                         "measurements beside it")
    ap.add_argument("--bdots-cube", type=int, default=24,
                    help="--workload bdots: GaAs cube edge in cells")
    ap.add_argument("--ref-iterations", type=int, default=19802,
                    help="iterations of a full solve (both passes of the plain FP64 method) "
                         "the CPU sample is scaled to")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.profile_case:
        run_profile_case(args)
    elif args.workload not in ("dot2M", "dome1M"):
        if rank == 0:
            run_extra(args)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
