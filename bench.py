"""Benchmark of the matrix-free IGA Poisson MatMult on B200.

Workload (one "step" = one MatMult y = A x): the unit-square p=3 patch with
2048 x 2048 elements (2051^2 = 4,206,601 DOFs, 16 Gauss points per element),
FP64, precomputed symmetric 2x2 geometric factor (3 doubles per quadrature
point: the mult_sf path), x ~ U[-1,1] from the SplitMix64 stream with seed 1.
The on-the-fly-geometry variant (mult_mf path) is timed too and reported
under "variants".

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Our arm: device time of K back-to-back applies (CUDA events on the launching
stream, barrier + synchronize on both sides, max over ranks); e2e: the same
MatMult through iga_apply_host (host buffers in pinned memory, H2D + apply +
D2H per step). Reference arm: the reference's own CPU element code
(oracle/_ref/libigaref.so, compiled from the reference sources) on all host
cores over a bounded sample of the workload. With N > 1 GPUs every rank
applies the operator of its own patch (independent patches, no collective on
the data path): weak scaling.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "parallel-computing_b200")
METRIC = "GDOF/s per MatMult (p=3); time-to-1e-10 PCG: FP32+refine vs FP64, 1 B200"
P, NE = 3, 2048
SEED = 1
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 2 ** 20


def splitmix_uniform(seed, lo, hi, n):
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return lo + (hi - lo) * ((z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(name):
    """dram bytes per launch recorded from an ncu capture in profiles/<name>.md
    (a line 'traffic_bytes_per_launch: <int>'), or None."""
    path = os.path.join(ROOT, "profiles", f"{name}.md")
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch:"):
                return int(line.split(":", 1)[1].strip().split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [v for v in sm if v > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# --------------------------------------------------------------- reference arm
def ref_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libigaref.so")
    if os.path.exists(path):
        return ctypes.CDLL(path), "reference"
    return None, None


class CpuReference:
    """The reference's CPU MatMult on a p=3 ne^2 unit-square patch built by
    the reference's own preprocessing (oracle/_ref/libigaref.so): rate(path)
    times ElementMF + LocalAssemblyMF ("mf", the mult_mf path of
    matrix_free/iteration_number_fempc_mf.cpp) or ElementMFSF +
    LocalAssemblyMFSF ("sf", the mult_sf path), each in the element loop of
    GlobalAssemblyMF::MatMulMF, on `threads` host threads (element-row
    blocks, one per thread, like the reference's MPI ranks). Falls back to
    the C oracle restatement (one thread) when the compiled reference is
    absent."""

    def __init__(self, ne):
        self.L, self.kind = ref_lib()
        self.ne = ne
        m = ne + P
        self.nf = m * m
        self.x = splitmix_uniform(SEED, -1.0, 1.0, self.nf)
        self.y = np.zeros(self.nf)
        if self.L is None:
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from iga_testlib import Oracle, unit_square_mesh
            self.orc = Oracle()
            self.mesh = unit_square_mesh(self.orc, P, P, ne, ne)
            self.kind = "port"
            return
        vp = ctypes.c_void_p
        self.a = dict(CP=np.zeros(2 * self.nf), IEN=np.zeros(ne * ne * 16, np.int32), ID=np.zeros(self.nf, np.int32),
                      Dir=np.zeros(self.nf, np.int32), C1=np.zeros(ne * 16), C2=np.zeros(ne * 16), h1=np.zeros(ne),
                      h2=np.zeros(ne))
        ptr = lambda k: self.a[k].ctypes.data_as(vp)  # noqa: E731
        nd = ctypes.c_int()
        self.L.ref_mesh(P, P, ne, ne, ctypes.c_double(1.0), ctypes.c_double(1.0), ptr("CP"), ptr("IEN"), ptr("ID"),
                        ptr("Dir"), ctypes.byref(nd), ptr("C1"), ptr("C2"), ptr("h1"), ptr("h2"))
        self.args = [P, P, ne, ne, ptr("CP"), ptr("IEN"), ptr("ID"), ptr("Dir"), nd.value, ptr("C1"), ptr("C2"),
                     ptr("h1"), ptr("h2"), self.x.ctypes.data_as(vp), self.y.ctypes.data_as(vp)]

    def rate(self, path, reps, threads):
        """(GDOF/s, threads used, median seconds per MatMult)."""
        if self.L is None:
            threads = 1
            run = (lambda: self.orc.apply_mf(self.mesh, self.x)) if path == "mf" else \
                (lambda: self.orc.apply_sf(self.mesh, self.x))
        else:
            fn = self.L.ref_apply_mf if path == "mf" else self.L.ref_apply_sf
            run = lambda: fn(*self.args, threads)  # noqa: E731
        times = []
        for _ in range(reps):
            t0 = time.perf_counter()
            run()
            times.append(time.perf_counter() - t0)
        t = statistics.median(times)
        return self.nf / t / 1e9, threads, t


def cpu_reference_apply_rate(ne_sample, reps, threads, path="mf"):
    """GDOF/s of the reference's CPU MatMult on a p=3 ne_sample^2 patch."""
    ref = CpuReference(ne_sample)
    rate, threads, t = ref.rate(path, reps, threads)
    return rate, ref.kind, threads, t


def reference_arm(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    # the benchmark's own configuration, p=3 2048^2 (about 7 s per MatMult on 16 cores)
    ref = CpuReference(NE)
    reps_mf, reps_sf = max(1, min(args.steps, 3)), max(1, min(args.steps, 2))
    rate, threads, t = ref.rate("mf", reps_mf, threads)
    rate_sf, _, t_sf = ref.rate("sf", reps_sf, threads)
    sample = (f"the full workload, p=3 {NE}x{NE} elements ({(NE + P) ** 2} DOFs): median of {reps_mf} MatMults, "
              f"{t:.3f} s each")
    out = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "GDOF/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"matmul_p3_{NE}x{NE}_fp64_precomputed_geometry", "p": P, "nElem": [NE, NE],
                      "dofs": (NE + P) ** 2, "same_config": True,
                      "reference_path": "matrix_free ElementMF+LocalAssemblyMF (CPU, the mult_mf path: the faster "
                                        "of the reference's two CPU MatMults)"},
           "cpu_baseline": {"value": rate, "unit": "GDOF/s", "cores": threads, "kind": ref.kind, "sample": sample},
           "mult_sf": {"value": rate_sf, "unit": "GDOF/s", "cores": threads, "kind": ref.kind,
                       "ms_per_step": t_sf * 1e3,
                       "what": f"ElementMFSF + LocalAssemblyMFSF (the mult_sf path), same patch, median of "
                               f"{reps_sf} MatMults"},
           "e2e": {"value": rate, "unit": "GDOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    gk = reference_gpu_kernel_rate(NE, max(1, min(args.steps, 5)))
    if gk is not None:
        out["gpu_kernel"] = gk
    print(json.dumps(out), flush=True)


def reference_gpu_kernel_rate(ne, reps):
    """GDOF/s of the reference's own GPU MatMult kernel (matrix_free_gpu/src/
    mult.cu: one quadrature point per thread, 16-thread CTAs, atomicAdd
    scatter), compiled for sm_100a into oracle/_ref, on the same p=3 ne^2
    patch with its tables uploaded once (the reference re-uploads them on
    every call); None when that library or a GPU is absent."""
    try:
        import torch
    except ImportError:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from iga_testlib import RefGpuKernel
    if not torch.cuda.is_available() or not RefGpuKernel.available():
        return None
    k = RefGpuKernel(ne, ne)
    x = torch.from_numpy(splitmix_uniform(SEED, -1.0, 1.0, k.N)).cuda()
    y = torch.empty_like(x)
    k.apply(x.data_ptr(), y.data_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        k.apply(x.data_ptr(), y.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    k.close()
    return {"value": k.N / (ms * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_step": ms, "steps": reps,
            "what": f"the reference's MatrixFreeMatMultCUDA kernel (matrix_free_gpu/src/mult.cu) compiled for "
                    f"sm_100a, p=3 {ne}x{ne} patch, tables uploaded once, y zeroed each call"}


def time_solves(ib, torch, mesh, ne, barrier, max_over_ranks):
    """Time-to-solution of K u = F (f = 2 pi^2 sin(pi x) sin(pi y)) to a relative
    true residual of 1e-10: plain FP64 PCG vs FP32 PCG sweeps + FP64 refinement,
    both with the FEM preconditioner inverted exactly; plus the reference's
    preconditioner (inner Jacobi-CG to 1e-10) on the p=2 64x64 configuration."""
    out = {"problem": f"p=3 {ne}x{ne}, f=2pi^2 sin(pi x) sin(pi y), K u = F, rtol 1e-10 (true residual)",
           "pc": "bilinear-FEM matrix, exact inverse (x eigenvectors by GEMM, y tridiagonal solves; own FP64 DMMA / FP32 tcgen05 TF32 GEMMs)"}
    plan = ib.Plan(mesh, precision=ib.MIXED)
    b = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
    plan.rhs(b, ib.F_SINSIN)
    stream = torch.cuda.current_stream()
    # FP32 sweeps to 1e-3 (the library default): shallow sweeps restart the
    # Krylov space before FP32 rounding slows it down
    # fp64_pcg_fp32_pc: FP64 PCG whose preconditioner runs in FP32 (IGA_MIXED_PC)
    for name, kw in (("fp64", dict(pc=ib.PC_FEM_EXACT)),
                     ("fp32_refine", dict(pc=ib.PC_FEM_EXACT, precision=ib.MIXED, sweep_rtol=1e-3)),
                     ("fp64_pcg_fp32_pc", dict(pc=ib.PC_FEM_EXACT, precision=ib.MIXED_PC))):
        x = torch.zeros_like(b)
        plan.solve(b, x, **kw)   # warm-up: eigen-decomposition, tensor maps, loop graph, allocations
        times, st = [], None
        for _ in range(3):
            x.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = plan.solve(b, x, stream=stream, **kw)
            e1.record(stream)
            barrier()
            times.append(max_over_ranks(e0.elapsed_time(e1) / 1e3))
        out[name] = {"seconds": statistics.median(times), "iterations": st.iterations, "sweeps": st.sweeps,
                     "relres": st.relres, **({"sweep_rtol": kw["sweep_rtol"]} if "sweep_rtol" in kw else {})}
    out["speedup_fp32_refine_vs_fp64"] = out["fp64"]["seconds"] / out["fp32_refine"]["seconds"]
    plan.close()
    # mixed-precision configuration: NURBS quarter annulus, p=4, 1024x1024,
    # u = sin(pi r) sin(2 theta); error of the FP32+refine solution vs the FP64 one
    ma = ib.quarter_annulus(4, 1024)
    pa = ib.Plan(ma, precision=ib.MIXED)
    ba = torch.empty(pa.nfunc, dtype=torch.float64, device="cuda")
    pa.rhs(ba, ib.F_ANNULUS)
    xs = {}
    ann = {"problem": "quarter annulus r in [1,2] (NURBS, p=4), 1024x1024, u = sin(pi r) sin(2 theta), rtol 1e-10"}
    # FP32 sweeps to 1e-2 (measured fastest here: five shallow sweeps)
    for name, kw in (("fp64", dict(pc=ib.PC_FEM_EXACT)),
                     ("fp32_refine", dict(pc=ib.PC_FEM_EXACT, precision=ib.MIXED, sweep_rtol=1e-2)),
                     ("fp64_pcg_fp32_pc", dict(pc=ib.PC_FEM_EXACT, precision=ib.MIXED_PC))):
        x = torch.zeros_like(ba)
        pa.solve(ba, x, **kw)
        times = []
        for _ in range(3):
            x.zero_()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = pa.solve(ba, x, stream=stream, **kw)
            e1.record(stream)
            barrier()
            times.append(max_over_ranks(e0.elapsed_time(e1) / 1e3))
        xs[name] = x
        ann[name] = {"seconds": statistics.median(times), "iterations": st.iterations, "sweeps": st.sweeps,
                     "relres": st.relres, **({"sweep_rtol": kw["sweep_rtol"]} if "sweep_rtol" in kw else {})}
    ann["speedup_fp32_refine_vs_fp64"] = ann["fp64"]["seconds"] / ann["fp32_refine"]["seconds"]
    ann["rel_error_fp32_refine_vs_fp64"] = float((xs["fp32_refine"] - xs["fp64"]).norm() / xs["fp64"].norm())
    out["annulus_p4_1024"] = ann
    pa.close()
    del xs
    torch.cuda.empty_cache()
    # adjoint configuration: p=3 512x512, kappa = exp(g) (Gaussian random field,
    # sigma 1, squared-exponential length 0.1, seed 3), u_obs = u(exp(0.8 g)) + 1%
    # noise, J = |u - u_obs|^2 / 2; forward solve + adjoint solve + dJ/dkappa.
    out["adjoint_p3_512"] = time_adjoint(ib, torch, stream, barrier, max_over_ranks)
    out["batched_256"] = time_batch(ib, torch, stream, barrier, max_over_ranks)
    # spectra (Lanczos on the PCG coefficients): kappa(K) grows like h^-2, the
    # FEM-preconditioned kappa(M^-1 K) stays bounded
    spectra = {}
    for ne in (64, 256, 1024):
        ps = ib.Plan(ib.unit_square(3, ne))
        lo, hi, k = ps.spectrum(pc=ib.PC_NONE, steps=600)
        plo, phi, pk = ps.spectrum(pc=ib.PC_FEM_EXACT, steps=200)
        spectra[f"p3_{ne}x{ne}"] = {"kappa_K": hi / lo, "lanczos_steps_K": k, "kappa_fem_pc": phi / plo,
                                     "lambda_fem_pc": [plo, phi], "lanczos_steps_pc": pk}
        ps.close()
    out["spectra"] = spectra
    # reference preconditioner, p=2 64x64 (the CPU-runnable configuration), for
    # f = 2 pi^2 sin sin and for the reference's own load x(1-x)y(1-y)
    m2 = ib.unit_square(2, 64)
    p2 = ib.Plan(m2)
    b2 = torch.empty(p2.nfunc, dtype=torch.float64, device="cuda")
    x2 = torch.zeros_like(b2)
    ref_pc = {"pc": "inner Jacobi-CG on the FEM matrix to 1e-10 (the reference's PCSHELL)"}
    for name, fk in (("f_sinsin", ib.F_SINSIN), ("f_reference", ib.F_REFERENCE)):
        p2.rhs(b2, fk)
        p2.solve(b2, x2, pc=ib.PC_FEM_CG)
        st = p2.solve(b2, x2, pc=ib.PC_FEM_CG)
        ref_pc[name] = {"seconds": st.seconds, "iterations": st.iterations, "inner_iterations": st.pc_iterations,
                        "relres": st.relres}
    out["p2_64x64_reference_pc"] = ref_pc
    p2.close()
    torch.cuda.empty_cache()
    return out


def time_batch(ib, torch, stream, barrier, max_over_ranks):
    """256 independent unit-square solves (p uniform in {2, 3}, element counts per
    direction uniform in {32, 48, ..., 256}, b ~ N(0,1) with zero boundary data,
    seed 2) in one graph launch per batch solve, to a relative true residual of
    1e-10 per problem; FP64 PCG and FP32 PCG sweeps + FP64 refinement, exact FEM
    preconditioner, tile shapes from the committed tuning table."""
    shapes = ib.batch_problems(256, seed=2)
    meshes = [ib.unit_square(p, a, c) for p, a, c in shapes]
    b = torch.from_numpy(ib.batch_rhs(shapes, seed=2)).cuda()
    out = {"problems": "256 unit-square Poisson solves, p in {2,3}, nElemX, nElemY in {32,48,...,256} (seed 2), "
                       "b ~ N(0,1), rtol 1e-10 per problem",
           "dofs": int(b.numel()), "tune_file": os.path.basename(ib.TUNE_FILE)}
    # FP32 sweep tolerance: 3e-4 needs three sweeps here, like 1e-5, with fewer
    # FP32 iterations per sweep
    for name, prec, kw in (("fp64", ib.FP64, {}), ("fp32_refine", ib.MIXED, {"sweep_rtol": 3e-4})):
        # set-up is host-bound and the host is shared: the median of three
        # creations (the samples are reported too)
        setups = []
        for rep in range(3):
            t0 = time.perf_counter()
            batch = ib.Batch(meshes, precision=prec, tune_file=ib.TUNE_FILE)
            setups.append(time.perf_counter() - t0)
            if rep < 2:
                batch.close()
        setup = statistics.median(setups)
        x = torch.zeros_like(b)
        batch.solve(b, x, **kw)   # warm-up: graph capture and instantiation
        times, st, its = [], None, None
        for _ in range(3):
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, its, rel = batch.solve(b, x, stream=stream, **kw)
            e1.record(stream)
            barrier()
            times.append(max_over_ranks(e0.elapsed_time(e1) / 1e3))
        sec = statistics.median(times)
        out[name] = {"seconds": sec, "solves_per_s": 256 / sec, "setup_seconds": setup,
                     "setup_seconds_samples": [round(v, 4) for v in setups],
                     "converged": st.converged, "max_iterations": st.max_iterations,
                     "mean_iterations": float(its.mean()), "max_sweeps": st.max_sweeps, "max_relres": st.max_relres,
                     **({"sweep_rtol": kw["sweep_rtol"]} if kw else {})}
        batch.close()
    out["speedup_fp32_refine_vs_fp64"] = out["fp64"]["seconds"] / out["fp32_refine"]["seconds"]
    torch.cuda.empty_cache()
    return out


def time_adjoint(ib, torch, stream, barrier, max_over_ranks):
    m = ib.unit_square(3, 512)
    plan = ib.Plan(m)
    n = plan.nfunc
    g = ib.grf_qp(m, sigma=1.0, ell=0.1, seed=3)
    F = torch.empty(n, dtype=torch.float64, device="cuda")
    plan.rhs(F, ib.F_SINSIN)
    mside = 515
    bmask = torch.zeros(mside, mside, dtype=torch.bool, device="cuda")
    bmask[0, :] = bmask[-1, :] = bmask[:, 0] = bmask[:, -1] = True
    bmask = bmask.ravel()
    kw = dict(pc=ib.PC_FEM_EXACT, rtol=1e-10)
    KS = ib.kappa_solve_function()
    with torch.no_grad():
        u_true = KS.apply(torch.from_numpy(np.exp(0.8 * g)).cuda(), plan, F, bmask, kw)
    noise = torch.from_numpy(ib.splitmix_normal(3, n, offset=10 ** 7)).cuda()
    u_obs = u_true + 0.01 * float(u_true.abs().max()) * noise
    u_obs[bmask] = 0.0
    kappa = torch.from_numpy(np.exp(g)).cuda()

    def J_and_grad():
        k = kappa.clone().requires_grad_(True)
        u = KS.apply(k, plan, F, bmask, kw)
        J = 0.5 * ((u - u_obs) ** 2).sum()
        J.backward()
        return J, k.grad

    J_and_grad()   # warm-up
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    J, grad = J_and_grad()
    e1.record(stream)
    barrier()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    # directional derivative vs central differences (2 random directions, step 1e-6)
    errs = []
    for k in range(2):
        d = torch.from_numpy(ib.splitmix_normal(100 + k, kappa.numel())).cuda()
        with torch.no_grad():
            jp = 0.5 * ((KS.apply(kappa + 1e-6 * d, plan, F, bmask, kw) - u_obs) ** 2).sum()
            jm = 0.5 * ((KS.apply(kappa - 1e-6 * d, plan, F, bmask, kw) - u_obs) ** 2).sum()
        fd = float((jp - jm) / 2e-6)
        ad = float((grad * d).sum())
        errs.append(abs(fd - ad) / abs(ad))
    plan.close()
    torch.cuda.empty_cache()
    return {"problem": "p=3 512x512, kappa = exp(GRF), J = |u - u_obs|^2 / 2",
            "seconds_forward_adjoint_gradient": t, "J": float(J.detach()), "quadrature_points": int(kappa.numel()),
            "fd_directional_rel_err": errs}


# --------------------------------------------------------------- our arm
def our_arm(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    sys.path.insert(0, PKG)
    import iga_b200 as ib

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.profile_batch_pc:
        shapes = ib.batch_problems(256, seed=2)
        batch = ib.Batch([ib.unit_square(p, a, c) for p, a, c in shapes], precision=ib.MIXED,
                         tune_file=ib.TUNE_FILE)
        v = torch.from_numpy(splitmix_uniform(SEED, -1.0, 1.0, batch.ntot)).cuda()
        w = torch.empty_like(v)
        v32, w32 = v.float(), torch.empty_like(v, dtype=torch.float32)
        for _ in range(3):
            batch.pc_apply(v, w)
            batch.pc_apply(v32, w32, precision=ib.FP32)
            batch.apply(v, w)
            batch.apply(v32, w32, precision=ib.FP32)
        torch.cuda.synchronize()
        batch.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.profile_pc:
        # the exact FEM preconditioner of the p=3 patch (FP32 and FP64) and the
        # FP32 operator, a few applies outside any graph; then the same
        # preconditioner with the full (not parity-split) x transforms
        plan = ib.Plan(ib.unit_square(P, args.ne, args.ne), precision=ib.MIXED)
        r = torch.from_numpy(splitmix_uniform(SEED, -1.0, 1.0, plan.nfunc)).cuda()
        z = torch.empty_like(r)
        r32, z32 = r.float(), torch.empty_like(r, dtype=torch.float32)
        for _ in range(3):
            plan.pc_apply(r32, z32, pc=ib.PC_FEM_EXACT, precision=ib.FP32)
            plan.pc_apply(r, z, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
            plan.apply(r32, z32, precision=ib.FP32)
        torch.cuda.synchronize()
        plan.set_pc_split(0)
        for _ in range(3):
            plan.pc_apply(r32, z32, pc=ib.PC_FEM_EXACT, precision=ib.FP32)
            plan.pc_apply(r, z, pc=ib.PC_FEM_EXACT, precision=ib.FP64)
        torch.cuda.synchronize()
        plan.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.profile_annulus:
        # the operators of the mixed-precision solve (p=4 NURBS quarter annulus,
        # 1024x1024): FP32 (the sweeps) and FP64 (the outer residual), a few
        # applies outside any graph
        plan = ib.Plan(ib.quarter_annulus(4, 1024), precision=ib.MIXED)
        x = torch.from_numpy(splitmix_uniform(SEED, -1.0, 1.0, plan.nfunc)).cuda()
        y = torch.empty_like(x)
        x32, y32 = x.float(), torch.empty_like(x, dtype=torch.float32)
        for _ in range(4):
            plan.apply(x32, y32, precision=ib.FP32)
            plan.apply(x, y, precision=ib.FP64)
        torch.cuda.synchronize()
        plan.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.profile_solve:
        # the mixed-precision solve of the p=4 1024x1024 NURBS annulus cut to
        # one FP32 sweep of 12 iterations (a target for a per-iteration launch list)
        plan = ib.Plan(ib.quarter_annulus(4, 1024), precision=ib.MIXED)
        b = torch.empty(plan.nfunc, dtype=torch.float64, device="cuda")
        plan.rhs(b, ib.F_ANNULUS)
        x = torch.zeros_like(b)
        plan.set_solver_graph(0)   # iterations launched from the host: visible kernel by kernel
        plan.solve(b, x, check=False, pc=ib.PC_FEM_EXACT, precision=ib.MIXED, sweep_rtol=1e-2, max_it=12,
                   max_sweeps=1)
        torch.cuda.synchronize()
        plan.close()
        if dist is not None:
            dist.destroy_process_group()
        return

    if args.batch_only:
        res = time_batch(ib, torch, torch.cuda.current_stream(), barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps({"batched_256": res}), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    ne = args.ne
    mesh = ib.unit_square(P, ne, ne)
    N = (ne + P) ** 2
    x_host = splitmix_uniform(SEED + rank, -1.0, 1.0, N)
    xd = torch.from_numpy(x_host).cuda()
    yd = torch.empty_like(xd)
    stream = torch.cuda.current_stream()

    def timed_loop(plan, steps, warmup, flush=None):
        for _ in range(warmup):
            plan.apply(xd, yd, stream)
        barrier()
        if flush is None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                plan.apply(xd, yd, stream)
            e1.record(stream)
            barrier()
            ms = e0.elapsed_time(e1)
        else:
            ms = 0.0
            for _ in range(steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                plan.apply(xd, yd, stream)
                e1.record(stream)
                e1.synchronize()
                ms += e0.elapsed_time(e1)
            barrier()
        return max_over_ranks(ms)

    peak, peak_kind = measured_peaks()
    variants = {}
    if not args.skip_variants:
        # on-the-fly geometry (mult_mf): its inputs (x, control points) fit in
        # L2, so L2 is flushed between timed applies.
        flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
        plan_mf = ib.Plan(mesh, geometry=ib.GEOM_ON_THE_FLY)
        k_mf = max(1, min(args.steps, 200))
        ms_mf = timed_loop(plan_mf, k_mf, args.warmup, flush=flush)
        variants["on_the_fly_geometry"] = {
            "value": ws * N * k_mf / (ms_mf * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_step": ms_mf / k_mf,
            "algo_bytes_per_step": plan_mf.info.algo_bytes_f64, "l2": "flushed between timed applies"}
        plan_mf.close()
        del flush
        torch.cuda.empty_cache()
        # FP32 operator (precomputed FP32 G): the operator of the mixed-precision sweeps
        plan32 = ib.Plan(mesh, precision=ib.FP32, geometry=ib.GEOM_PRECOMPUTED)
        x32, y32 = xd.float(), torch.empty(N, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup):
            plan32.apply(x32, y32, stream)
        barrier()
        k32 = max(1, min(args.steps, 200))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k32):
            plan32.apply(x32, y32, stream)
        e1.record(stream)
        barrier()
        ms32 = max_over_ranks(e0.elapsed_time(e1))
        variants["fp32_precomputed_geometry"] = {
            "value": ws * N * k32 / (ms32 * 1e-3) / 1e9, "unit": "GDOF/s", "ms_per_step": ms32 / k32,
            "algo_bytes_per_step": plan32.info.algo_bytes_f32,
            "achieved_gbs": plan32.info.algo_bytes_f32 / (ms32 / k32 * 1e-3) / 1e9,
            "l2": "inputs larger than L2 (0.8 GB of FP32 geometry per apply)"}
        plan32.close()
        del x32, y32
        torch.cuda.empty_cache()

    plan = ib.Plan(mesh, geometry=ib.GEOM_PRECOMPUTED)
    algo = plan.info.algo_bytes_f64
    with ClockSampler(local) as clk:
        ms = timed_loop(plan, args.steps, args.warmup)
    clocks = clk.summary()
    value = ws * N * args.steps / (ms * 1e-3) / 1e9
    ms_step = ms / args.steps
    achieved = algo / (ms_step * 1e-3) / 1e9

    # e2e through the host-buffer C ABI call (pinned host memory).
    e2e = None
    if not args.no_e2e:
        xh = torch.from_numpy(x_host).pin_memory()
        yh = torch.empty_like(xh).pin_memory()
        xh_np, yh_np = xh.numpy(), yh.numpy()
        for _ in range(max(3, args.warmup // 4)):
            plan.apply_host(xh_np, yh_np)
        barrier()
        k_e2e = max(3, min(args.steps, 100))
        t0 = time.perf_counter()
        for _ in range(k_e2e):
            plan.apply_host(xh_np, yh_np)
        barrier()
        t_e2e = max_over_ranks(time.perf_counter() - t0)
        e2e = {"value": ws * N * k_e2e / t_e2e / 1e9, "unit": "GDOF/s", "h2d_bytes_per_step": 8 * N,
               "d2h_bytes_per_step": 8 * N, "call": "iga_apply_host (MATSHELL MatMult on host vectors)"}

    solve = None
    if not args.skip_solve:
        plan.close()
        torch.cuda.empty_cache()
        solve = time_solves(ib, torch, mesh, ne, barrier, max_over_ranks)
        plan = ib.Plan(mesh, geometry=ib.GEOM_PRECOMPUTED)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        ref = CpuReference(512)
        rate, threads, t = ref.rate("mf", 3, os.cpu_count() or 1)
        cpu = {"value": rate, "unit": "GDOF/s", "cores": threads, "kind": ref.kind,
               "sample": f"p=3 512x512-element patch ({515 ** 2} DOFs), median of 3 MatMults ({t:.3f} s each); "
                         "the per-element cost does not depend on the patch size"}
        rate_sf, _, t_sf = ref.rate("sf", 2, os.cpu_count() or 1)
        cpu["mult_sf"] = {"value": rate_sf, "unit": "GDOF/s", "cores": threads, "kind": ref.kind,
                          "sample": f"ElementMFSF + LocalAssemblyMFSF (the mult_sf path), same patch, median of 2 "
                                    f"MatMults ({t_sf:.3f} s each)"}
        del ref
        # the same element code on one core (the reference's per-rank rate)
        rate1, kind1, _, t1 = cpu_reference_apply_rate(128, 3, 1)
        cpu["one_core"] = {"value": rate1, "unit": "GDOF/s", "cores": 1, "kind": kind1,
                           "sample": f"p=3 128x128-element patch ({131 ** 2} DOFs), median of 3 MatMults "
                                     f"({t1:.3f} s each)"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "GDOF/s", "n_gpus": ws, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"matmul_p3_{ne}x{ne}_fp64_precomputed_geometry", "p": P,
                          "nElem": [ne, ne], "dofs_per_gpu": N, "quadrature_points_per_element": 16,
                          "geometry_bytes": plan.info.geom_bytes, "parallelism": f"replicas{ws}",
                          "l2": f"inputs larger than L2 ({plan.info.geom_bytes / 1e9:.2f} GB of geometry streamed per apply)",
                          "rows_per_strip": plan.info.rows_per_strip, "warps_per_cta": plan.info.warps_per_cta},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": profiled_traffic("apply_c2_p3_fp64_precomputed"),
                            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                            else "fallback 6650 GB/s",
                            "kernel": "apply_kernel + seam_fixup_kernel (one MatMult)",
                            "algo_bytes_per_launch": algo},
               "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks, "gpu_launches": 2 * args.steps,
               "variants": variants, "solve": solve}
        print(json.dumps(out), flush=True)
    plan.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ne", type=int, default=NE, help="elements per direction (profiling runs use smaller cases)")
    ap.add_argument("--skip-variants", action="store_true", help="skip the on-the-fly-geometry timing")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer timing")
    ap.add_argument("--skip-solve", action="store_true", help="skip the time-to-1e-10 solves")
    ap.add_argument("--batch-only", action="store_true",
                    help="time only the 256-problem batched solves (prints their JSON object)")
    ap.add_argument("--profile-pc", action="store_true",
                    help="run the exact FEM preconditioner (FP32, FP64) and the FP32 operator of the p=3 patch "
                         "(--ne) a few times outside any graph, then the preconditioner with full x transforms "
                         "(a target for ncu; prints nothing else)")
    ap.add_argument("--profile-annulus", action="store_true",
                    help="run the FP32 and FP64 operators of the p=4 1024x1024 NURBS annulus a few times "
                         "outside any graph (a target for ncu; prints nothing else)")
    ap.add_argument("--profile-solve", action="store_true",
                    help="run one 12-iteration FP32 sweep of the annulus mixed-precision solve with its "
                         "iterations launched from the host (a target for a per-iteration ncu launch list; prints "
                         "nothing else)")
    ap.add_argument("--profile-batch-pc", action="store_true",
                    help="run the batched preconditioner and operator of the 256-problem batch a few times "
                         "outside any graph (a target for ncu; prints nothing else)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
