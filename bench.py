"""Benchmark: Jacobi-PCG solves/s on the 256^3 7-point Poisson system.

Workload (plain FP64 path): interior 256^3 Poisson (16,777,216 rows,
117,047,296 non-zeros), CSR FP64, b = A x_true with x_true ~ U[0,1) from
numpy default_rng(1), x0 = 0, stop at ||r|| <= 1e-8 ||b||, every solve
verified by an FP64 recomputation of ||b - A x|| / ||b||.  Data are seeded
synthetic (no dataset is used).  A step is one complete solve; the matrix
and b stay resident in HBM (1.9 GB, far above the 126 MB L2, so no L2 flush
is needed between steps).

Also reported on the same line:
  roofline      the dominant kernel (the CSR SpMV), timed alone with CUDA
                events, algorithmic bytes 12 nnz + 4 (n+1) + 16 n per launch
  e2e           the same solves through the reference-facing ELM interface
                (celg_elm_doit + celg_elm_collect_solution: b copied from
                pinned host memory, x copied back) inside the timed region
  forms         the other configurations, each against its plain FP64
                counterpart on the GPU: FP32 refinement on the 256^3
                lognormal-coefficient diffusion system (rel-res 1e-10), 64
                batched uneven systems, 32 right-hand sides on 128^3, and the
                adjoint gradients of a batch of 8 128^3 diffusion solves
  cpu_baseline  the C restatement of the reference's MPI+OpenMP PCG (oracle/)
                on the host cores: one complete solve of the same system
  summary       last on the line: one number per form, and the parity of the
                headline solve against that oracle solve (b = A x_true and the
                JAD permutation bit for bit; residual history and solution
                within 1e-10 relative, iterations +-1)

--impl reference times that CPU restatement alone (the Fortran reference
cannot be built here: no Fortran compiler or MPI), each step a bounded sample
of iterations of the same solve, scaled to solves/s.

Multi-GPU (torchrun, N > 1): every rank solves its own copy of the system
(independent replicas, no collective on the data path); value = all ranks'
solves / max-over-ranks time.  Reported beside it (forms.distributed_256):
the row-block solve of one 256^3 system over all N GPUs (z-slabs, halo and
all-reduces over NCCL inside the library call), max-over-ranks time.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIDE = 256
SEED = 1
EPS_REL = 1e-8
METRIC = "PCG solves/s at 256^3 to rel-res 1e-8 (Jacobi-PCG, CSR FP64)"
UNIT = "solves/s"


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel_tag):
    """dram bytes per launch of the kernel from the committed ncu summary."""
    for f in sorted(os.listdir(os.path.join(ROOT, "profiles"))) if os.path.isdir(
            os.path.join(ROOT, "profiles")) else []:
        if not f.endswith((".txt", ".md")):
            continue
        for line in open(os.path.join(ROOT, "profiles", f)):
            m = re.match(r"\s*dram_bytes_per_launch\[(\w+)\]\s*=\s*([0-9.eE+]+)", line)
            if m and m.group(1) == kernel_tag:
                return float(m.group(2)), f
    return None, None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def rel_err(x, ref):
    """max |x - ref| / max |ref| of two device vectors."""
    return float((x - ref).abs().max() / ref.abs().max())


def build_problem():
    from cel_v3_b200 import synth
    rp, ci, v, x_true = synth.plain(SIDE, SEED)
    return rp, ci, v, x_true


def plain_large_form(h, celgpu, torch, stream, m, b, x, iters_csr):
    """The rest of the plain-large configuration: the SpMV bandwidth sweep at
    64^3, 128^3 and 256^3 (CSR and JAD; the two smaller sizes fit the 126 MB
    L2), Jacobi-PCG in JAD format and restarted GMRES(30)-Jacobi in CSR on
    the 256^3 system, each to rel-res 1e-8."""
    from cel_v3_b200 import synth
    peak, _ = measured_peaks()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"spmv_sweep": {}}

    def time_it(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, r

    for side in (64, 128, 256):
        rp, ci, v = synth.poisson7(side)
        n, nnz = rp.size - 1, int(rp[-1])
        mm = m if side == 256 else h.matrix_from_csr(rp, ci, v)
        perm = mm.to_jad()
        if side == 256:
            out["jad_perm"] = perm
        xs = torch.from_numpy(np.random.default_rng(1).random(n)).cuda()
        ys = torch.zeros(n, dtype=torch.float64, device="cuda")
        row = {}
        # JAD reads no column data when the matrix has row patterns: 8 bytes
        # per non-zero and one pattern byte per row instead of 12
        pat = mm.column_form() == celgpu.COLS_PATTERN
        jad_bytes = (8 * nnz + n if pat else 12 * nnz) + 4 * 8 + 20 * n
        row["jad_columns"] = "row patterns" if pat else "int32"
        for name, fmt, nbytes in (("csr", celgpu.FMT_CSR, 12 * nnz + 4 * (n + 1) + 16 * n),
                                  ("jad", celgpu.FMT_JAD, jad_bytes)):
            ms, _ = time_it(lambda: h.spmv(mm, xs.data_ptr(), ys.data_ptr(), fmt=fmt), 50)
            gbs = nbytes / (ms / 1e3) / 1e9
            row[name] = {"ms": ms, "gbs": gbs, "frac_of_measured": gbs / peak, "bytes": nbytes}
        row["l2_resident"] = side < 256
        out["spmv_sweep"][f"{side}^3"] = row
        if mm is not m:
            mm.destroy()
    pj = celgpu.params(eps_rel=EPS_REL, iter_max=5000, x0_mode=celgpu.X0_ZERO, fmt=celgpu.FMT_JAD)
    ms, inf = time_it(lambda: h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), pj), 2)
    out["pcg_jad_256"] = {"solves_per_s": 1e3 / ms, "ms": ms, "iters": inf.iter_done,
                          "verified_relres": inf.verified_relres, "status": inf.status,
                          "csr_iters": iters_csr}
    pg = celgpu.params(eps_rel=EPS_REL, iter_max=2000, x0_mode=celgpu.X0_ZERO, restart=30)
    ms, inf = time_it(lambda: h.gmres_jacobi(m, b.data_ptr(), x.data_ptr(), pg), 1)
    out["gmres30_csr_256"] = {"solves_per_s": 1e3 / ms, "ms": ms, "restarts": inf.iter_done,
                              "arnoldi_steps": inf.arnoldi_steps,
                              "verified_relres": inf.verified_relres, "status": inf.status}
    return out


def distributed_form(h, celgpu, torch, stream, rp, ci, v, b_host, rank, world, local,
                     max_over_ranks, barrier, reps=2):
    """The row-block Jacobi-PCG of one 256^3 system over all ranks: z-slabs,
    one per GPU (strong scaling), each rank's whole solve one library call
    (celg_dist_pcg_solve_nccl: per iteration the halo of p and two
    all-reduces of 5 doubles over the library's own NCCL communicator).  At
    world size 1 it is the cost of that path against the single-graph solve.
    Also timed with the halo of p overlapped with the interior rows' SpMV."""
    from cel_v3_b200 import dist as D
    n = rp.size - 1
    blk = D.RowBlock(rp, ci, v, D.partition(n, world, SIDE * SIDE), rank)
    rk = D.GpuRank(h, blk, b_host[blk.r0:blk.r1], eps_rel=EPS_REL, iter_max=5000)
    comm = D.nccl_communicator(rank, world, local)
    out = {"world": world, "rows_per_rank": blk.n, "scaling": "strong", "poll_every": 8,
           "api": "celg_dist_pcg_solve_nccl"}
    try:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for overlap in (False, True):
            rk.solve_nccl(comm, poll_every=8, overlap=overlap)
            barrier()
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                res = rk.solve_nccl(comm, poll_every=8, overlap=overlap)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / reps)
            key = "overlap" if overlap else "plain"
            out[key] = {"solves_per_s": 1e3 / ms, "ms": ms, "iters": res.iter_done,
                        "verified_relres": res.verified_relres, "status": res.status}
        out["solves_per_s"] = max(out["plain"]["solves_per_s"], out["overlap"]["solves_per_s"])
    finally:
        rk.close()
        celgpu.nccl_comm_destroy(comm)
    return out


def precision_form(h, celgpu, torch, stream, side=256, reps=2):
    """-div(k grad u) on side^3, k = exp(g), g ~ N(0,1) per face (seed 2),
    b ~ U[-1,1) (seed 3), assembled in device memory: plain FP64 PCG, FP32
    refinement (restarted inner PCG, inner tol 1e-4) and FP32 PCG with FP64
    reliable updates, each to FP64-verified rel-res 1e-10."""
    from cel_v3_b200 import synth
    g, _ = synth.lognormal_faces(np.random.default_rng(2), side, side, side)
    rp_d, ci_d, v_d = synth.diffusion7_device(side, side, side, np.exp(g))
    n, nnz = side ** 3, int(ci_d.numel())
    m = h.matrix_from_csr_device(n, nnz, rp_d.data_ptr(), ci_d.data_ptr(), v_d.data_ptr()).jacobi()
    del rp_d, ci_d, v_d
    b = torch.from_numpy(np.random.default_rng(3).uniform(-1.0, 1.0, n)).cuda()
    x = torch.zeros_like(b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {"rows": n, "nnz": nnz, "rel_res": 1e-10}
    x64 = None
    for name, kw in (("fp64_pcg", dict()),
                     ("fp32_ir", dict(precision=celgpu.PREC_FP32_IR, inner_eps_rel=1e-4)),
                     ("fp32_ru", dict(precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2))):
        pf = celgpu.params(eps_rel=1e-10, iter_max=20000, x0_mode=celgpu.X0_ZERO, **kw)
        h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), pf)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            inf = h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), pf)
        e1.record(stream)
        torch.cuda.synchronize()
        fms = e0.elapsed_time(e1) / reps
        out[name] = {"solves_per_s": 1e3 / fms, "ms": fms, "iters": inf.iter_done,
                     "inner_iters": inf.arnoldi_steps, "verified_relres": inf.verified_relres,
                     "status": inf.status}
        if x64 is None:
            x64 = x.clone()
        else:
            out[name]["err_vs_fp64"] = rel_err(x, x64)
    base = out["fp64_pcg"]["solves_per_s"]
    for k in ("fp32_ir", "fp32_ru"):
        out[k]["speedup_vs_fp64"] = out[k]["solves_per_s"] / base
    # the block-Jacobi preconditioner (8-row blocks) on the same system, FP64
    m.block_jacobi(8)
    pf = celgpu.params(eps_rel=1e-10, iter_max=20000, x0_mode=celgpu.X0_ZERO,
                       precond=celgpu.PRECOND_BLOCK_JACOBI)
    h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), pf)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        inf = h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), pf)
    e1.record(stream)
    torch.cuda.synchronize()
    fms = e0.elapsed_time(e1) / reps
    out["fp64_pcg_block_jacobi8"] = {"solves_per_s": 1e3 / fms, "ms": fms, "iters": inf.iter_done,
                                     "verified_relres": inf.verified_relres, "status": inf.status,
                                     "speedup_vs_fp64": 1e3 / fms / base,
                                     "err_vs_fp64": rel_err(x, x64)}
    out["err_vs_fp64"] = ("max |x - x_fp64| / max |x_fp64|, x_fp64 = the plain FP64 PCG "
                          "solution of the same system (rel-res 1e-10)")
    m.destroy()
    return out


def batch_form(h, celgpu, torch, stream):
    """64 variable-coefficient systems (sides 16..96, seed 4) to rel-res 1e-8:
    one batched launch against the plain path solving them one by one."""
    from cel_v3_b200 import synth
    probs = synth.batch_problems()
    mats = [h.matrix_from_csr(rp, ci, v).jacobi() for _, rp, ci, v, _ in probs]
    bs = [torch.from_numpy(b).cuda() for *_, b in probs]
    xs = [torch.zeros_like(b) for b in bs]
    p = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def one_by_one():
        return [h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), p) for m, b, x in zip(mats, bs, xs)]

    def batched():
        return h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], p)

    # the FP32-refinement variant: FP32 inner solves (tol 1e-4) inside FP64
    # refinement of every system, to the same FP64-verified 1e-8
    p32 = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO,
                        precision=celgpu.PREC_FP32_IR, inner_eps_rel=1e-4, inner_iter_max=5000)

    def batched_fp32_ir():
        return h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], p32)

    # FP32 PCG with FP64 reliable updates of every system
    p32ru = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO,
                          precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)

    def batched_fp32_ru():
        return h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], p32ru)

    out = {}
    x64 = None
    for name, fn in (("one_by_one", one_by_one), ("batched", batched),
                     ("batched_fp32_ir", batched_fp32_ir), ("batched_fp32_ru", batched_fp32_ru)):
        fn()
        torch.cuda.synchronize()
        reps = 3
        e0.record(stream)
        for _ in range(reps):
            infos = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "solves_per_s": len(mats) * 1e3 / ms,
                     "max_iters": max(i.iter_done for i in infos),
                     "sum_iters": sum(i.iter_done for i in infos),
                     "worst_verified_relres": max(i.verified_relres for i in infos),
                     "all_ok": all(i.status == celgpu.OK for i in infos)}
        if name == "batched":
            x64 = [x.clone() for x in xs]
        elif name in ("batched_fp32_ir", "batched_fp32_ru"):
            out[name]["worst_err_vs_fp64"] = max(rel_err(x, y) for x, y in zip(xs, x64))
    out["speedup_batched_vs_one_by_one"] = out["batched"]["solves_per_s"] / out["one_by_one"]["solves_per_s"]
    out["speedup_batched_fp32_ir_vs_one_by_one"] = (out["batched_fp32_ir"]["solves_per_s"] /
                                                    out["one_by_one"]["solves_per_s"])
    out["speedup_batched_fp32_ru_vs_one_by_one"] = (out["batched_fp32_ru"]["solves_per_s"] /
                                                    out["one_by_one"]["solves_per_s"])
    out["systems"] = len(mats)
    out["rows"] = int(sum(s ** 3 for s, *_ in probs))
    csr_ctas, sweep_ctas = h.tuned_config(celgpu.TUNE_BATCH)
    out["tuned_launch"] = {"spmv_ctas_per_sm": csr_ctas or "max resident",
                           "vector_sweep_ctas_per_sm": sweep_ctas}
    for m in mats:
        m.destroy()
    return out


def multirhs_form(h, celgpu, torch, stream):
    """128^3 Poisson with 32 right-hand sides ~ U[-1,1) (seed 5) to rel-res 1e-8:
    one multi-RHS solve against 32 single solves."""
    from cel_v3_b200 import synth
    rp, ci, v, B = synth.multirhs_problem()
    n, k = B.shape
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    Bd = torch.from_numpy(B).cuda()
    Xd = torch.zeros_like(Bd)
    cols = [Bd[:, c].contiguous() for c in range(k)]
    xs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(k)]
    p = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = {}
    p32 = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO,
                        precision=celgpu.PREC_FP32_IR, inner_eps_rel=1e-4, inner_iter_max=5000)
    p32ru = celgpu.params(eps_rel=1e-8, iter_max=5000, x0_mode=celgpu.X0_ZERO,
                          precision=celgpu.PREC_FP32_RU, inner_eps_rel=1e-2)
    runs = (("one_by_one", lambda: [h.pcg_jacobi(m, c.data_ptr(), x.data_ptr(), p) for c, x in zip(cols, xs)]),
            ("multirhs", lambda: h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), p)),
            ("multirhs_fp32_ir", lambda: h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), p32)),
            ("multirhs_fp32_ru", lambda: h.pcg_multirhs(m, k, Bd.data_ptr(), Xd.data_ptr(), p32ru)))
    for name, fn in runs:
        fn()
        torch.cuda.synchronize()
        reps = 2
        e0.record(stream)
        for _ in range(reps):
            infos = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        out[name] = {"ms": ms, "solves_per_s": k * 1e3 / ms,
                     "max_iters": max(i.iter_done for i in infos),
                     "worst_verified_relres": max(i.verified_relres for i in infos),
                     "all_ok": all(i.status == celgpu.OK for i in infos)}
        if name == "multirhs":
            X64 = Xd.clone()
        elif name in ("multirhs_fp32_ir", "multirhs_fp32_ru"):
            out[name]["worst_err_vs_fp64"] = max(rel_err(Xd[:, c], X64[:, c]) for c in range(k))
        if name == "multirhs_fp32_ru":
            out[name]["max_reliable_updates"] = max(i.arnoldi_steps for i in infos)
    out["tuned_spmm_variant"], out["tuned_spmm32_shape"] = h.tuned_config(celgpu.TUNE_SPMM)
    out["speedup_multirhs_vs_one_by_one"] = out["multirhs"]["solves_per_s"] / out["one_by_one"]["solves_per_s"]
    out["speedup_multirhs_fp32_ir_vs_one_by_one"] = (out["multirhs_fp32_ir"]["solves_per_s"] /
                                                     out["one_by_one"]["solves_per_s"])
    out["speedup_multirhs_fp32_ru_vs_one_by_one"] = (out["multirhs_fp32_ru"]["solves_per_s"] /
                                                     out["one_by_one"]["solves_per_s"])
    m.destroy()
    return out


def differentiation_form(h, celgpu, torch, stream, side=128, batch=8, fd_dirs=64, step=1e-6):
    """Gradients of L = 0.5 ||x - x_target||^2, x = A(k)^{-1} b, k = exp(g) per
    face of a side^3 7-point diffusion operator, for `batch` instances (seeds
    6 and 7): one batched forward solve, one batched adjoint solve
    (A lambda = x - x_target; A is symmetric), the face gradients
    dL/dk = -(lambda_i - lambda_j)(x_i - x_j) (boundary: -lambda_i x_i) and
    dL/dg = k dL/dk.  Checked by central differences of L along random unit
    directions of g (instance 0), each perturbed operator rebuilt in device
    memory from the face map."""
    from cel_v3_b200 import synth
    probs = synth.differentiation_problems(side, batch)
    n = side ** 3
    cx, cy, cz = synth.face_counts(side, side, side)
    eps = 1e-10
    p = celgpu.params(eps_rel=eps, iter_max=20000, x0_mode=celgpu.X0_ZERO)
    # finite differences resolve 1e-6 steps only with tighter solves
    p_fd = celgpu.params(eps_rel=1e-13, iter_max=20000, x0_mode=celgpu.X0_ZERO)

    def operator(g_d):
        rp_d, ci_d, v_d = synth.diffusion7_device(side, side, side, torch.exp(g_d))
        return h.matrix_from_csr_device(n, int(ci_d.numel()), rp_d.data_ptr(), ci_d.data_ptr(),
                                        v_d.data_ptr()).jacobi()

    gs = [torch.from_numpy(g).cuda() for g, _, _ in probs]
    bs = [torch.from_numpy(b).cuda() for _, b, _ in probs]
    xts = [torch.from_numpy(xt).cuda() for _, _, xt in probs]
    mats = [operator(g) for g in gs]
    xs = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in probs]
    lams = [torch.zeros_like(x) for x in xs]
    gks = [torch.zeros(cx + cy + cz, dtype=torch.float64, device="cuda") for _ in probs]
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))

    def forward():
        return h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs], p)

    def backward():
        rhs = [x - xt for x, xt in zip(xs, xts)]
        infos = h.pcg_batched(mats, [r.data_ptr() for r in rhs], [l.data_ptr() for l in lams], p)
        for lam, x, gk in zip(lams, xs, gks):
            h.diffusion7_face_grad(side, side, side, lam.data_ptr(), x.data_ptr(), gk.data_ptr(),
                                   gk[cx:].data_ptr(), gk[cx + cy:].data_ptr())
        return infos, [torch.exp(g) * gk for g, gk in zip(gs, gks)]

    forward()
    backward()
    torch.cuda.synchronize()
    e0.record(stream)
    fi = forward()
    e1.record(stream)
    bi, dLdg = backward()
    e2.record(stream)
    torch.cuda.synchronize()
    fwd_ms, bwd_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)

    def loss(g_d, b_d, xt_d):
        m = operator(g_d)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        info = h.pcg_jacobi(m, b_d.data_ptr(), x.data_ptr(), p_fd)
        m.destroy()
        return 0.5 * float(((x - xt_d) ** 2).sum()), info

    rng = np.random.default_rng(64)
    g0, b0, xt0, d0 = gs[0], bs[0], xts[0], dLdg[0]
    scale = float(d0.abs().max())
    errs = []
    for _ in range(fd_dirs):
        d = torch.from_numpy(rng.standard_normal(g0.numel())).cuda()
        d /= torch.linalg.vector_norm(d)
        lp, _ = loss(g0 + step * d, b0, xt0)
        lm, _ = loss(g0 - step * d, b0, xt0)
        fd = (lp - lm) / (2 * step)
        errs.append(abs(fd - float(d0 @ d)) / max(abs(fd), scale))
    e = torch.from_numpy(rng.standard_normal(n)).cuda()
    e /= torch.linalg.vector_norm(e)
    lp, _ = loss(g0, b0 + step * e, xt0)
    lm, _ = loss(g0, b0 - step * e, xt0)
    db_err = abs((lp - lm) / (2 * step) - float(lams[0] @ e)) / float(lams[0].abs().max())
    for m in mats:
        m.destroy()
    return {"instances": batch, "rows_per_instance": n, "faces_per_instance": cx + cy + cz,
            "rel_res": eps, "fd_rel_res": 1e-13, "forward_ms": fwd_ms, "backward_ms": bwd_ms,
            "backward_over_forward": bwd_ms / fwd_ms,
            "gradients_per_s": batch * 1e3 / (fwd_ms + bwd_ms),
            "forward_max_iters": max(i.iter_done for i in fi),
            "adjoint_max_iters": max(i.iter_done for i in bi),
            "all_ok": all(i.status == celgpu.OK for i in list(fi) + list(bi)),
            "fd_check": {"directions": fd_dirs, "step": step,
                         "max_rel_err_dLdg": max(errs), "rel_err_dLdb": db_err,
                         "scale": "max(|fd|, max|dL/dg|)"}}


def forms_summary(forms, value):
    """One number per form: each speed-up against its plain FP64 GPU
    counterpart, the FP32 forms' errors against the FP64 solutions."""
    def g(*keys):
        d = forms
        for k in keys:
            if not isinstance(d, dict) or k not in d:
                return None
            d = d[k]
        return float(f"{d:.4g}") if isinstance(d, float) else d

    out = {
        "fp32_ru_x": g("precision_diffusion256", "fp32_ru", "speedup_vs_fp64"),
        "fp32_ir_x": g("precision_diffusion256", "fp32_ir", "speedup_vs_fp64"),
        "fp32_ru_err": g("precision_diffusion256", "fp32_ru", "err_vs_fp64"),
        "fp32_ir_err": g("precision_diffusion256", "fp32_ir", "err_vs_fp64"),
        "fp64_diffusion_solves_s": g("precision_diffusion256", "fp64_pcg", "solves_per_s"),
        "batched_x": g("batched_64", "speedup_batched_vs_one_by_one"),
        "batched_fp32_ir_x": g("batched_64", "speedup_batched_fp32_ir_vs_one_by_one"),
        "batched_fp32_ru_x": g("batched_64", "speedup_batched_fp32_ru_vs_one_by_one"),
        "multirhs_x": g("multirhs_128_k32", "speedup_multirhs_vs_one_by_one"),
        "multirhs_fp32_ir_x": g("multirhs_128_k32", "speedup_multirhs_fp32_ir_vs_one_by_one"),
        "multirhs_fp32_ru_x": g("multirhs_128_k32", "speedup_multirhs_fp32_ru_vs_one_by_one"),
        "grad_per_s": g("differentiation_128_b8", "gradients_per_s"),
        "grad_fd_err": g("differentiation_128_b8", "fd_check", "max_rel_err_dLdg"),
        "jad_pcg_solves_s": g("plain_large_256", "pcg_jad_256", "solves_per_s"),
        "gmres30_solves_s": g("plain_large_256", "gmres30_csr_256", "solves_per_s"),
        "spmv256_csr_frac": g("plain_large_256", "spmv_sweep", "256^3", "csr", "frac_of_measured"),
        "spmv256_jad_frac": g("plain_large_256", "spmv_sweep", "256^3", "jad", "frac_of_measured"),
    }
    dist = g("distributed_world1_256", "solves_per_s")
    if dist is not None:
        out["dist_world1_x"] = float(f"{dist / value:.4g}")
    dist = g("distributed_256", "solves_per_s")
    if dist is not None:
        out["dist_solves_s"] = dist
    return {k: v for k, v in out.items() if v is not None}


def cpu_baseline_and_parity(h, celgpu, torch, m, rp, ci, v, x_true, b, p, perm_gpu):
    """The CPU baseline and the parity of the headline solve.

    Baseline: one complete solve of the oracle's reference-order Jacobi-PCG
    (the C restatement of cel_cgalg_jacobi with the reference's thread model:
    an idle master plus one OpenMP worker per other host core), timed on the
    host cores; plus a bounded sample with one worker.

    Parity, against that same oracle solve and the oracle's row sums: the
    GPU's b = A x_true bit for bit, the JAD permutation bit for bit, and the
    GPU solve's residual history and solution within 1e-10 relative at the
    same iteration count +-1."""
    from oracle import celref as R
    cores = os.cpu_count() or 1
    workers = max(1, cores - 1)
    n = rp.size - 1
    b_ref = R.spmv_csr(rp, ci, v, x_true, nworkers=workers)
    b_host = b.cpu().numpy()
    perm_ref, _ = R.jad_perm(rp)
    if perm_gpu is None:
        perm_gpu = m.to_jad()
    xg = torch.zeros(n, dtype=torch.float64, device="cuda")
    info = h.pcg_jacobi(m, b.data_ptr(), xg.data_ptr(), p, history=True)
    x_gpu = xg.cpu().numpy()
    A = R.Matrix(rp, ci, v)
    J = R.jacobi(R.diag(rp, ci, v))
    t0 = time.perf_counter()
    xs, io = R.pcg_jacobi(A, J, b_ref, eps_rel=EPS_REL, iter_max=5000, red=R.RED_SEQ,
                          nworkers=workers)
    t_full = time.perf_counter() - t0
    t0 = time.perf_counter()
    R.pcg_jacobi(A, J, b_ref, eps_rel=0.0, eps_abs=0.0, iter_max=4, red=R.RED_SEQ, nworkers=1)
    t1 = time.perf_counter() - t0
    k = min(len(io["history"]), len(info.history))
    hist_rel = float(np.max(np.abs(info.history[:k] - io["history"][:k]) / io["history"][:k]))
    x_rel = float(np.abs(x_gpu - xs).max() / np.abs(xs).max())
    parity = {"spmv_256_bitexact": bool(np.array_equal(b_host, b_ref)),
              "jad_perm_256_bitexact": bool(np.array_equal(perm_gpu, perm_ref)),
              "iters_gpu": info.iter_done, "iters_ref": io["iter_done"],
              "pcg_256_hist_max_rel": hist_rel, "pcg_256_x_max_rel": x_rel,
              "pass": bool(np.array_equal(b_host, b_ref) and np.array_equal(perm_gpu, perm_ref)
                           and abs(info.iter_done - io["iter_done"]) <= 1 and hist_rel < 1e-10
                           and x_rel < 1e-10),
              "ref": f"oracle reference order, {workers} workers"}
    cpu = {"value": 1.0 / t_full, "unit": UNIT, "cores": cores, "threads": workers + 1,
           "kind": "port",
           "sample": f"one complete oracle Jacobi-PCG solve (reference order, {workers} workers + "
                     f"idle master) of the 256^3 system: {io['iter_done']} iterations in "
                     f"{t_full:.2f} s",
           "one_worker": {"value": 1.0 / (t1 / 5 * io["iter_done"]), "unit": UNIT, "threads": 1,
                          "sample": f"4 iterations + set-up in {t1:.2f} s, scaled by "
                                    f"{io['iter_done']} iterations per solve"}}
    return cpu, parity


def run_reference(args):
    """--impl reference: the CPU restatement of the reference path, timed."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from oracle import celref as R
    rp, ci, v, x_true = build_problem()
    b = R.spmv_csr(rp, ci, v, x_true, nworkers=max(1, (os.cpu_count() or 2) - 1))
    cores = os.cpu_count() or 1
    workers = max(1, cores - 1)
    A = R.Matrix(rp, ci, v)
    J = R.jacobi(R.diag(rp, ci, v))
    # iterations of a full solve: the recurrence is the same as the GPU's; the
    # count is taken from one full reference-order solve
    t0 = time.perf_counter()
    _, full = R.pcg_jacobi(A, J, b, eps_rel=EPS_REL, iter_max=5000, red=R.RED_SEQ, nworkers=workers)
    t_full = time.perf_counter() - t0
    iters = full["iter_done"]
    sample_iters = max(2, int(round(6.0 / max(t_full / max(iters, 1), 1e-4))))
    sample_iters = min(sample_iters, iters)

    def step():
        R.pcg_jacobi(A, J, b, eps_rel=0.0, eps_abs=0.0, iter_max=sample_iters, red=R.RED_SEQ,
                     nworkers=workers)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    t = time.perf_counter() - t0
    per_iter = t / (args.steps * (sample_iters + 1))
    value = 1.0 / (per_iter * iters)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "poisson7_256^3_pcg_jacobi_csr_fp64", "rows": int(rp.size - 1),
                   "nnz": int(rp[-1]), "rel_res": EPS_REL, "x0": "zero",
                   "reference_iterations": iters, "reference_full_solve_s": t_full,
                   "sample_iterations_per_step": sample_iters},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "threads": workers + 1,
                         "kind": "port",
                         "sample": f"{args.steps} steps of {sample_iters} PCG iterations, scaled "
                                   f"by the {iters} iterations of a full reference-order solve"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the Fortran reference cannot be built here (no gfortran/MPI); this arm times "
                "oracle/, the C restatement of its MPI+OpenMP path, at mpirun -n 1",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from cel_v3_b200 import celgpu

    rp, ci, v, x_true = build_problem()
    n, nnz = rp.size - 1, int(rp[-1])
    stream = torch.cuda.current_stream()
    h = celgpu.Handle(local, stream.cuda_stream)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    xt = torch.from_numpy(x_true).cuda()
    b = torch.empty(n, dtype=torch.float64, device="cuda")
    h.spmv(m, xt.data_ptr(), b.data_ptr())            # b = A x_true (bit-exact to the oracle)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = celgpu.params(eps_rel=EPS_REL, iter_max=5000, x0_mode=celgpu.X0_ZERO)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(val):
        if world == 1:
            return val
        t = torch.tensor([val], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident solves (value) ----
    infos = []
    for _ in range(args.warmup):
        infos.append(h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), p))
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        infos.append(h.pcg_jacobi(m, b.data_ptr(), x.data_ptr(), p))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(ms)
    last = infos[-1]
    assert all(i.status == celgpu.OK for i in infos), [i.status for i in infos]
    iters = last.iter_done
    value = world * args.steps / (ms / 1e3)
    ms_per_step = ms / args.steps
    # algorithmic bytes of one iteration, as the library accounts them for the
    # solve it ran: K1 (matrix, p gathered, v stored), K2 (r, v, J read, r
    # stored), K3 (p, r, J, x read, p, x stored); the matrix is 9 bytes per
    # non-zero with 1-byte column offsets, else 12
    pcg_bytes = int(h.elm_performance()[2])

    # ---- roofline: the CSR SpMV kernel alone ----
    y = torch.empty_like(b)
    for _ in range(3):
        h.spmv(m, xt.data_ptr(), y.data_ptr())
    reps = 50
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        h.spmv(m, xt.data_ptr(), y.data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = e0.elapsed_time(e1) / reps
    spmv_bytes = 12 * nnz + 4 * (n + 1) + 16 * n
    peak, peak_kind = measured_peaks()
    achieved = spmv_bytes / (spmv_ms / 1e3) / 1e9
    traffic, traffic_src = ncu_traffic("spmv_csr_256")

    # ---- other precision forms on the same system (reported, not the value) ----
    forms = {}
    # the other configurations are single-GPU measurements (run at N = 1)
    if not args.quick and world == 1:
        forms["precision_diffusion256"] = precision_form(h, celgpu, torch, stream)
        forms["batched_64"] = batch_form(h, celgpu, torch, stream)
        forms["multirhs_128_k32"] = multirhs_form(h, celgpu, torch, stream)
        forms["differentiation_128_b8"] = differentiation_form(h, celgpu, torch, stream)
        forms["plain_large_256"] = plain_large_form(h, celgpu, torch, stream, m, b, x, iters)

    # ---- the distributed row-block solve of the same system over all ranks ----
    if not args.quick:
        dist_key = "distributed_256" if world > 1 else "distributed_world1_256"
        forms[dist_key] = distributed_form(h, celgpu, torch, stream, rp, ci, v, b.cpu().numpy(),
                                           rank, world, local, max_over_ranks, barrier)

    # ---- e2e through the ELM interface with host buffers ----
    h.elm_init(n, n, 1, (7, 0))
    h.elm_insert_rows(1, rp + 1, ci + 1, v)
    h.elm_set_solver(celgpu.SOLVER_PCG, p, diag_scaling=False)
    h.elm_matrix_completed()
    b_host = b.cpu().pin_memory()
    x_host = torch.empty(n, dtype=torch.float64).pin_memory()
    bh, xh = b_host.numpy(), x_host.numpy()
    for _ in range(max(1, min(args.warmup, 2))):
        h.elm_doit(bh)
        h.elm_collect_solution(n, xh)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        ierr, niter, ftol = h.elm_doit(bh)
        h.elm_collect_solution(n, xh)
    e1.record(stream)
    torch.cuda.synchronize()
    wall_e2e = time.perf_counter() - t0
    e2e_ms = max_over_ranks(e0.elapsed_time(e1))
    h.elm_destroy()
    assert ierr == 0, ierr

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        perm_gpu = forms.get("plain_large_256", {}).pop("jad_perm", None)
        cpu, parity = cpu_baseline_and_parity(h, celgpu, torch, m, rp, ci, v, x_true, b, p,
                                              perm_gpu)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": "poisson7_256^3_pcg_jacobi_csr_fp64", "rows": n, "nnz": nnz,
                   "rel_res": EPS_REL, "x0": "zero", "rhs": "A*x_true, x_true~U[0,1) seed 1",
                   "iterations": iters, "verified_relres": last.verified_relres,
                   "l2": "inputs 1.9 GB resident, > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "pcg": {"ms_per_iteration": ms_per_step / max(iters, 1),
                "bytes_per_iteration": pcg_bytes,
                "achieved_gbs": pcg_bytes * iters / (ms_per_step / 1e3) / 1e9,
                "frac_of_peak": pcg_bytes * iters / (ms_per_step / 1e3) / 1e9 / peak},
        "roofline": {"kernel": "csr_tma_kernel<double, EpiStore> (SpMV 256^3)", "bound": "hbm",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": f"{peak_kind} hbm_gbs (copy, burst)",
                     "bytes_per_launch": spmv_bytes, "ms_per_launch": spmv_ms,
                     "traffic": traffic, "traffic_source": traffic_src},
        "e2e": {"value": world * args.steps / (e2e_ms / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                "api": "celg_elm_doit + celg_elm_collect_solution (pinned host b/x)",
                "wall_s": wall_e2e},
        "forms": forms,
        # one solve: 2 set-up sweeps, 3 per iteration and 1 verification; the
        # graph's loop body holds two iterations (an odd count ends with one
        # body of 3 kernels that return at once); every rank runs its own
        # replica of the solve, so the whole job launches world times that
        "gpu_launches": world * args.steps * (3 + 3 * (iters + iters % 2)),
        "clocks": clk,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    # last on the line, so that a reader of only its tail sees them
    line["summary"] = {"forms": forms_summary(forms, value), "parity": parity}
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.destroy()
    h.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_profile(argv):
    """--profile WHAT SIDE ...: one workload of the library for a kernel profiler
    (ncu), with no timing of its own.

      spmv SIDE [REPS]          REPS CSR SpMVs, SIDE^3 Poisson
      jad SIDE [REPS]           REPS JAD SpMVs of the same system
      gmres SIDE [M]            one GMRES(M)-Jacobi solve to 1e-8
      spmv32 SIDE [REPS]        the same on the FP32 copy (1-byte columns)
      pcg SIDE ITERS [fp64|ru|ir]
                                one solve capped at ITERS iterations
      mrhs SIDE ITERS K [fp64|ir|ru]
                                K right-hand sides, capped at ITERS (ir: one
                                outer step of FP32 refinement, ITERS inner;
                                ru: FP32 with reliable updates)
      batch 0 ITERS             the 64 uneven systems, capped at ITERS

    Set CELG_GRAPH=0 to launch the solver kernels from a host loop instead of
    one CUDA graph, so that a kernel profiler can attribute time to each
    kernel."""
    import torch

    from cel_v3_b200 import celgpu, synth
    what, side = argv[0], int(argv[1])
    if what == "batch":
        h = celgpu.Handle(0, torch.cuda.current_stream().cuda_stream)
        probs = synth.batch_problems()
        mats = [h.matrix_from_csr(rp, ci, v).jacobi() for _, rp, ci, v, _ in probs]
        bs = [torch.from_numpy(b).cuda() for *_, b in probs]
        xs = [torch.zeros_like(b) for b in bs]
        infos = h.pcg_batched(mats, [b.data_ptr() for b in bs], [x.data_ptr() for x in xs],
                              eps_rel=1e-8, iter_max=int(argv[2]))
        torch.cuda.synchronize()
        print("batch", len(mats), max(i.iter_done for i in infos))
        h.close()
        return 0
    rp, ci, v, xt = synth.plain(side, 1)
    n = rp.size - 1
    h = celgpu.Handle(0, torch.cuda.current_stream().cuda_stream)
    m = h.matrix_from_csr(rp, ci, v).jacobi()
    x = torch.from_numpy(xt).cuda()
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    if what == "spmv32":
        m.make_fp32()
        x32, y32 = x.float(), y.float()
        for _ in range(int(argv[2]) if len(argv) > 2 else 4):
            h.spmv_f32(m, x32.data_ptr(), y32.data_ptr())
        torch.cuda.synchronize()
        print("spmv32", side, float(y32.sum()))
    elif what == "spmv":
        for _ in range(int(argv[2]) if len(argv) > 2 else 4):
            h.spmv(m, x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        print("spmv", side, float(y.sum()))
    elif what == "jad":
        m.to_jad()
        for _ in range(int(argv[2]) if len(argv) > 2 else 4):
            h.spmv(m, x.data_ptr(), y.data_ptr(), fmt=celgpu.FMT_JAD)
        torch.cuda.synchronize()
        print("jad", side, float(y.sum()))
    elif what == "gmres":
        restart = int(argv[2]) if len(argv) > 2 else 30
        h.spmv(m, x.data_ptr(), y.data_ptr())  # b = A x_true
        xs = torch.zeros_like(y)
        info = h.gmres_jacobi(m, y.data_ptr(), xs.data_ptr(), restart=restart, eps_rel=1e-8,
                              iter_max=2000, x0_mode=celgpu.X0_ZERO)
        torch.cuda.synchronize()
        print("gmres", side, restart, info.arnoldi_steps, info.status)
    elif what == "pcg":
        iters = int(argv[2])
        mode = argv[3] if len(argv) > 3 else "fp64"
        h.spmv(m, x.data_ptr(), y.data_ptr())  # b = A x_true
        xs = torch.zeros_like(y)
        prec = {"fp64": celgpu.PREC_FP64, "ru": celgpu.PREC_FP32_RU,
                "ir": celgpu.PREC_FP32_IR}[mode]
        kw = dict(inner_iter_max=iters, outer_max=1) if mode == "ir" else {}
        info = h.pcg_jacobi(m, y.data_ptr(), xs.data_ptr(), precision=prec, eps_rel=1e-12,
                            iter_max=iters, **kw)
        torch.cuda.synchronize()
        print("pcg", side, mode, info.iter_done, info.status)
    elif what == "mrhs":
        iters, k = int(argv[2]), int(argv[3])
        mode = argv[4] if len(argv) > 4 else "fp64"
        kw = {"ir": dict(precision=celgpu.PREC_FP32_IR, inner_iter_max=iters, outer_max=1),
              "ru": dict(precision=celgpu.PREC_FP32_RU)}.get(mode, {})
        B = torch.rand((n, k), dtype=torch.float64, device="cuda")
        X = torch.zeros_like(B)
        infos = h.pcg_multirhs(m, k, B.data_ptr(), X.data_ptr(), eps_rel=1e-12, iter_max=iters,
                               **kw)
        torch.cuda.synchronize()
        print("mrhs", side, k, max(i.iter_done for i in infos))
    else:
        raise SystemExit(run_profile.__doc__)
    h.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip the extra precision forms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--profile", nargs="+", metavar="ARG",
                    help="run one workload for a kernel profiler (WHAT SIDE ...), no timing")
    args = ap.parse_args()
    if args.profile:
        return run_profile(args.profile)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
