"""Runs one workload of the library for profiling (e.g. under ncu).

  python -m cel_v3_b200.drive spmv SIDE [REPS]          REPS CSR SpMVs, SIDE^3 Poisson
  python -m cel_v3_b200.drive spmv32 SIDE [REPS]        the same on the FP32 copy (1-byte columns)
  python -m cel_v3_b200.drive pcg SIDE ITERS [fp64|ru|ir]
                                                        one solve capped at ITERS iterations
  python -m cel_v3_b200.drive mrhs SIDE ITERS K         K right-hand sides, capped at ITERS
  python -m cel_v3_b200.drive batch 0 ITERS             the 64 uneven systems, capped at ITERS

Set CELG_GRAPH=0 to launch the solver kernels from a host loop instead of
one CUDA graph, so that a kernel profiler can attribute time to each kernel.
"""
import sys

import numpy as np


def main(argv):
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
        B = torch.rand((n, k), dtype=torch.float64, device="cuda")
        X = torch.zeros_like(B)
        infos = h.pcg_multirhs(m, k, B.data_ptr(), X.data_ptr(), eps_rel=1e-12, iter_max=iters)
        torch.cuda.synchronize()
        print("mrhs", side, k, max(i.iter_done for i in infos))
    else:
        raise SystemExit(__doc__)
    h.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
