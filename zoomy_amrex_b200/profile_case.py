"""A fixed, small run of each hot path, for profilers (ncu) and quick checks.

    python -m zoomy_amrex_b200.profile_case fp32    [--n 3072] [--variant V] [--steps 3]
    python -m zoomy_amrex_b200.profile_case fp64    [--n 3072] [--steps 3]
    python -m zoomy_amrex_b200.profile_case adjoint [--n 512]  [--steps 20] [--variant V]

Each runs the benchmark's wet/dry bump level (``workloads.bump_workload_*``)
on an n x n grid: the FP32 form as a batch of one with the given strip shape,
the FP64 form through a Level, or the forward + backward of the FP64 adjoint
with checkpoints every 20 steps. The launches are the product's own; a
profiler selects them by kernel name (k32b_stage, k_stage, k_adj_face, ...).
"""
from __future__ import annotations

import argparse


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("form", choices=["fp32", "fp64", "adjoint"])
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--variant", type=int, default=None)
    a = ap.parse_args(argv)

    import torch
    from ._abi import ZFV_PREC_FP32
    from .workloads import bump_workload_config, bump_workload_fields

    if a.form == "fp32":
        from .batch import Batch
        n, steps = a.n or 3072, a.steps or 3
        Q0, A0 = bump_workload_fields(n)
        cfg = bump_workload_config(n)
        cfg.precision = ZFV_PREC_FP32
        b = Batch([cfg], [Q0], [A0], variant=a.variant if a.variant is not None else 0)
        b.begin()
        b.evolve(steps)
        b.sync()
        st = b.status()[0]
        b.close()
    elif a.form == "fp64":
        from .level import Level
        n, steps = a.n or 3072, a.steps or 3
        Q0, A0 = bump_workload_fields(n)
        lev = Level(bump_workload_config(n), Q0, A0)
        lev.begin()
        lev.evolve(steps)
        st = lev.status()
        lev.close()
    else:
        from . import _lib
        from .adjoint import evolve_differentiable
        n, steps = a.n or 512, a.steps or 20
        if a.variant is not None:
            _lib.check(_lib.lib().zfv_adj_set_variant(a.variant), "zfv_adj_set_variant")
        Q0, A0 = bump_workload_fields(n)
        q = torch.from_numpy(Q0).cuda().requires_grad_(True)
        nm = torch.tensor(0.03, dtype=torch.float64, device="cuda", requires_grad=True)
        QT = evolve_differentiable(q, nm, torch.from_numpy(A0).cuda(), bump_workload_config(n), steps)
        loss = 0.5 * ((QT[0] + QT[1] - 1.0) ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        st = {"step": steps, "loss": float(loss), "dL/dn_m": float(nm.grad)}
    if st["step"] != steps:
        raise SystemExit(f"ran {st['step']} of {steps} steps")
    print(a.form, st)


if __name__ == "__main__":
    main()
