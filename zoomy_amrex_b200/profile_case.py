"""A fixed, small run of each hot path, for profilers (ncu) and quick checks.

    python -m zoomy_amrex_b200.profile_case fp32    [--n 3072] [--variant V] [--steps 3]
    python -m zoomy_amrex_b200.profile_case fp64    [--n 3072] [--steps 3]
    python -m zoomy_amrex_b200.profile_case adjoint [--n 512]  [--steps 20] [--variant V]
    python -m zoomy_amrex_b200.profile_case amr     [--n 1024] [--steps 4]  [--variant V]
    python -m zoomy_amrex_b200.profile_case sme64   [--n 1024] [--steps 3]
    python -m zoomy_amrex_b200.profile_case sme32   [--n 1024] [--steps 3]  [--variant V]

Each runs the benchmark's wet/dry bump level (``workloads.bump_workload_*``)
on an n x n grid: the FP32 form as a batch of one with the given strip shape,
the FP64 form through a Level, or the forward + backward of the FP64 adjoint
with checkpoints every 20 steps, or (amr) the 3-level AMR hierarchy of a dam
break over bumps on an n x n base grid (boxes 64^2, one CUDA graph per coarse
step), or (sme64 / sme32) the shallow-moment level-2 benchmark level
(``workloads.sme_workload_*``) on n x n in the FP64 plain form or the FP32
chosen form (tile shape V). The launches are the product's own; a
profiler selects them by kernel name (k32b_stage, k_stage, k_adj_face, ...).
"""
from __future__ import annotations

import argparse


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("form", choices=["fp32", "fp64", "adjoint", "amr", "sme64", "sme32"])
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
    elif a.form in ("sme64", "sme32"):
        from .level import Level
        from .workloads import sme_workload_config, sme_workload_fields
        n, steps = a.n or 1024, a.steps or 3
        Q0, A0 = sme_workload_fields(n)
        cfg = sme_workload_config(n)
        if a.form == "sme32":
            cfg.precision = ZFV_PREC_FP32
        lev = Level(cfg, Q0, A0, variant=a.variant if a.form == "sme32" else None)
        lev.begin()
        lev.evolve(steps)
        st = lev.status()
        lev.close()
    elif a.form == "amr":
        from .amr import AmrHierarchy
        from .workloads import dam_break_level
        n, steps = a.n or 1024, a.steps or 4
        cfg, Q0 = dam_break_level(n)
        hier = AmrHierarchy(cfg, Q0, max_level=2, B=64, threshold=0.01, regrid_int=2,
                            variant=a.variant if a.variant is not None else 9)
        hier.run(steps)
        st = {"step": hier.steps, "boxes": [lv.n for lv in hier.levels], "time": hier.time}
        hier.close()
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
