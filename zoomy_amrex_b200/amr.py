"""Block-structured AMR hierarchy of the FP32 shallow-water form.

The reference's AmrCore driver (ZoomyAmr.cpp:161-288, 733-762): a base level
plus up to ``max_level`` refined levels (ratio 2), tagging by an eta-gradient
threshold or by the reference's ErrorEst criterion (``tag="reference"``:
undivided |grad h| > threshold or h > 1e-2, below ``tag_b_max``), regridding,
per-stage ghost filling from the same level
or the coarser one (FillPatch / FillPatchTwoLevels with conservative linear
interpolation), subcycling (a level-l step is followed by two level-(l+1)
steps), and averaging the fine solution down onto the coarse level after them.
There is no flux register, as in the reference (ZoomyAmr.H:85).

Here every level is refined in B x B blocks on a regular block grid (the
layout of a quadtree rather than AMReX's Berger-Rigoutsos clustering); the
blocks of a level are grouped into patches, rectangles of up to
``patch_blocks`` x ``patch_blocks`` blocks, each one instance of a grouped batch:
one launch per RK stage advances all patches of a level, the patches of a
level share one run record, and a patch's ghost ring is a small frame array
the stage kernels read in place of the physical mirror.

The step law is a choice (``dt_mode``): "aligned" (the default) steps level
l with dt_0 / 2^l, dt_0 the largest step every level's CFL law allows, so the
levels stay time-aligned; "level" is the reference's law (ZoomyAmr.cpp:739-749):
before each of its steps a level takes its own CFL dt from its current
state (level 0 clamped to land on time_end), so a fine level's two substeps
need not add up to the coarse step. Regridding happens every ``regrid_int``
coarse steps (the reference regrids at every coarse step).
"""
from __future__ import annotations

import ctypes as C
import numpy as np
import torch

from . import _lib
from ._abi import ZFV_PREC_FP32, zfv_amr_level, zfv_config
from .batch import Batch


def _cfg_copy(c: zfv_config) -> zfv_config:
    d = zfv_config()
    C.memmove(C.byref(d), C.byref(c), C.sizeof(c))
    return d


def group_patches(blocks, max_side: int) -> list[tuple[int, int, int, int]]:
    """Blocks (bx, by) -> patches (bx0, by0, nbx, nby): rectangles made of
    runs of consecutive blocks of a block row (at most ``max_side`` long),
    stacked while the run below starts and ends in the same columns (at most
    ``max_side`` runs high)."""
    runs = []
    for bx, by in sorted(blocks, key=lambda p: (p[1], p[0])):
        if runs and runs[-1][1] == by and runs[-1][0] + runs[-1][2] == bx and runs[-1][2] < max_side:
            runs[-1] = (runs[-1][0], by, runs[-1][2] + 1)
        else:
            runs.append((bx, by, 1))
    rects, open_ = [], {}
    for bx0, by, nb in runs:
        r = open_.get((bx0, nb))
        if r is not None and rects[r][1] + rects[r][3] == by and rects[r][3] < max_side:
            rects[r] = (bx0, rects[r][1], nb, rects[r][3] + 1)
        else:
            rects.append((bx0, by, nb, 1))
            r = len(rects) - 1
        open_[(bx0, nb)] = r
    return sorted(rects, key=lambda p: (p[1], p[0]))


class AmrLevel:
    """All blocks of one level: a grouped batch of patches (horizontal runs
    of blocks), their block map and ghost frames."""

    def __init__(self, hier, lev: int, blocks: list[tuple[int, int]], Q0=None, variant=None):
        self.h, self.lev = hier, lev
        B = hier.B
        self.B = B
        self.nbx, self.nby = hier.nbx0 << lev, hier.nby0 << lev
        self.nx, self.ny = self.nbx * B, self.nby * B
        self.dx = hier.dx0 / (1 << lev)
        self.dy = hier.dy0 / (1 << lev)
        self.blocks = sorted(blocks, key=lambda p: (p[1], p[0]))
        self.patches = group_patches(self.blocks, hier.patch_blocks)
        self.max_blocks = max(nbx * nby for _, _, nbx, nby in self.patches)
        dev = hier.device
        cfgs, Q0s = [], None if Q0 is None else []
        for (bx, by, nbx, nby) in self.patches:
            c = _cfg_copy(hier.cfg)
            c.nx, c.ny = nbx * B, nby * B
            c.prob_lo[0] = hier.lo[0] + bx * B * self.dx
            c.prob_lo[1] = hier.lo[1] + by * B * self.dy
            c.prob_hi[0] = c.prob_lo[0] + nbx * B * self.dx
            c.prob_hi[1] = c.prob_lo[1] + nby * B * self.dy
            c.precision = ZFV_PREC_FP32
            c.time_end = 1.0e30
            c.max_step = -1
            cfgs.append(c)
            if Q0 is not None:
                Q0s.append(np.ascontiguousarray(Q0[:, by * B:(by + nby) * B, bx * B:(bx + nbx) * B]))
        self.batch = Batch(cfgs, Q0s, None, device=dev, stream=hier.stream, groups=[0] * len(cfgs),
                           variant=hier.variant if variant is None else variant)
        n = len(self.patches)
        self.frames = [torch.zeros((4, nby * B + 4, nbx * B + 4), dtype=torch.float32, device=dev)
                       for (_, _, nbx, nby) in self.patches]
        self.batch.set_frames(self.frames)
        m = torch.full((self.nby, self.nbx), -1, dtype=torch.int32)
        for k, (bx, by, nbx, nby) in enumerate(self.patches):
            for oy in range(nby):
                for ox in range(nbx):
                    m[by + oy, bx + ox] = (k << 10) | (oy << 5) | ox
        self.map = m.to(dev)
        self.pdesc = torch.tensor([list(p) for p in self.patches], dtype=torch.int32,
                                  device=dev).reshape(n, 4).contiguous()
        self.frame_ptrs = torch.tensor([f.data_ptr() for f in self.frames], dtype=torch.int64, device=dev)
        self.dts = torch.zeros(n, dtype=torch.float64, device=dev)
        self.view = zfv_amr_level(C.c_void_p(self.batch.descriptors), C.c_void_p(self.map.data_ptr()),
                                  self.nbx, self.nby, B, self.nx, self.ny, hier.wall, 0)

    @property
    def n(self) -> int:
        """Blocks of the level."""
        return len(self.blocks)

    @property
    def n_patches(self) -> int:
        return len(self.patches)

    def close(self):
        self.batch.close()


class AmrHierarchy:
    """A ``max_level``-deep hierarchy over a base grid of ``nx0 x ny0`` cells.

    cfg: an SWE2D configuration of the base grid (scheme switches, CFL
    constants, parameters, boundary tags; nx/ny multiples of ``B``). Q0: the
    base level's FP64 state [b, h, hu, hv]. Finer levels start as
    interpolations of the coarser one, refined where tagged (a negative
    ``threshold`` refines everywhere the nesting allows).
    """

    TAGS = {"eta_gradient": 0, "reference": 1}

    def __init__(self, cfg: zfv_config, Q0, max_level: int = 2, B: int = 64, threshold: float = 0.01,
                 regrid_int: int = 2, device="cuda:0", variant: int = 9, patch_blocks: int = 16,
                 tag: str = "eta_gradient", tag_b_max: float = 1.0e30, dt_mode: str = "aligned"):
        if cfg.nx % B or cfg.ny % B or B % 2:
            raise ValueError("the base grid must be a multiple of the (even) box side B in both directions")
        self.cfg = _cfg_copy(cfg)
        self.B, self.max_level, self.threshold, self.regrid_int = B, max_level, threshold, regrid_int
        self.device = torch.device(device)
        self.stream = torch.cuda.Stream(self.device)
        self.variant = variant
        if not 1 <= patch_blocks <= 32:
            raise ValueError("patch_blocks must be in 1 .. 32")
        if tag not in self.TAGS:
            raise ValueError(f"tag must be one of {sorted(self.TAGS)}")
        if dt_mode not in ("aligned", "level"):
            raise ValueError("dt_mode must be 'aligned' or 'level'")
        self.dt_mode = dt_mode
        self.criterion, self.tag_b_max = self.TAGS[tag], float(tag_b_max)
        self.patch_blocks = patch_blocks
        self.nbx0, self.nby0 = cfg.nx // B, cfg.ny // B
        self.lo = (cfg.prob_lo[0], cfg.prob_lo[1])
        self.dx0 = (cfg.prob_hi[0] - cfg.prob_lo[0]) / cfg.nx
        self.dy0 = (cfg.prob_hi[1] - cfg.prob_lo[1]) / cfg.ny
        self.wall = sum(1 << s for s in range(4) if cfg.bc_tag[s] == 1)
        self.div = float(cfg.cfl_dimension * cfg.cfl_degree_factor)
        self.steps = 0
        self.use_graph = True
        self._graph = None
        self._time = torch.zeros(1, dtype=torch.float64, device=self.device)
        Q0 = np.asarray(Q0, dtype=np.float64)
        blocks = [(bx, by) for by in range(self.nby0) for bx in range(self.nbx0)]
        self.levels: list[AmrLevel] = [AmrLevel(self, 0, blocks, Q0)]
        self.levels[0].batch.begin()
        for _ in range(max_level):          # initial hierarchy (InitData's repeated regrid)
            if not self.regrid():
                break
        self.sync()

    # -- small helpers -------------------------------------------------------------
    def _s(self):
        return C.c_void_p(self.stream.cuda_stream)

    def sync(self):
        self.stream.synchronize()

    def _coarse_view(self, lev):
        return C.byref(self.levels[lev - 1].view) if lev > 0 else None

    def fill(self, lev: int, stage: int):
        L = self.levels[lev]
        _lib.check(_lib.lib().zfv_amr_fill(C.byref(L.view), self._coarse_view(lev), L.pdesc.data_ptr(),
                                           L.frame_ptrs.data_ptr(), L.n_patches, L.max_blocks, stage, self._s()),
                   "zfv_amr_fill")

    def average_down(self, lev: int):
        F, Cl = self.levels[lev], self.levels[lev - 1]
        _lib.check(_lib.lib().zfv_amr_average_down(C.byref(F.view), C.byref(Cl.view), F.pdesc.data_ptr(),
                                                   F.n_patches, F.max_blocks, self._s()), "zfv_amr_average_down")

    # -- regridding ------------------------------------------------------------------
    def tags(self, lev: int) -> np.ndarray:
        """Tagged blocks of level ``lev`` as a boolean (nby, nbx) array."""
        L = self.levels[lev]
        with torch.cuda.stream(self.stream):
            flags = torch.zeros((L.nby, L.nbx), dtype=torch.int32, device=self.device)
            _lib.check(_lib.lib().zfv_amr_tag(C.byref(L.view), L.pdesc.data_ptr(), L.n_patches, L.max_blocks,
                                              L.dx, L.dy, self.threshold, self.criterion, self.tag_b_max,
                                              flags.data_ptr(), self._s()), "zfv_amr_tag")
        self.sync()
        return flags.cpu().numpy() != 0

    def _refined_blocks(self, lev: int) -> list[tuple[int, int]]:
        """Level-(lev+1) blocks: children of tagged level-lev blocks and their
        neighbours, restricted to level-lev blocks whose 8 neighbours exist at
        level lev (or lie outside the domain), so that every ghost cell and
        every interpolation stencil of the new level has coarse data."""
        L = self.levels[lev]
        have = np.zeros((L.nby, L.nbx), dtype=bool)
        for bx, by in L.blocks:
            have[by, bx] = True
        if self.threshold < 0:            # refine everything the nesting allows
            tagged = have.copy()
        else:
            tagged = self.tags(lev) & have
        want = tagged.copy()
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                want |= np.roll(np.roll(tagged, dy, 0), dx, 1) & self._in_domain_shift(tagged.shape, dy, dx)
        ok = have.copy()
        padded = np.pad(have, 1, constant_values=True)       # outside the domain counts as present
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok &= padded[1 + dy:1 + dy + L.nby, 1 + dx:1 + dx + L.nbx]
        sel = want & ok
        out = []
        for by, bx in zip(*np.nonzero(sel)):
            for cy in (0, 1):
                for cx in (0, 1):
                    out.append((2 * int(bx) + cx, 2 * int(by) + cy))
        return sorted(out, key=lambda p: (p[1], p[0]))

    @staticmethod
    def _in_domain_shift(shape, dy, dx):
        m = np.ones(shape, dtype=bool)
        if dy > 0:
            m[:dy, :] = False
        elif dy < 0:
            m[dy:, :] = False
        if dx > 0:
            m[:, :dx] = False
        elif dx < 0:
            m[:, dx:] = False
        return m

    def regrid(self) -> bool:
        """Rebuild levels 1..max_level from the tags, top down. Returns whether
        the finest level count or any box set changed."""
        changed = False
        for lev in range(self.max_level):
            if lev >= len(self.levels):
                break
            blocks = self._refined_blocks(lev)
            old = self.levels[lev + 1] if lev + 1 < len(self.levels) else None
            if old is not None and blocks == old.blocks:
                continue
            changed = True
            if not blocks:
                for L in self.levels[lev + 1:]:
                    L.close()
                del self.levels[lev + 1:]
                break
            new = AmrLevel(self, lev + 1, blocks)
            ov = C.byref(old.view) if old is not None else None
            with torch.cuda.stream(self.stream):
                _lib.check(_lib.lib().zfv_amr_regrid_fill(C.byref(new.view), ov, C.byref(self.levels[lev].view),
                                                          new.pdesc.data_ptr(), new.n_patches, new.max_blocks,
                                                          self._s()), "zfv_amr_regrid_fill")
            new.batch.begin()
            self.sync()
            if old is not None:
                old.close()
                self.levels[lev + 1] = new
            else:
                self.levels.append(new)
        return changed

    # -- time stepping -----------------------------------------------------------------
    def _set_dt(self):
        """dt_0 from every level's last CFL maximum, on the device (zfv_amr_set_dt)."""
        n = len(self.levels)
        descs = (C.c_void_p * n)(*[L.batch.descriptors for L in self.levels])
        dts = (C.c_void_p * n)(*[L.dts.data_ptr() for L in self.levels])
        cnt = (C.c_int * n)(*[L.n_patches for L in self.levels])
        c = self.cfg
        _lib.check(_lib.lib().zfv_amr_set_dt(descs, dts, cnt, n, c.cfl, self.div, c.dtmin, c.dtmax, c.time_end,
                                             self._time.data_ptr(), self._s()), "zfv_amr_set_dt")

    def _advance(self, lev: int):
        L = self.levels[lev]
        if self.dt_mode == "level":
            L.batch.compute_dt()
            if lev == 0:
                _lib.check(_lib.lib().zfv_amr_level_dt(C.c_void_p(L.batch.descriptors), self.cfg.time_end,
                                                       self._time.data_ptr(), self._s()), "zfv_amr_level_dt")
        else:
            L.batch.set_dt(L.dts)
        self.fill(lev, 1)
        L.batch.stage(1)
        self.fill(lev, 2)
        L.batch.stage(2)

    def _time_step(self, lev: int):
        self._advance(lev)
        if lev + 1 < len(self.levels):
            for _ in range(2):
                self._time_step(lev + 1)
            self.average_down(lev + 1)

    def _coarse_step(self):
        if self.dt_mode == "aligned":
            self._set_dt()
        self._time_step(0)

    def step(self):
        """One coarse step of the whole hierarchy (ZoomyAmr::TimeStep's
        recursion), replayed from a CUDA graph captured after each regrid."""
        if self.steps > 0 and self.regrid_int > 0 and self.steps % self.regrid_int == 0 and self.max_level > 0:
            if self.regrid():
                self._graph = None
        if self.use_graph:
            if self._graph is None:
                self.sync()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.stream(self.stream):
                    with torch.cuda.graph(g, stream=self.stream):
                        self._coarse_step()
                self._graph = g
            with torch.cuda.stream(self.stream):
                self._graph.replay()
        else:
            self._coarse_step()
        self.steps += 1

    @property
    def time(self) -> float:
        self.sync()
        return float(self._time.item())

    def run(self, n_steps: int):
        for _ in range(n_steps):
            self.step()
        self.sync()

    def evolve(self, check_every: int = 16) -> int:
        """Coarse steps until the configuration's time_end (the last dt_0 lands
        on it) or max_step, like ZoomyAmr::Evolve; returns the steps taken.
        The time is read every ``check_every`` steps; steps past time_end have
        dt_0 = 0 and change nothing."""
        c = self.cfg
        while (c.max_step < 0 or self.steps < c.max_step) and self.time < c.time_end:
            n = check_every if c.max_step < 0 else min(check_every, c.max_step - self.steps)
            self.run(n)
        return self.steps

    # -- output ----------------------------------------------------------------------------
    def cells_per_coarse_step(self) -> int:
        """Cell updates of one coarse step: level l's cells times its 2^l substeps."""
        return sum(L.n * self.B * self.B * (1 << L.lev) for L in self.levels)

    def level_state(self, lev: int) -> np.ndarray:
        """Level ``lev`` as a dense (4, ny, nx) FP64 array [b, h, hu, hv]; NaN where no box."""
        L = self.levels[lev]
        B = self.B
        out = np.full((4, L.ny, L.nx), np.nan)
        for (bx, by, nbx, nby), q in zip(L.patches, L.batch.state64()):
            out[:, by * B:(by + nby) * B, bx * B:(bx + nbx) * B] = q.cpu().numpy()
        return out

    def write_plotfile(self, out_dir, identifier: str = "", step: int | None = None) -> str:
        """All levels as one AMReX plotfile, as ZoomyAmr::WritePlotFile does
        (ZoomyAmr.cpp:821-882): per level its patches (boxes) with components
        var0..var3 (b, h, hu, hv) then aux0..aux6, ref ratio 2, level l's step
        count = coarse steps x 2^l. Returns the plotfile's path."""
        import os
        from .plotfile import LevelData, PatchData, component_names, plotfile_name, write_plotfile
        step = self.steps if step is None else int(step)
        B = self.B
        levels = []
        for L in self.levels:
            qs = L.batch.state64()                       # also refreshes the aux hinv row
            patches = [PatchData(np.concatenate([q.cpu().numpy(), a.cpu().numpy()], axis=0), (bx * B, by * B))
                       for (bx, by, _, _), q, a in zip(L.patches, qs, L.batch.aux)]
            levels.append(LevelData((0, 0), (L.nx - 1, L.ny - 1), (L.dx, L.dy), patches,
                                    step=self.steps << L.lev))
        c = self.cfg
        n_aux = self.levels[0].batch.aux[0].shape[0]
        path = os.path.join(str(out_dir), plotfile_name(identifier, step))
        return write_plotfile(path, levels, component_names(4, n_aux), self.time,
                              (c.prob_lo[0], c.prob_lo[1]), (c.prob_hi[0], c.prob_hi[1]),
                              [2] * (len(levels) - 1))

    def mass(self) -> float:
        """Sum of h dx dy over the base level (finer levels are averaged onto it)."""
        q = self.level_state(0)
        return float(q[1].sum() * self.dx0 * self.dy0)

    def close(self):
        self._graph = None
        for L in self.levels:
            L.close()
        self.levels = []
