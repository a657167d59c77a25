"""Launch-shape autotuner of the batched engine.

The engine advances each box with one thread-block cluster. Two shape
parameters decide how a batch maps onto the GPU:

- the cluster size: CTAs per box, which split the framework and the wave
  vectors between them;
- the CTA size: warps per CTA, which split the trial positions and
  framework chunks of one energy evaluation.

- the CTAs per SM (1, 2 or 4): CTAs of different boxes sharing an SM fill
  each other's barrier waits, with smaller CTAs and less shared memory each.

The best shape depends on the number of boxes against the SM count, on the
framework sizes and on the loadings. Measured on a B200 for 64 CO2 boxes of
512-4096 atoms, cluster x threads gave 0.22-1.48 M moves/s.

When the best shape leaves SMs idle (64 boxes at 2 CTAs each fill 128 of
148), the costliest boxes, by the clock cycles they spent in the best run,
can run in a second launch at a larger cluster size (one or two times
more CTAs) beside the first (`Engine.set_split`); the tuner times such
splits too.

`tune()` times every admissible shape on copies of the caller's boxes (same
force fields, configurations and random seeds), so the caller's state does
not move, and returns the fastest. Results are cached per batch signature
for the life of the process.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import native

_CACHE: Dict[tuple, "Shape"] = {}


@dataclasses.dataclass
class Shape:
    cluster: int
    threads: int
    moves_per_s: float
    table: List[dict]
    split: Tuple[int, ...] = ()     # boxes run in a second launch
    cluster_b: int = 0              # its cluster size
    ctas_per_sm: int = 1

    def apply(self, eng: "native.Engine") -> None:
        """Sets the split of this shape on an engine built with its cluster
        and threads."""
        if self.split:
            eng.set_split(self.split, self.cluster_b)

    def engine(self, systems: Sequence["native.GpuSystem"], precision: int) -> "native.Engine":
        """An engine of `systems` with this shape."""
        eng = native.Engine(systems, precision=precision, threads=self.threads, cluster=self.cluster,
                            ctas_per_sm=self.ctas_per_sm)
        self.apply(eng)
        return eng

    def describe(self) -> dict:
        return {"cluster": self.cluster, "threads": self.threads, "ctas_per_sm": self.ctas_per_sm,
                "split": {"systems": len(self.split), "cluster": self.cluster_b}}


def _signature(systems: Sequence["native.GpuSystem"], precision: int, ordered: bool = False) -> tuple:
    """Key of a batch: its boxes' sizes, sorted (in order when `ordered`,
    for shapes that name boxes by index)."""
    sig = []
    for g in systems:
        fw = g.sysm.framework()[0]
        sig.append((len(fw), g.natom, tuple(g.sysm.kmax), g.maxmol, bool(getattr(g, "grids_active", False))))
    return (precision, tuple(sig) if ordered else tuple(sorted(sig)))


def candidates(nsys: int, precision: int, sms: int) -> List[Tuple[int, int, int]]:
    """Shapes (cluster, threads, CTAs per SM) worth timing. A shape whose
    CTAs do not all fit the SMs at once runs in waves and is skipped; several
    CTAs per SM need the 64-register build (mixed precision) and at most
    1024 threads per SM between them."""
    mixed = precision != native.RGPU_FP64
    threads = (256, 512, 1024) if mixed else (128, 256, 512)
    out = []
    for c in (1, 2, 4, 8):
        if nsys * c > sms and c > 1:
            continue
        for t in threads:
            out.append((c, t, 1))
    if mixed:
        for occ in (2, 4):
            for c in (2, 4, 8):
                if nsys * c > sms * occ or nsys * c <= sms:
                    continue
                for t in (256, 512):
                    if t * occ <= 1024:
                        out.append((c, t, occ))
    return out


def _clone(g: "native.GpuSystem", xyz: np.ndarray) -> "native.GpuSystem":
    c = native.GpuSystem(g.sysm, **g.init_args)
    if getattr(g, "grids_active", False):
        c.share_grids_of(g)
    c.set_adsorbates(xyz)
    return c


def tune(systems: Sequence["native.GpuSystem"], precision: int = native.RGPU_MIXED, moves: int = 400,
         warm: int = 100, shapes: Optional[Sequence[Tuple[int, int]]] = None, use_cache: bool = True,
         split: bool = True) -> Shape:
    """Times each candidate shape on copies of `systems` and returns the
    fastest as a Shape (with the full table of measurements). With `split`,
    and when the candidates are the default ones, splits of the best shape
    that fill the idle SMs are timed as well."""
    import torch

    key = (_signature(systems, precision, ordered=split), split)
    if use_cache and shapes is None and key in _CACHE:
        return _CACHE[key]
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    auto_split = split and shapes is None
    shapes = list(shapes) if shapes is not None else candidates(len(systems), precision, props.multi_processor_count)
    start = [g.adsorbates() for g in systems]
    clones = [_clone(g, x) for g, x in zip(systems, start)]
    stream = torch.cuda.Stream()
    table = []
    best = None

    def time_shape(c, t, split=(), cb=0, occ=1):
        """moves/s of one shape and each box's clock cycles in the timed run"""
        for g, x in zip(clones, start):
            g.set_adsorbates(x)
        eng = native.Engine(clones, precision=precision, threads=t, cluster=c, ctas_per_sm=occ)
        try:
            if split:
                eng.set_split(split, cb)
            eng.run(warm, stream.cuda_stream)
            torch.cuda.synchronize()
            c0 = [g.state()["counters"] for g in clones]
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            eng.run(moves, stream.cuda_stream)
            ev1.record(stream)
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1)
            c1 = [g.state()["counters"] for g in clones]
        finally:
            eng.close()
        rate = sum(int(b[8]) - int(a[8]) for a, b in zip(c0, c1)) / (ms / 1e3)
        return rate, [int(b[15]) - int(a[15]) for a, b in zip(c0, c1)]

    cycles = None
    for shp in shapes:
        c, t = shp[0], shp[1]
        occ = shp[2] if len(shp) > 2 else 1
        try:
            rate, cyc = time_shape(c, t, occ=occ)
        except native.NativeError as e:
            table.append({"cluster": c, "threads": t, "ctas_per_sm": occ, "error": str(e)})
            continue
        table.append({"cluster": c, "threads": t, "ctas_per_sm": occ, "moves_per_s": rate})
        if best is None or rate > best[2]:
            best = (c, t, rate, (), 0, occ)
            cycles = cyc
    if best is not None and auto_split and best[5] == 1:
        c, t = best[0], best[1]
        spare = props.multi_processor_count - len(systems) * c
        by_cost = list(np.argsort(cycles)[::-1])
        for cb in sorted({c + 1, 2 * c}):
            if cb > 8:
                continue
            kmax = min(spare // (cb - c), len(systems) - 1)
            for k in sorted({kmax, kmax // 2} - {0}, reverse=True):
                split = tuple(int(i) for i in by_cost[:k])
                try:
                    rate, _ = time_shape(c, t, split, cb)
                except native.NativeError as e:
                    table.append({"cluster": c, "threads": t, "split": k, "cluster_b": cb, "error": str(e)})
                    continue
                table.append({"cluster": c, "threads": t, "split": k, "cluster_b": cb, "moves_per_s": rate})
                if rate > best[2]:
                    best = (c, t, rate, split, cb, 1)
    for g in clones:
        g.close()
    if best is None:
        raise native.NativeError("no launch shape could be created for this batch")
    shape = Shape(cluster=best[0], threads=best[1], moves_per_s=best[2], table=table, split=best[3],
                  cluster_b=best[4], ctas_per_sm=best[5])
    if use_cache:
        _CACHE[key] = shape
    return shape
