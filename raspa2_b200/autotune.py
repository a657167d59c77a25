"""Launch-shape autotuner of the batched engine.

The engine advances each box with one thread-block cluster. Two shape
parameters decide how a batch maps onto the GPU:

- the cluster size: CTAs per box, which split the framework and the wave
  vectors between them;
- the CTA size: warps per CTA, which split the trial positions and
  framework chunks of one energy evaluation.

The best pair depends on the number of boxes against the SM count, on the
framework sizes and on the loadings. Measured on a B200 for 64 CO2 boxes of
512-4096 atoms, cluster x threads gave 0.22-1.48 M moves/s.

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


def _signature(systems: Sequence["native.GpuSystem"], precision: int) -> tuple:
    sig = []
    for g in systems:
        fw = g.sysm.framework()[0]
        sig.append((len(fw), g.natom, tuple(g.sysm.kmax), g.maxmol, bool(getattr(g, "grids_active", False))))
    return (precision, tuple(sorted(sig)))


def candidates(nsys: int, precision: int, sms: int) -> List[Tuple[int, int]]:
    """Shapes worth timing. A cluster size that needs more CTAs than there
    are SMs runs in waves (the engine's CTAs hold most of an SM's shared
    memory) and is skipped."""
    threads = (256, 512, 1024) if precision == native.RGPU_MIXED else (128, 256, 512)
    out = []
    for c in (1, 2, 4, 8):
        if nsys * c > sms and c > 1:
            continue
        for t in threads:
            out.append((c, t))
    return out


def _clone(g: "native.GpuSystem", xyz: np.ndarray) -> "native.GpuSystem":
    c = native.GpuSystem(g.sysm, **g.init_args)
    if getattr(g, "grids_active", False):
        c.share_grids_of(g)
    c.set_adsorbates(xyz)
    return c


def tune(systems: Sequence["native.GpuSystem"], precision: int = native.RGPU_MIXED, moves: int = 400,
         warm: int = 100, shapes: Optional[Sequence[Tuple[int, int]]] = None, use_cache: bool = True) -> Shape:
    """Times each candidate shape on copies of `systems` and returns the
    fastest as a Shape (with the full table of measurements)."""
    import torch

    key = _signature(systems, precision)
    if use_cache and shapes is None and key in _CACHE:
        return _CACHE[key]
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    shapes = list(shapes) if shapes is not None else candidates(len(systems), precision, props.multi_processor_count)
    start = [g.adsorbates() for g in systems]
    clones = [_clone(g, x) for g, x in zip(systems, start)]
    stream = torch.cuda.Stream()
    table = []
    best = None
    for c, t in shapes:
        for g, x in zip(clones, start):
            g.set_adsorbates(x)
        try:
            eng = native.Engine(clones, precision=precision, threads=t, cluster=c)
        except native.NativeError as e:
            table.append({"cluster": c, "threads": t, "error": str(e)})
            continue
        eng.run(warm, stream.cuda_stream)
        torch.cuda.synchronize()
        m0 = sum(int(g.state()["counters"][8]) for g in clones)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        eng.run(moves, stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        m1 = sum(int(g.state()["counters"][8]) for g in clones)
        rate = (m1 - m0) / (ms / 1e3)
        eng.close()
        table.append({"cluster": c, "threads": t, "moves_per_s": rate})
        if best is None or rate > best[2]:
            best = (c, t, rate)
    for g in clones:
        g.close()
    if best is None:
        raise native.NativeError("no launch shape could be created for this batch")
    shape = Shape(cluster=best[0], threads=best[1], moves_per_s=best[2], table=table)
    if use_cache:
        _CACHE[key] = shape
    return shape
