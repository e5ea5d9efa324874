"""Trace autotuner: picks the launch shape of the RESIDUALS / MERIT kernel per batch shape.

Two runtime knobs shape a trace launch without changing a single result bit:

* ``pack_rays`` -- the rays of the consecutive tuples one CTA traces (its four warps each take
  pack_rays / 4 rays: the rays per warp);
* ``variants_per_cta`` -- how many variants one CTA traces side by side, sharing its threads,
  its per-tuple reductions and its barriers.

Small systems (a singlet's 450 rays) leave threads idle in the last round of a pack and at the
barrier before the tuple sums; long ones want fewer, fuller packs. The best pair depends on the
surface count, the rays per tuple, the precision mode and the device, so the tuner measures:
each candidate pair is timed with CUDA events on the launching stream over a few launches on
(a sample of) the caller's batch, after warm-up, and the fastest is cached under the batch's
shape key. Every candidate gives bit-identical results, so the choice is free to change.
"""

from __future__ import annotations

import dataclasses
import json
import os
import threading

import torch

from .batch import ResidualLayout, SystemBatchHost

PACK_RAYS = (128, 256, 384, 512, 768, 1024)
VARIANTS_PER_CTA = (1, 2, 3, 4, 6, 8)


@dataclasses.dataclass(frozen=True)
class TracePlan:
    pack_rays: int = 512
    variants_per_cta: int = 1


def shape_key(host: SystemBatchHost, layout: ResidualLayout, mode: str) -> str:
    """What the best plan depends on: surfaces, wavelengths, the rays of each field, the
    failure and precision modes, the features the kernel is built for, and the device."""
    st = layout.settings
    rays = list(layout.samples)
    feat = (1 if host.non_coaxial else 0) | (2 if host.topology.ghost_plates else 0)
    dev = torch.cuda.get_device_name(torch.cuda.current_device())
    uneven = host.variant_surfaces is not None
    return (f"{mode}|S{host.surfaces}|L{host.wavelengths}|rays{rays}|fail{st.failure}|"
            f"prec{st.precision}|feat{feat}|uneven{int(uneven)}|{dev}")


class TraceAutotuner:
    """Measures and caches the fastest TracePlan per shape key. `cache_path` (optional) keeps
    the choices in a JSON file across processes."""

    def __init__(self, cache_path: str | None = None, sample_variants: int = 8192,
                 launches: int = 5, candidates=None):
        self.cache_path = cache_path
        self.sample_variants = sample_variants
        self.launches = launches
        self.candidates = list(candidates) if candidates is not None else \
            [TracePlan(r, v) for r in PACK_RAYS for v in VARIANTS_PER_CTA]
        self.cache: dict[str, dict] = {}
        self._lock = threading.Lock()
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as fh:
                self.cache = json.load(fh)

    def plan(self, host: SystemBatchHost, layout: ResidualLayout, mode: str = "merit",
             dbatch=None) -> TracePlan:
        """The cached plan for this shape, measuring it first when it is not known."""
        key = shape_key(host, layout, mode)
        with self._lock:
            hit = self.cache.get(key)
        if hit is None:
            hit = self.tune(host, layout, mode, dbatch)
        return TracePlan(hit["pack_rays"], hit["variants_per_cta"])

    def tune(self, host: SystemBatchHost, layout: ResidualLayout, mode: str = "merit",
             dbatch=None) -> dict:
        """Times every candidate on up to `sample_variants` variants of the batch and records
        the fastest; returns {pack_rays, variants_per_cta, ms, timings}."""
        from . import engine
        n = min(host.variants, self.sample_variants)
        sample = host if n == host.variants else host.subset(0, n)
        db = dbatch if dbatch is not None and n == host.variants else \
            engine.DeviceSystemBatch(sample)
        stream = torch.cuda.current_stream()
        ws = None
        if mode == "merit":
            import ctypes as C
            from . import _capi
            plan_c = layout.plan(sample)
            ws = torch.empty(int(_capi.lib().mkb_merit_workspace_bytes(n, C.byref(plan_c))),
                             dtype=torch.uint8, device=db.device)

        def launch(tp: TracePlan):
            if mode == "merit":
                engine.merit_device(db, layout, sample, workspace=ws, pack_rays=tp.pack_rays,
                                    variants_per_cta=tp.variants_per_cta)
            else:
                engine.residuals_device(db, layout, sample, pack_rays=tp.pack_rays,
                                        variants_per_cta=tp.variants_per_cta)

        timings = []
        for tp in self.candidates:
            try:
                launch(tp)  # warm-up (and the shared-memory attribute, outside any capture)
                launch(tp)
            except (RuntimeError, ValueError, NotImplementedError):
                continue  # a plan the device cannot take (shared memory): not a candidate
            # the launches replayed from a CUDA graph, so that the host's enqueue time never
            # shows in the events of a small batch
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph):
                for _ in range(self.launches):
                    launch(tp)
            graph.replay()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            graph.replay()
            e1.record(stream)
            e1.synchronize()
            del graph
            timings.append((e0.elapsed_time(e1) / self.launches, tp))
        if not timings:
            raise RuntimeError("trace autotuner: no candidate plan could be launched")
        ms, best = min(timings, key=lambda t: t[0])
        entry = {"pack_rays": best.pack_rays, "variants_per_cta": best.variants_per_cta,
                 "ms": ms, "sample_variants": n,
                 "timings": [[t.pack_rays, t.variants_per_cta, m] for m, t in timings]}
        key = shape_key(host, layout, mode)
        with self._lock:
            self.cache[key] = entry
            if self.cache_path:
                tmp = self.cache_path + ".tmp"
                with open(tmp, "w") as fh:
                    json.dump(self.cache, fh, indent=1)
                os.replace(tmp, self.cache_path)
        return entry
