"""Launch-shape autotuner for the persistent trace kernel.

Searches the occupancy class (resident 128-thread blocks per SM, i.e. the
register cap of the kernel instantiation), the per-warp refill threshold (idle
lanes before a warp pulls new photons), the photons a warp claims per queue
access and, in image mode, whether the rays' backward leg and the rest run as
split launches (backward leg, packet generation, the rest) or one, timing each candidate with the library's own CUDA
events around the trace launch on the actual workload.  Results are cached per
(workload key, precision, integrator) for the life of the process.
"""

from __future__ import annotations

import itertools

_CACHE: dict = {}

BLOCKS_PER_SM = (2, 3, 4)   # 128-thread blocks; register caps 255 / 170 / 128
REFILL = (1, 8, 16, 32)
GRAB = (32, 128)
SPLIT_LEGS = (1, 0)         # image mode: split legs (three launches per chunk), or one launch


def candidates(image_mode: bool = True):
    """Occupancy classes (resident 128-thread blocks per SM, which fix the
    register cap of the instantiation) crossed with the queue knobs and, in
    image mode, the leg split."""
    for bps, refill, grab, split in itertools.product(BLOCKS_PER_SM, REFILL, GRAB,
                                                      SPLIT_LEGS if image_mode else (0,)):
        yield dict(threads_per_block=128, blocks_per_sm=bps, refill_threshold=refill, photons_per_grab=grab,
                   split_legs=split)


def tune(ctx, prepare, key, reps: int = 2, log=None):
    """Pick the fastest launch shape for `ctx`.

    prepare(ctx) must reset the photons (e.g. re-initialise the pixel grid);
    each candidate is run `reps` times after one warm-up and scored by its
    best trace-kernel time.  Returns (best_config, best_ms, table).
    """
    k = (key, ctx.params.precision, ctx.params.integrator)
    if k in _CACHE:
        cfg, ms, table = _CACHE[k]
        ctx.set_launch_config(**cfg)
        return cfg, ms, table
    table = []
    best = None
    from .abi import MODE_IMAGE
    for cfg in candidates(ctx.params.mode == MODE_IMAGE):
        ctx.set_launch_config(**cfg)
        prepare(ctx)
        ctx.run()
        t = []
        for _ in range(reps):
            prepare(ctx)
            t.append(ctx.run()["trace_ms"])
        ms = min(t)
        table.append((cfg, ms))
        if log:
            log(f"autotune {key} {cfg} {ms:.3f} ms")
        if best is None or ms < best[1]:
            best = (cfg, ms)
    ctx.set_launch_config(**best[0])
    _CACHE[k] = (best[0], best[1], table)
    return best[0], best[1], table
