"""Autotuner of the pass kernels' forms for one context and workload.

The library's kernel choices (tcg_forms: the XY and Z kernel forms, the
prefetching inverse XY pass, pruning of band-limited grids, the shared
transforms of tc2x / tc3a3b3b4b6 / tc3a2a4b2b5, the shared-memory
accumulations, the targets per chunk) have per-term defaults measured on the
36^3 production grid.  autotune() times the caller's own step -- the
per-state refresh and one apply of the given terms on device buffers -- for
each value of one knob at a time, keeps the fastest (coordinate descent, a
second sweep while it still improves) and leaves the context set to it.  Every
candidate computes the same result up to rounding; forms that the grid does
not support are skipped.
"""
from ._lib import TCError

#: knobs in the order they are swept, with the values tried
KNOBS = (
    ("fuse", (1, 0)),
    ("prune", (1, 0)),
    ("xy", (0, 1, 2, 3)),
    ("z", (0, 1, 2, 3, 4)),
    ("prefetch", (1, 0)),
    ("qp_sacc", (1, 0)),
    ("sacc", (0, 1)),
    ("min_targets", (0, 300, 1200)),
)


def _timer(ctx):
    """ms of one call of fn(), timed with CUDA events on the context's stream."""
    import torch
    stream = torch.cuda.ExternalStream(int(ctx.stream))

    def run(fn):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b)
    return run


def autotune(ctx, terms, psi_ptr, h2_ptr, h3_ptr, nb_apply=None, knobs=KNOBS, repeats=1, sweeps=2,
             include_state=True, log=None):
    """Choose the fastest kernel forms for ctx's workload: step = (per-state
    refresh if include_state) + apply of `terms` to the device arrays.
    Returns (best forms dict, [(forms dict, ms)] of every timed candidate)."""
    timer = _timer(ctx)

    def step():
        if include_state:
            ctx.refresh_state()
        ctx.apply_device(terms, psi_ptr, h2_ptr, h3_ptr, nb_apply=nb_apply)

    def measure(forms):
        ctx.set_forms(**forms)
        step()                                   # warm-up: tables, buffers, attributes
        return min(timer(step) for _ in range(max(1, repeats)))

    best = ctx.forms()
    best_ms = measure(best)
    trials = [(dict(best), best_ms)]
    if log:
        log(f"autotune start {best} {best_ms:.1f} ms")
    for _ in range(max(1, sweeps)):
        improved = False
        for name, values in knobs:
            for v in values:
                if best.get(name) == v:
                    continue
                cand = dict(best, **{name: v})
                try:
                    ms = measure(cand)
                except TCError:
                    continue                     # form not available for this grid
                trials.append((dict(cand), ms))
                if log:
                    log(f"autotune {name}={v}: {ms:.1f} ms")
                if ms < best_ms * 0.99:          # a gain above the timing noise
                    best, best_ms, improved = cand, ms, True
        if not improved:
            break
    ctx.set_forms(**best)
    return best, trials
