"""Launch-shape tuner for the persistent tracing kernels.

Times a workload once per candidate launch shape — the refill threshold
(how empty a warp gets before its idle lanes take new rays from the queue)
and the resident blocks per SM — and returns the fastest, with every
candidate's device time. The workload is a callable that renders with the
current shape and returns its device milliseconds; each candidate runs it
`repeats` times after one untimed run (the first run of a shape captures
its CUDA graph) and keeps the median.
"""

import statistics

REFILL = (16, 20, 24, 28)
BLOCKS = (0, 4)


def tune(apply, workload, refill=REFILL, blocks=BLOCKS, repeats=2):
    """apply(refill_below, blocks_per_sm) sets a shape; workload() -> ms.
    Returns ((refill_below, blocks_per_sm), {shape: ms})."""
    times = {}
    for r in refill:
        for b in blocks:
            apply(r, b)
            workload()
            times[(r, b)] = statistics.median(workload() for _ in range(repeats))
    best = min(times, key=times.get)
    apply(*best)
    return best, times


def tune_batch(batch, frames, **kw):
    """Tunes a CudaBatch on one sample of `frames` (their frame_count is
    replaced by 1)."""
    from . import renderer
    one = []
    for f in frames:
        g = type(f).from_buffer_copy(f)
        g.frame_count = 1
        g.target.read_back = 0
        one.append(g)

    def workload():
        _, _, total = batch.render(one)
        renderer.check(total, "batch tuning sample")
        return total.gpu_ms

    return tune(batch.set_tuning, workload, **kw)
