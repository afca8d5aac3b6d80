"""Launch-shape tuner for the batched wavefront.

Knobs (each 0 picks the library's default):
  refill_below   how empty a warp of the persistent tracing kernels gets
                 before its idle lanes take new rays from the queue;
  blocks_per_sm  resident blocks of those kernels per SM (0: as many as fit);
  rounds         the bounces run as wavefront rounds before the tail kernel
                 takes the paths still queued (the queue size at which one
                 thread per path beats a round; 0: chosen from the first
                 sample's queue counts);
  camera_tile    the camera pass's order within each scene: the image's
                 rows, or warp tiles of 4x8, 8x4 or 16x2 pixels.

The search is coordinate descent: starting from the defaults, each knob in
turn is swept over its candidates with the others at their best so far,
for `passes` passes. The workload is a callable that renders with the
current shape and returns its device milliseconds; each candidate runs it
`repeats` times after one untimed run (the first run of a shape captures
its CUDA graph) and keeps the median. Returns the best shape and every
measured candidate's time.
"""

import statistics

from . import abi

KNOBS = ("refill_below", "blocks_per_sm", "rounds", "camera_tile")
CANDIDATES = {
    "refill_below": (0, 16, 24, 28),
    "blocks_per_sm": (0, 4, 5),
    "rounds": (0, 5, 9),
    "camera_tile": (abi.CAMERA_TILE_ROWS, abi.CAMERA_TILE_4X8, abi.CAMERA_TILE_8X4, abi.CAMERA_TILE_16X2),
}


def shape_name(shape):
    return "/".join(f"{k}={v}" for k, v in zip(KNOBS, shape))


def tune(apply, workload, candidates=None, repeats=2, passes=1):
    """apply(*shape) sets a shape (one value per KNOBS entry); workload() ->
    ms. Returns (best shape, {shape: ms})."""
    candidates = candidates or CANDIDATES
    times = {}

    def measure(shape):
        if shape not in times:
            apply(*shape)
            workload()
            times[shape] = statistics.median(workload() for _ in range(repeats))
        return times[shape]

    best = tuple(candidates[k][0] for k in KNOBS)
    measure(best)
    for _ in range(passes):
        for i, knob in enumerate(KNOBS):
            for value in candidates[knob]:
                shape = best[:i] + (value,) + best[i + 1:]
                if measure(shape) < times[best]:
                    best = shape
    apply(*best)
    return best, times


def tune_batch(batch, frames, **kw):
    """Tunes a CudaBatch on one sample of `frames` (their frame_count is
    replaced by 1, and depth kept): returns tune()'s result."""
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

    def apply(refill_below, blocks_per_sm, rounds, camera_tile):
        batch.set_tuning(refill_below, blocks_per_sm, rounds, camera_tile)

    return tune(apply, workload, **kw)
