"""Launch-shape autotuner for the batched explicit Euler engine (NsBatch).

The batched step runs persistent kernels over a table of problems; its launch shape is
the node-kernel layout (one thread per vertex, or a group of lanes per vertex), the
vertex block (64/128/256 vertices per work block) and the persistent grid sizes of the
vertex and cell kernels (multiples of the 148 SMs). Results do not depend on the shape,
so candidates are timed on the live batch: each trial advances the problems by real
steps, timed on the device with CUDA events.
"""

SMS = 148
DEFAULT = (0, 128, SMS * 8, SMS * 8)


def apply(batch, shape):
    lanes, block_v, grid_v, grid_c = shape
    batch.set_node_kernel(lanes)
    batch.set_launch(block_v, grid_v, grid_c)


def tune_ns_batch(batch, steps=2, log=None, layouts=(0, 1)):
    """Coordinate search from DEFAULT: node-kernel layout, cell grid, vertex block,
    vertex grid, each candidate timed over `steps` steps after one untimed step (the
    graph for the new shape is captured there). Leaves the batch on the best shape and
    returns (shape, ms per step); `log` receives every trial."""
    best = DEFAULT
    apply(batch, best)
    batch.time_steps(1)
    t_best = batch.time_steps(steps)
    trials = [(best, t_best)]

    def try_(shape):
        nonlocal best, t_best
        apply(batch, shape)
        batch.time_steps(1)
        t = batch.time_steps(steps)
        trials.append((shape, t))
        if t < t_best:
            best, t_best = shape, t

    for lanes in layouts:
        if lanes != best[0]:
            try_((lanes,) + best[1:])
    for mult in (2, 4, 16, 32, 64):
        try_((best[0], best[1], best[2], SMS * mult))
    for bv in (64, 256):
        try_((best[0], bv, best[2], best[3]))
    for mult in (2, 4, 16, 32, 64):
        try_((best[0], best[1], SMS * mult, best[3]))
    if best != DEFAULT:
        # short trials are noisy: keep the pick only if it beats the default again over
        # a longer run
        confirm = 4 * steps
        apply(batch, DEFAULT)
        batch.time_steps(1)
        t_def = batch.time_steps(confirm)
        apply(batch, best)
        batch.time_steps(1)
        t_pick = batch.time_steps(confirm)
        trials.append((DEFAULT, t_def * steps / confirm))
        trials.append((best, t_pick * steps / confirm))
        if t_pick >= t_def:
            best, t_best = DEFAULT, t_def * steps / confirm
        else:
            t_best = t_pick * steps / confirm
    apply(batch, best)
    if log is not None:
        log.extend({"node_lanes": s[0], "block_v": s[1], "grid_v": s[2], "grid_c": s[3], "ms_per_step": t / steps}
                   for s, t in trials)
    return best, t_best / steps
