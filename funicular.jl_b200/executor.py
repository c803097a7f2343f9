"""sweep!: the streaming pipeline over panel matrices (src/executor.jl).

Three queues: uploads on one, the panel function on a second, writebacks on a
third, ordered by events alone so that with nbuffers = 2 step s + 1 uploads
while step s computes (src/executor.jl:165-239). A staging slot is reused only
after the event of the step that held it nbuffers steps earlier. The host loop
never synchronizes and never allocates; it waits once, at the end. A producer
thread runs FEED_DEPTH steps ahead, bringing each step's panels into host
memory (src/executor.jl:102-111); ghost panels need no host memory here, so
for them it only paces the loop.
"""
from __future__ import annotations

import queue as _queue
import threading

from ._lib import ArgumentError
from .panels import (PanelMatrix, assert_same_panels, assert_same_rows, host_storage_eltype, materialize,
                     materialize_rows, writeback, writeback_rows)
from .plan import FEED_DEPTH, checkin_device_buffers, checkout_device_buffers, checkout_staging_storage, \
    row_block_height


class SweepOperand:
    """readpanels / writepanels / updatepanels (src/executor.jl:3-11)."""

    def __init__(self, pm: PanelMatrix, read: bool, write: bool):
        self.pm, self.read, self.write = pm, read, write


def readpanels(pm):
    """readpanels(pm) (src/executor.jl:9): a sweep operand staged up, not written back."""
    return SweepOperand(pm, True, False)


def writepanels(pm):
    """writepanels(pm) (src/executor.jl:10): a sweep operand written back, not staged up (its buffer starts undefined)."""
    return SweepOperand(pm, False, True)


def updatepanels(pm):
    """updatepanels(pm) (src/executor.jl:11): a sweep operand staged up and written back."""
    return SweepOperand(pm, True, True)


class PanelSteps:
    """One step per listed panel, repeats allowed read-only (src/executor.jl:22-27)."""

    def __init__(self, panels, labels=None):
        self.panels = list(panels)
        self.labels = list(labels) if labels is not None else list(range(len(self.panels)))

    @classmethod
    def count(cls, n):
        return cls(range(n))

    def nsteps(self):
        return len(self.panels)

    def label(self, step):
        return self.labels[step]

    def repeats_a_panel(self):
        return len(set(self.panels)) != len(self.panels)

    def buffer_dims(self, pm):
        return (pm.N, pm.w)

    def check(self, X, Y):
        assert_same_panels(X, Y)

    def view(self, buffer, step, pm):
        return buffer.view(slice(None), slice(0, pm.panels[self.panels[step]].width))

    def stage_in(self, dst, pm, step, queue, via):
        return materialize(dst, pm, self.panels[step], queue, via)

    def stage_out(self, pm, src, step, queue, via):
        return writeback(pm, self.panels[step], src, queue, via)

    def step_panels(self, pm, step):
        return [pm.panels[self.panels[step]]]


class RowSteps:
    """Blocks of rows spanning every panel (src/executor.jl:29-38)."""

    def __init__(self, N, height):
        h = max(1, min(int(height), int(N)))
        self.blocks = [range(top, min(top + h, N)) for top in range(0, N, h)]

    def nsteps(self):
        return len(self.blocks)

    def label(self, step):
        return step

    def repeats_a_panel(self):
        return False

    def buffer_dims(self, pm):
        return (len(self.blocks[0]), pm.k)

    def check(self, X, Y):
        assert_same_rows(X, Y)

    def view(self, buffer, step, pm):
        return buffer.view(slice(0, len(self.blocks[step])), slice(None))

    def stage_in(self, dst, pm, step, queue, via):
        return materialize_rows(dst, pm, self.blocks[step], queue, via)

    def stage_out(self, pm, src, step, queue, via):
        return writeback_rows(pm, src, self.blocks[step], queue, via)

    def step_panels(self, pm, step):
        return pm.panels


def rowtraversal(pm: PanelMatrix) -> RowSteps:
    """rowtraversal(pm) (src/executor.jl:38): row blocks of row_block_height rows."""
    return RowSteps(pm.N, row_block_height(pm.N, pm.k, pm.w))


def _stage_channel(steps, operands, errors):
    """stage_channel (src/executor.jl:102-111): the producer thread."""
    feed = _queue.Queue(maxsize=FEED_DEPTH)
    stop = threading.Event()

    def produce():
        try:
            for step in range(steps.nsteps()):
                for op in operands:
                    for panel in steps.step_panels(op.pm, step):
                        with op.pm.plan.hostpool.lock:
                            panel.pins += 1
                while not stop.is_set():
                    try:
                        feed.put(step, timeout=0.1)
                        break
                    except _queue.Full:
                        continue
                if stop.is_set():
                    return
        except BaseException as e:  # surfaced by the consumer
            errors.append(e)
            feed.put(None)

    t = threading.Thread(target=produce, daemon=True)
    t.start()
    return feed, stop, t


def sweep(f, *operands: SweepOperand, nbuffers=None, traversal=None) -> None:
    """sweep!(f!, operands...; nbuffers, traversal) (src/executor.jl:165-239):
    calls f(label, buffers...) once per step with one device staging buffer
    per operand, the work landing on the compute queue."""
    if not operands:
        raise ArgumentError("a sweep needs at least one panel matrix, wrapped as readpanels(pm), writepanels(pm) "
                            "or updatepanels(pm)")
    reference = operands[0].pm
    plan = reference.plan
    steps = traversal if traversal is not None else PanelSteps.count(reference.npanels())
    for op in operands:
        steps.check(reference, op.pm)
        if op.pm.plan is not plan:
            raise ArgumentError("every panel matrix in one sweep must belong to the same ResidencyPlan, since the "
                                "plan is what owns the staging buffers the sweep runs through. Build both matrices "
                                "from one plan")
        if op.write:
            op.pm.assert_writable()
    for i in range(1, len(operands)):
        for l in range(i):
            if operands[i].pm is operands[l].pm:
                raise ArgumentError("the same panel matrix takes part in one sweep twice. Pass it once as "
                                    "updatepanels(pm) if the sweep both reads and writes it")
    requested = plan.nbuffers if nbuffers is None else int(nbuffers)
    if requested < 1:
        raise ArgumentError(f"nbuffers must be at least 1, got {requested}")
    writing = any(op.write for op in operands)
    if writing and steps.repeats_a_panel():
        raise ArgumentError("this sweep visits a panel more than once and writes back, so the second visit would "
                            "overwrite the first. Repeated panels are only allowed in a read-only sweep")

    backend = plan.backend
    count = steps.nsteps()
    nb = min(requested, count)
    dims = [steps.buffer_dims(op.pm) for op in operands]
    buffers = []
    staging = []
    try:
        for op, d in zip(operands, dims):
            buffers.append(checkout_device_buffers(plan, op.pm.dtype, d, nb))
        for op, d in zip(operands, dims):
            S = host_storage_eltype(plan, op.pm.dtype)
            narrowed = S != op.pm.dtype and not op.pm.is_ghost()
            staging.append(checkout_staging_storage(plan, S, d, nb) if narrowed else None)
    except BaseException:
        for b in buffers:
            checkin_device_buffers(plan, b)
        for s in staging:
            if s is not None:
                checkin_device_buffers(plan, s)
        raise
    up, compute, down = backend.make_sweep_queues()
    slotfree = [None] * nb
    errors = []
    feed, stop, producer = _stage_channel(steps, operands, errors)
    try:
        for _ in range(count):
            step = feed.get()
            if step is None:
                raise errors[0]
            slot = step % nb
            targets = [steps.view(b[slot], step, op.pm) for op, b in zip(operands, buffers)]
            vias = [None if s is None else steps.view(s[slot], step, op.pm) for op, s in zip(operands, staging)]
            label = steps.label(step)
            free = slotfree[slot]
            if free is not None:
                backend.wait_event(up, free)
            for op, target, via in zip(operands, targets, vias):
                if op.read:
                    steps.stage_in(target, op.pm, step, up, via)
            backend.wait_event(compute, backend.record_event(up))
            done = backend.submit(compute, lambda: f(label, *targets))
            if writing:
                backend.wait_event(down, done)
                for op, target, via in zip(operands, targets, vias):
                    if op.write:
                        steps.stage_out(op.pm, target, step, down, via)
                done = backend.record_event(down)
            slotfree[slot] = done
            for op in operands:
                for panel in steps.step_panels(op.pm, step):
                    with plan.hostpool.lock:
                        panel.pins -= 1
                        panel.hold = done
        # Compute first, so the caller sees a failure of the panel function.
        backend.sync_queue(compute)
        backend.sync_queue(up)
        backend.sync_queue(down)
    except BaseException:
        for op in operands:
            with plan.hostpool.lock:
                for panel in op.pm.panels:
                    panel.pins = 0
        raise
    finally:
        stop.set()
        producer.join()
        sync_quietly(backend, (up, compute, down))
        for b in buffers:
            checkin_device_buffers(plan, b)
        for s in staging:
            if s is not None:
                checkin_device_buffers(plan, s)


def sync_quietly(backend, queues) -> None:
    """sync_quietly (src/executor.jl:113-122): drains the queues on the way out
    of a sweep, failed or not, so no pending copy still uses a staging buffer
    once it goes back to the pool; a failure here was already raised."""
    for q in queues:
        try:
            backend.sync_queue(q)
        except Exception:
            pass


def foreachpanel(f, pm: PanelMatrix, *, write=True, nbuffers=None) -> None:
    """foreachpanel (src/executor.jl:265-267)."""
    sweep(f, updatepanels(pm) if write else readpanels(pm), nbuffers=nbuffers)
