"""Run-loop failure semantics on the GPU, without faulting it.

  * A neighbour list that overflows in the middle of a run is raised within
    two captured chunks (16 steps each) of the chunk whose build overflowed:
    the engine reads each chunk's status words while the next two chunks
    run, so the GPU always has queued work while the host waits.  (The
    reference raises right after the overflowing build,
    native/src/simulation/neighbor/neighbor_system.cpp:143.)  The overflow
    itself is an ordinary status bit: the build clamps its writes at the
    capacity, so nothing runs out of bounds.
  * A replica whose state has failed (a kinetic energy beyond the
    fixed-point range) builds no more lists: the rest of the chunk steps on
    the last list, and the error arrives at the chunk's end.
  * An interrupt (a pending signal, as Ctrl-C leaves it) stops
    execute_simulation at the next poll, well before the run would end (the
    reference polls every max(1, 100000 / N) steps,
    native/src/simulation/simulation_run.cpp:92).
"""

from __future__ import annotations

import signal
import time

import pytest

from beads_b200 import _native, workloads
from beads_b200.engine import Engine

pytestmark = pytest.mark.gpu

CHUNK = 16


def _tight_lattice():
    """A hot lattice whose list capacity is exactly its step-0 maximum: the
    melting lattice's neighbour counts spread and overflow at a later build."""
    spec = workloads.lj_lattice(temperature=3.0, check_every=1)
    with Engine(spec) as eng:
        eng.eval()
        spec.max_neighbors = int(eng.list_stats()["max"])
    return spec


def test_overflow_mid_run_raises_within_a_chunk():
    spec = _tight_lattice()
    limit = 3000
    # First failing step, one step per call (each call checks the status).
    first = None
    with Engine(spec) as eng:
        eng.eval()
        for s in range(1, limit + 1):
            try:
                eng.run(1)
            except RuntimeError as e:
                assert "NeighborList overflow" in str(e)
                first = s
                break
    assert first is not None and first > 1, "the lattice never overflowed its list"
    # The same dynamics in one long call: the error arrives at most two
    # chunks after the chunk holding the overflowing build.
    with Engine(spec) as eng:
        eng.eval()
        with pytest.raises(RuntimeError, match="NeighborList overflow"):
            eng.run(limit)
        done = eng.counters()["steps"]
    assert first <= done <= first + 3 * CHUNK, (first, done)


def test_interrupt_stops_execute_simulation(tmp_path, monkeypatch):
    from tests.golden.make_reference_fixtures import spec_for

    monkeypatch.chdir(tmp_path)
    r = workloads.lj_lattice()
    spec = spec_for(r, 2_000_000, "long", forces=False, thermo_every=100_000)

    def on_alarm(signum, frame):
        raise KeyboardInterrupt

    old = signal.signal(signal.SIGALRM, on_alarm)
    try:
        signal.setitimer(signal.ITIMER_REAL, 1.0)
        t0 = time.perf_counter()
        with pytest.raises(KeyboardInterrupt):
            _native.execute_simulation(spec)
        elapsed = time.perf_counter() - t0
    finally:
        signal.setitimer(signal.ITIMER_REAL, 0.0)
        signal.signal(signal.SIGALRM, old)
    # 2,000,000 steps of 4096 beads take about a minute; the poll stops it
    # within a few chunks of the signal.
    assert elapsed < 15.0, elapsed


def test_failed_state_stops_list_builds():
    import numpy as np

    import dataclasses

    # Berendsen on: the kinetic-energy total (fixed point) is formed every
    # step, so the failure is a status bit inside the chunk.
    spec = dataclasses.replace(workloads.lj_lattice(check_every=1), thermostat=(1.0, 1.0))
    with Engine(spec) as eng:
        eng.eval()
        pos = eng.state()["positions"].copy()
        # Two particles 0.05 sigma apart: energy (1.6e16) and virial (2e16)
        # are inside the fixed-point range at the evaluation, but the first
        # kick gives them ~1e16 sigma/tau, whose kinetic energy is not; the
        # next drifts throw them across the box, a rebuild on every step if
        # builds went on.
        pos[1] = pos[0] + np.array([0.05, 0.0, 0.0], np.float32)
        eng.set_state(0, positions=pos)
        eng.eval()
        builds0 = eng.counters()["builds"]
        with pytest.raises(OverflowError):
            eng.run(4 * CHUNK)
        c = eng.counters()
    # Step 1 may rebuild (its decision comes before the failing kick); none of
    # the later steps does, and the error arrives while at most two more
    # chunks run.
    assert c["steps"] >= 2, c
    assert c["builds"] <= builds0 + 1, (builds0, c)
    assert c["steps"] <= 3 * CHUNK, c
