"""CPU model of the persistent batch kernel's tile tickets
(sph_batch_persistent_kernel, coffee_b200/csrc/axisym_kernels.cuh): in
every stage or KO phase the CTAs take kTicketTiles tiles at a time from
counter tp & 1 (tp: tile phases begun), asking for the next ticket before
working on the current one, and CTA 0 clears the other counter at the start
of the phase.  With the CTAs interleaved at random between their atomic
operations (each phase ending at a grid barrier), every tile of every phase
is worked on exactly once."""
import random

import pytest

TICKET = 4


def run_phases(nblocks, grid, nphases, seed):
    rng = random.Random(seed)
    tickets = [0, 0]
    done = []
    for tp in range(nphases):
        ctr = tp & 1
        seen = [0] * nblocks
        # CTA 0 clears the other counter at the start of the phase; the
        # others may already be taking tickets of this phase's counter
        events = []  # per CTA: a generator of its atomic steps
        def cta(b):
            if b == 0:
                tickets[(tp + 1) & 1] = 0
                yield
            base = tickets[ctr]
            tickets[ctr] += TICKET
            yield
            while base < nblocks:
                pending = tickets[ctr]
                tickets[ctr] += TICKET
                yield
                for t in range(base, min(base + TICKET, nblocks)):
                    seen[t] += 1
                yield
                base = pending
        live = [cta(b) for b in range(grid)]
        while live:
            g = rng.choice(live)
            try:
                next(g)
            except StopIteration:
                live.remove(g)
        done.append(seen)
    return done


@pytest.mark.parametrize("nblocks,grid", [(1, 1), (7, 3), (100, 16), (1000, 37), (5, 40)])
def test_every_tile_once_per_phase(nblocks, grid):
    for seed in range(5):
        for seen in run_phases(nblocks, grid, 12, seed):
            assert seen == [1] * nblocks
