"""The parallel redistribution deciders, restated on the CPU, against the
reference's sequential loop (solver.rs:476-555) on random small grids.

The device decides a sweep's candidates in rounds instead of one after
another (sdr_b200/csrc/particles.cuh):

* short lists (k_redist_replay): every pending candidate claims its cell and
  its neighbours below the cap with a stamp that orders lower particle indices
  first, and runs once it holds all of them; once a round decides fewer than
  kRoundsMinDecided candidates, thread 0 decides the pending rest in index
  order;
* long lists (redist_par_run): the list is put in index order and cut into
  units (maximal runs of consecutive candidates in one cell); a unit claims
  like a candidate and, holding all its claims, moves its first
  min(excess, total room, unit length) candidates on its counts held in
  registers.

Within a round the decisions of ready candidates or units run concurrently on
the device. The model applies them one by one in a random order, reading the
counts as they change, so a check may see a neighbour before or after another
decider's write; every order must give the sequential loop's moves. No GPU."""
import random

import pytest

CAP = 8
MIN_DECIDED = 32  # kRoundsMinDecided


def neighbours(c, dims):
    nx, ny, nz = dims
    i, j, k = c % nx, (c // nx) % ny, c // (nx * ny)
    sxy = nx * ny
    return [c - 1 if i > 0 else -1, c + 1 if i + 1 < nx else -1, c - nx if j > 0 else -1,
            c + nx if j + 1 < ny else -1, c - sxy if k > 0 else -1, c + sxy if k + 1 < nz else -1]


def best_of(c, count, cavity, down, dims):
    """Most downhill neighbour below the cap, then the emptiest, then visit order."""
    best, best_down, best_room = -1, None, 0
    for q, n in enumerate(neighbours(c, dims)):
        if n < 0 or not cavity[n] or count[n] >= CAP:
            continue
        room = CAP - count[n]
        if best < 0 or down[q] > best_down or (down[q] == best_down and room > best_room):
            best, best_down, best_room = n, down[q], room
    return best


def sequential(cell, count, cavity, down, dims):
    """solver.rs:476-555: every particle in index order."""
    count = list(count)
    moves = {}
    for p, c in enumerate(cell):
        if count[c] <= CAP:
            continue
        b = best_of(c, count, cavity, down, dims)
        if b >= 0:
            count[c] -= 1
            count[b] += 1
            moves[p] = b
    return moves, count


def candidates(cell, count, cavity, dims):
    """k_redist_append: particles of over-cap cells with a neighbour below the cap."""
    out = []
    for p, c in enumerate(cell):
        if count[c] <= CAP:
            continue
        if any(n >= 0 and cavity[n] and count[n] < CAP for n in neighbours(c, dims)):
            out.append(p)
    return out


def claims_of(c, count, cavity, dims):
    return [n for n in neighbours(c, dims) if n >= 0 and cavity[n] and count[n] < CAP]


def candidate_rounds(cell, count, cavity, down, dims, rng, cands):
    """k_redist_replay's shared-memory rounds with the serial finish."""
    count = list(count)
    pend = sorted(cands)
    moves = {}
    for rnd in range(1, len(pend) + 2):
        claim = {}
        live = []
        for p in pend:  # claims (or leave the list)
            c = cell[p]
            if count[c] <= CAP:
                continue
            room = claims_of(c, count, cavity, dims)
            if not room:
                continue
            key = (rnd, -p)
            for n in room + [c]:
                claim[n] = max(claim.get(n, key), key)
            live.append(p)
        nxt = []
        decided = len(pend) - len(live)
        for p in rng.sample(live, len(live)):  # concurrent decisions, in a random order
            c = cell[p]
            key = (rnd, -p)
            if claim[c] != key or any(claim.get(n) != key for n in claims_of(c, count, cavity, dims)):
                nxt.append(p)
                continue
            decided += 1
            b = best_of(c, count, cavity, down, dims)
            if b >= 0:
                count[c] -= 1
                count[b] += 1
                moves[p] = b
        pend = sorted(nxt)
        if not pend:
            return moves, count
        if decided < MIN_DECIDED:  # thread 0 in index order over the pending rest
            for p in pend:
                c = cell[p]
                if count[c] <= CAP:
                    continue
                b = best_of(c, count, cavity, down, dims)
                if b >= 0:
                    count[c] -= 1
                    count[b] += 1
                    moves[p] = b
            return moves, count
    raise AssertionError("rounds did not end")


def unit_rounds(cell, count, cavity, down, dims, rng, cands):
    """redist_par_run: index order, units of one cell's consecutive candidates."""
    count = list(count)
    order = sorted(cands)
    heads = [q for q in range(len(order)) if q == 0 or cell[order[q - 1]] != cell[order[q]]]
    moves = {}
    pend = heads
    for rnd in range(1, len(heads) + 2):
        if not pend:
            return moves, count
        claim = {}
        live = []
        for m in pend:
            p = order[m]
            c = cell[p]
            if count[c] <= CAP:
                continue
            room = claims_of(c, count, cavity, dims)
            if not room:
                continue
            key = (rnd, -p)
            for n in room + [c]:
                claim[n] = max(claim.get(n, key), key)
            live.append(m)
        nxt = []
        for m in rng.sample(live, len(live)):
            p = order[m]
            c = cell[p]
            key = (rnd, -p)
            if claim[c] != key or any(claim.get(n) != key for n in claims_of(c, count, cavity, dims)):
                nxt.append(m)
                continue
            nbs = neighbours(c, dims)
            cn = [count[n] if n >= 0 and cavity[n] else CAP for n in nbs]
            room = sum(CAP - v for v in cn if v < CAP)
            need = min(max(count[c] - CAP, 0), room)
            nmov = 1 if need > 0 else 0
            while nmov < need and m + nmov < len(order) and cell[order[m + nmov]] == c:
                nmov += 1
            for u in range(nmov):
                best, best_down, best_room = -1, None, 0
                for q in range(6):
                    if cn[q] >= CAP:
                        continue
                    rq = CAP - cn[q]
                    if best < 0 or down[q] > best_down or (down[q] == best_down and rq > best_room):
                        best, best_down, best_room = q, down[q], rq
                assert best >= 0
                cn[best] += 1
                moves[order[m + u]] = nbs[best]
            if nmov:
                count[c] -= nmov
                for q in range(6):
                    if nbs[q] >= 0 and cavity[nbs[q]]:
                        count[nbs[q]] = cn[q]
        pend = nxt
    raise AssertionError("rounds did not end")


def scene(seed):
    """A random grid, cavity and particle layout: spread, crowded into a few
    cells (a jet's pile-up) or a checkerboard, in cell order or shuffled."""
    rng = random.Random(seed)
    dims = (rng.randint(3, 7), rng.randint(3, 7), rng.randint(2, 6))
    ncell = dims[0] * dims[1] * dims[2]
    cavity = [rng.random() < 0.85 for _ in range(ncell)]
    inside = [c for c in range(ncell) if cavity[c]] or [0]
    kind = rng.choice(["spread", "crowded", "checker"])
    per = []
    for c in range(ncell):
        if not cavity[c]:
            per.append(0)
        elif kind == "spread":
            per.append(rng.choice([0, 2, 5, 8, 9, 11, 14]))
        elif kind == "checker":
            i, j, k = c % dims[0], (c // dims[0]) % dims[1], c // (dims[0] * dims[1])
            per.append(rng.randint(9, 30) if (i + j + k) % 2 == 0 else rng.randint(0, 3))
        else:
            per.append(rng.randint(0, 6))
    if kind == "crowded":
        for c in rng.sample(inside, min(3, len(inside))):
            per[c] = rng.randint(40, 160)
    cell = [c for c in range(ncell) for _ in range(per[c])]
    if rng.random() < 0.5:
        rng.shuffle(cell)  # particles no longer in cell order: short units
    elif rng.random() < 0.5:  # mostly in cell order with a few swaps (an advected sorted list)
        for _ in range(len(cell) // 20):
            a, b = rng.randrange(len(cell)), rng.randrange(len(cell))
            cell[a], cell[b] = cell[b], cell[a]
    count = [0] * ncell
    for c in cell:
        count[c] += 1
    g = [rng.uniform(-1, 1) for _ in range(3)]
    down = [-g[0], g[0], -g[1], g[1], -g[2], g[2]]
    if rng.random() < 0.3:  # axis-aligned gravity: ties in `down`, so room and visit order decide
        down = [0.0, 0.0, 9.81, -9.81, 0.0, 0.0]
    return cell, count, cavity, down, dims, rng


@pytest.mark.parametrize("seed", range(120))
def test_parallel_deciders_give_the_sequential_moves(seed):
    cell, count, cavity, down, dims, rng = scene(seed)
    ref_moves, ref_count = sequential(cell, count, cavity, down, dims)
    cands = candidates(cell, count, cavity, dims)
    for order_seed in range(3):
        r = random.Random(1000 * seed + order_seed)
        mv, cn = candidate_rounds(cell, count, cavity, down, dims, r, cands)
        assert mv == ref_moves and cn == ref_count
        mv, cn = unit_rounds(cell, count, cavity, down, dims, r, cands)
        assert mv == ref_moves and cn == ref_count


def test_model_scenes_exercise_the_hard_cases():
    """The seeds above include crowded cells (many rounds, the serial finish),
    multi-candidate units and lists with no move at all."""
    crowded = units = serial = 0
    for seed in range(120):
        cell, count, cavity, down, dims, rng = scene(seed)
        cands = sorted(candidates(cell, count, cavity, dims))
        crowded += max(count) >= 40
        units += any(cell[a] == cell[b] for a, b in zip(cands, cands[1:]))
        serial += len(cands) >= 2 * MIN_DECIDED and max(count) >= 40
    assert crowded >= 10 and units >= 60 and serial >= 5
