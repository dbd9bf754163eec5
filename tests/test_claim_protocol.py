"""CPU model of the Hex20 claim protocol of csrc/claim_hex20.cuh.

A row node's first chunk is a hashed table of S slots (linear probing from
the column key's start slot). Several CTAs (element groups) insert columns
into the same row concurrently. Each CTA:
  * copies the row slot by slot (not atomically: every slot read is a
    scheduling point), probes every column in the copy;
  * runs placement rounds: pending columns take the first slot of their
    sequence that is empty in the copy (tentative, in shared memory), then all
    tentative claims go to the row with CAS (each a scheduling point) and the
    outcomes are written back to the copy; a claim that met a column this CTA
    also inserts reports the earliest step known to hold that column, which
    becomes the column's entry unless it has an earlier one, and a later slot
    the CTA claimed for it is retired (tombstone);
  * after the last round, walks the remaining columns one by one.

The model interleaves the CTAs at random and checks the invariants the kernel
relies on: no column is held by two live slots of the row, and every CTA's
entry for a column is the live slot that holds it (or the row is full and the
column goes to the overflow chunks).
"""
import random

import pytest

TOMB = -1


def _run(seed, S, nkeys, ncta, iters):
    rnd = random.Random(seed)
    row = [0] * S
    start = {k: rnd.randrange(S) for k in range(1, nkeys + 1)}
    ctas = [rnd.sample(range(1, nkeys + 1), rnd.randint(1, nkeys)) for _ in range(ncta)]
    entries = {}

    def slot(k, t):
        return (start[k] + t) % S

    def cta(cid, keys):
        view = [0] * S
        order = list(range(S))
        rnd.shuffle(order)
        for s in order:
            view[s] = row[s]
            yield
        res = {}
        for k in keys:
            r = ("chain", 255)
            for t in range(S):
                x = view[slot(k, t)]
                if x == k:
                    r = ("found", t)
                    break
                if x == 0:
                    r = ("try", t)
                    break
            res[k] = r
        for _ in range(iters):
            pending = False
            for k in keys:
                st, t = res[k]
                if st not in ("try", "fail"):
                    continue
                pending = True
                out = ("chain", 255)
                for t2 in range(t + 1 if st == "fail" else t, S):
                    s = slot(k, t2)
                    if view[s] == 0:
                        view[s] = k
                        out = ("tent", t2)
                        break
                    if view[s] == k:
                        out = ("found", t2)
                        break
                res[k] = out
            if not pending:
                break
            tent = [k for k in keys if res[k][0] == "tent"]
            rnd.shuffle(tent)
            for k in tent:
                t = res[k][1]
                s = slot(k, t)
                old = row[s]
                if old == 0:
                    row[s] = k
                yield
                if old not in (0, k):
                    view[s] = old
                res[k] = ("claimed" if old == 0 else "found" if old == k else "fail", t)
            home = {}
            for k in keys:
                st, t = res[k]
                if st != "fail":
                    continue
                s = slot(k, t)
                w = view[s]
                if w <= 0 or w not in keys:
                    continue
                home[w] = min(home.get(w, 255), (s - start[w]) % S)
            for w, tw in home.items():
                st, t = res[w]
                if (t < tw) if st == "fail" else (st != "chain" and t <= tw):
                    continue
                res[w] = ("found", tw)
                if st == "claimed":
                    so = slot(w, t)
                    row[so] = TOMB
                    view[so] = TOMB
                    yield
        for k in keys:
            st, t = res[k]
            if st != "fail":
                continue
            out = ("chain", 255)
            for t2 in range(t + 1, S):
                s = slot(k, t2)
                x = view[s]
                if x == k:
                    out = ("found", t2)
                    break
                if x != 0:
                    continue
                old = row[s]
                if old == 0:
                    row[s] = k
                yield
                view[s] = k if old == 0 else old
                if old in (0, k):
                    out = ("claimed" if old == 0 else "found", t2)
                    break
            res[k] = out
        entries[cid] = {k: (None if res[k][0] == "chain" else slot(k, res[k][1])) for k in keys}

    gens = [cta(i, ks) for i, ks in enumerate(ctas)]
    alive = list(range(ncta))
    while alive:
        i = rnd.choice(alive)
        try:
            next(gens[i])
        except StopIteration:
            alive.remove(i)
    live = [x for x in row if x > 0]
    assert len(live) == len(set(live)), (seed, row)
    for cid, mp in entries.items():
        for k, s in mp.items():
            if s is None:
                assert k not in row and all(x != 0 for x in row), (seed, cid, k, row)
            else:
                assert row[s] == k, (seed, cid, k, s, row)
    return row.count(TOMB)


@pytest.mark.parametrize("iters", [1, 2, 8])
def test_claim_rounds_keep_columns_unique(iters):
    tombs = 0
    for seed in range(1500):
        r = random.Random(seed * 7 + iters)
        tombs += _run(seed, S=r.choice([5, 6, 8, 10, 12]), nkeys=r.choice([4, 6, 9, 12]),
                      ncta=r.choice([2, 3, 4, 6]), iters=iters)
    assert tombs > 0  # the retire path is exercised
