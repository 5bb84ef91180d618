"""Model check of the persistent tcgen05 kernels' barrier protocols (CPU).

tc05_stream_kernel (kami_b200/csrc/tc05_gemm.cu) runs one producer thread,
one or two MMA-issuing threads and G epilogue groups over a ring of S
shared-memory slots and NA tensor-memory accumulators.  Problem j uses slot
j % S and accumulator j % NA, is issued by thread j % I and drained by group
j % G.  Every wait is an mbarrier wait on phase parity, which passes as soon
as the barrier's current phase has the other parity: it cannot tell the
phase it wants from the one two ahead.  A waiter that reaches a barrier
while an earlier phase it does not own is still open would pass early.

This test replays the kernel's roles as a discrete-event simulation over
random schedules (copies, MMAs and epilogues of random length; roles
advancing in random order) with that parity rule, and checks that no wait
ever passes before the phase the waiter needs has completed -- for every
(S, NA, G, I) the launcher chooses over the shapes it admits.  It also shows
that the two forms the launcher avoids do violate it: two issuers sharing an
odd number of slots, and more epilogue groups than accumulators.  The same
check covers the grouped kernel (grouped_tc05.cu), whose slots hold K chunks.
"""
import random

import pytest

SMEM = 227 * 1024
EPI_TILE = 32 * 20 * 4      # per-thread-store transpose tile per warp
STORE_BOX = 4096            # bulk-store staging box


def launcher_config(stage_bytes, bn, bulk_store):
    """(S, NA, G, I) as stream_launch chooses them; None when it declines
    (fewer than two slots, or a 16-32 KB problem without two issuers)."""
    naccs = min(8, 512 // bn)
    if bulk_store:
        groups, bufs = 2, 2
        budget = SMEM - 1024 - 512 - 4 * groups * bufs * STORE_BOX
        if budget // stage_bytes < 3:
            bufs = 1
            budget = SMEM - 1024 - 512 - 4 * groups * bufs * STORE_BOX
    else:
        groups = 4
        budget = SMEM - 1024 - 512 - 4 * groups * EPI_TILE
        if budget // stage_bytes < 3 or naccs < groups:
            groups = 2
            budget = SMEM - 1024 - 512 - 4 * groups * EPI_TILE
    stages = min(6, budget // stage_bytes)
    if bulk_store and 65536 <= stage_bytes <= 90 * 1024:
        return 1, 2, 1, 1  # two CTAs per SM: one slot, two accumulators, one group each
    if stages < 2:
        return None
    issuers = 2 if stage_bytes < 32768 and stages % 2 == 0 and naccs % 2 == 0 else 1
    if stage_bytes < 32768 and issuers != 2:
        return None
    return stages, naccs, groups, issuers


def admitted_configs():
    """Every configuration over the shapes the streaming form accepts (1D,
    M <= 128, padded N <= 256 in 16s, K <= 256, >= 16 KB of operands)."""
    out = set()
    for bm in (64, 128):
        for bn in range(16, 257, 16):
            for nkb in (1, 2, 3, 4):
                stage = nkb * (bm + bn) * 128
                if stage < 16384 or 2 * stage > SMEM - 1024 - 512 - 8 * EPI_TILE:
                    continue
                for bulk in (False, True):
                    if bulk and bn % 32:
                        continue
                    c = launcher_config(stage, bn, bulk)
                    if c is not None:
                        out.add(c)
    return sorted(out)


class Barrier:
    """mbarrier phase bookkeeping: `phase` = index of the current (open)
    phase; a wait on parity p passes when phase % 2 != p."""

    def __init__(self, count):
        self.count, self.pending, self.phase = count, count, 0

    def arrive(self):
        self.pending -= 1
        if self.pending == 0:
            self.phase += 1
            self.pending = self.count

    def passes(self, parity):
        return self.phase % 2 != parity


def simulate(S, NA, G, I, nprob, rng):
    """Run one random schedule; return the violations (a wait passing while
    the phase it needs is still open)."""
    full = [Barrier(1) for _ in range(S)]
    empty = [Barrier(1) for _ in range(S)]
    tfull = [Barrier(1) for _ in range(NA)]
    tempty = [Barrier(1) for _ in range(NA)]
    bad = []
    # asynchronous completions: (time, kind, payload)
    events = []
    now = 0
    prod_j = 0
    iss_j = list(range(I))            # next problem of each issuer
    iss_last_done = [0] * I           # per-issuer in-order completion time
    grp_j = list(range(G))
    grp_busy = [0] * G
    acc_holds = [None] * NA           # problem whose product is complete in acc b

    def need_phase_done(bar, k, who):
        # the wait for phase k passes now; it is correct only if k < bar.phase
        if k >= bar.phase:
            bad.append((who, k, bar.phase))

    steps = 0
    while steps < 200000:
        steps += 1
        progressed = False
        order = ["prod"] + [("iss", t) for t in range(I)] + [("grp", g) for g in range(G)]
        rng.shuffle(order)
        for role in order:
            if role == "prod" and prod_j < nprob:
                j = prod_j
                st = j % S
                if j >= S:
                    k = j // S - 1
                    if not empty[st].passes(k & 1):
                        continue
                    need_phase_done(empty[st], k, ("producer", j))
                events.append((now + rng.randint(1, 40), "load", st))
                prod_j += 1
                progressed = True
            elif isinstance(role, tuple) and role[0] == "iss":
                t = role[1]
                j = iss_j[t]
                if j >= nprob:
                    continue
                st, b = j % S, j % NA
                if not full[st].passes((j // S) & 1):
                    continue
                if j >= NA and not tempty[b].passes(((j // NA) - 1) & 1):
                    continue
                need_phase_done(full[st], j // S, ("issuer full", j))
                if j >= NA:
                    need_phase_done(tempty[b], j // NA - 1, ("issuer acc", j))
                done = max(now, iss_last_done[t]) + rng.randint(1, 30)   # in order per issuer
                iss_last_done[t] = done
                events.append((done, "mma", (st, b, j)))
                iss_j[t] += I
                progressed = True
            elif isinstance(role, tuple) and role[0] == "grp":
                g = role[1]
                j = grp_j[g]
                if j >= nprob or grp_busy[g] > now:
                    continue
                b = j % NA
                if not tfull[b].passes((j // NA) & 1):
                    continue
                need_phase_done(tfull[b], j // NA, ("epilogue", j))
                if acc_holds[b] != j:
                    bad.append(("epilogue reads a product it does not own", j, acc_holds[b]))
                end = now + rng.randint(1, 50)
                grp_busy[g] = end
                events.append((end, "drain", b))
                grp_j[g] += G
                progressed = True
        if not progressed:
            if not events:
                break
            events.sort(key=lambda e: e[0])
            t0, kind, payload = events.pop(0)
            now = max(now, t0)
            if kind == "load":
                full[payload].arrive()
            elif kind == "mma":
                st, b, j = payload
                acc_holds[b] = j
                empty[st].arrive()
                tfull[b].arrive()
            elif kind == "drain":
                tempty[payload].arrive()
    done = all(j >= nprob for j in iss_j) and all(j >= nprob for j in grp_j)
    if not done and not bad:
        bad.append(("stalled", iss_j, grp_j))
    return bad


def test_launcher_configs_cover_both_issuer_counts():
    cfgs = admitted_configs()
    assert any(c[3] == 2 for c in cfgs) and any(c[3] == 1 for c in cfgs)
    for S, NA, G, I in cfgs:
        assert NA >= G
        if I == 2:
            assert S % 2 == 0 and NA % 2 == 0


@pytest.mark.parametrize("cfg", admitted_configs())
def test_admitted_configs_never_pass_a_wait_early(cfg):
    S, NA, G, I = cfg
    rng = random.Random(hash(cfg) & 0xffff)
    for trial in range(12):
        nprob = rng.randint(1, 60)
        assert simulate(S, NA, G, I, nprob, rng) == [], (cfg, trial)


@pytest.mark.parametrize("cfg", [(3, 4, 2, 2),   # two issuers sharing three slots
                                 (6, 2, 4, 1),   # four groups over two accumulators
                                 (4, 3, 4, 1)])
def test_avoided_forms_do_pass_waits_early(cfg):
    S, NA, G, I = cfg
    rng = random.Random(7)
    found = any(simulate(S, NA, G, I, 48, rng) for _ in range(40))
    assert found, cfg


def simulate_grouped(S, NA, G, chunks, rng, acc_wait=True):
    """grouped_tc05_kernel (kami_b200/csrc/grouped_tc05.cu): loaders fill slot
    c % S for chunk c (problems take 1-2 K chunks of 64), one issuer consumes
    the chunks in order (freeing each slot with a commit) and, after a
    problem's last chunk, publishes accumulator p % NA; epilogue group p % G
    drains it.  `acc_wait` False drops the issuer's wait for a free
    accumulator (shown to break).  Returns the violations."""
    nchunk = sum(chunks)
    owner = [p for p, n in enumerate(chunks) for _ in range(n)]
    last = {c for c in range(nchunk) if c + 1 == nchunk or owner[c + 1] != owner[c]}
    full = [Barrier(1) for _ in range(S)]
    empty = [Barrier(1) for _ in range(S)]
    accf = [Barrier(1) for _ in range(NA)]
    acce = [Barrier(1) for _ in range(NA)]
    bad, events = [], []
    now, lc, ic, iss_done = 0, 0, 0, 0
    started = set()
    grp_p = list(range(G))
    grp_busy = [0] * G
    acc_holds = [None] * NA
    nprob = len(chunks)
    for _ in range(400000):
        progressed = False
        order = ["load", "iss"] + [("grp", g) for g in range(G)]
        rng.shuffle(order)
        for role in order:
            if role == "load" and lc < nchunk:
                s = lc % S
                if lc >= S:
                    if not empty[s].passes(((lc // S) - 1) & 1):
                        continue
                    if lc // S - 1 >= empty[s].phase:
                        bad.append(("loader", lc))
                events.append((now + rng.randint(1, 40), "load", s))
                lc += 1
                progressed = True
            elif role == "iss" and ic < nchunk:
                p, s, b = owner[ic], ic % S, owner[ic] % NA
                if p not in started:
                    if acc_wait and p >= NA:
                        if not acce[b].passes(((p // NA) - 1) & 1):
                            continue
                        if p // NA - 1 >= acce[b].phase:
                            bad.append(("issuer acc", p))
                    elif not acc_wait and acc_holds[b] is not None and acc_holds[b] != "drained" and p >= NA:
                        bad.append(("issuer overwrites an undrained accumulator", p))
                if not full[s].passes((ic // S) & 1):
                    continue
                if ic // S >= full[s].phase:
                    bad.append(("issuer full", ic))
                started.add(p)
                iss_done = max(now, iss_done) + rng.randint(1, 30)
                events.append((iss_done, "mma", (s, b, p, ic in last)))
                ic += 1
                progressed = True
            elif isinstance(role, tuple):
                g = role[1]
                p = grp_p[g]
                if p >= nprob or grp_busy[g] > now:
                    continue
                b = p % NA
                if not accf[b].passes((p // NA) & 1):
                    continue
                if p // NA >= accf[b].phase:
                    bad.append(("epilogue", p))
                if acc_holds[b] != p:
                    bad.append(("epilogue reads a product it does not own", p, acc_holds[b]))
                grp_busy[g] = now + rng.randint(1, 50)
                events.append((grp_busy[g], "drain", b))
                grp_p[g] += G
                progressed = True
        if not progressed:
            if not events:
                break
            events.sort(key=lambda e: e[0])
            t0, kind, x = events.pop(0)
            now = max(now, t0)
            if kind == "load":
                full[x].arrive()
            elif kind == "mma":
                s, b, p, is_last = x
                empty[s].arrive()
                if is_last:
                    acc_holds[b] = p
                    accf[b].arrive()
            else:
                acc_holds[x] = "drained"
                acce[x].arrive()
    if not bad and (ic < nchunk or any(p < nprob for p in grp_p)):
        bad.append(("stalled", ic, grp_p))
    return bad


@pytest.mark.parametrize("S,NA,G", [(2, 2, 2),   # the kernel's constants (two CTAs per SM)
                                    (6, 4, 2)])  # its earlier one-CTA-per-SM form
def test_grouped_kernel_protocol(S, NA, G):
    """The grouped kernel's constants (S slots, NA accumulators, G epilogue
    groups, one issuer) never pass a wait early over random chunk mixes."""
    rng = random.Random(11 + S)
    for _ in range(60):
        chunks = [rng.choice((1, 1, 1, 2)) for _ in range(rng.randint(1, 50))]
        assert simulate_grouped(S, NA, G, chunks, rng) == []


def test_grouped_kernel_needs_its_accumulator_wait():
    rng = random.Random(3)
    chunks = [1] * 40
    assert any(simulate_grouped(6, 4, 2, chunks, rng, acc_wait=False) for _ in range(30))


def simulate_two_loaders(S, ntiles, rng):
    """spmm_tc05_kernel (kami_b200/csrc/spmm_tc05.cu): two loader warps take
    the tiles alternately (tile j by loader j % 2) and fill slot j % S, each
    first waiting for the slot's previous use to be committed; one issuer
    consumes the tiles in order and frees each slot with a commit.  Returns
    the violations (a wait passing before the phase it needs completed)."""
    full = [Barrier(1) for _ in range(S)]
    empty = [Barrier(1) for _ in range(S)]
    bad, events = [], []
    now, ic, iss_done = 0, 0, 0
    lj = [0, 1]  # next tile of each loader
    filled = [None] * S
    for _ in range(200000):
        progressed = False
        order = [("load", 0), ("load", 1), ("iss", 0)]
        rng.shuffle(order)
        for kind, w in order:
            if kind == "load" and lj[w] < ntiles:
                j = lj[w]
                s = j % S
                if j >= S:
                    if not empty[s].passes(((j // S) - 1) & 1):
                        continue
                    if j // S - 1 >= empty[s].phase:
                        bad.append(("loader", w, j))
                events.append((now + rng.randint(1, 40), "load", (s, j)))
                lj[w] += 2
                progressed = True
            elif kind == "iss" and ic < ntiles:
                s = ic % S
                if not full[s].passes((ic // S) & 1):
                    continue
                if ic // S >= full[s].phase:
                    bad.append(("issuer", ic))
                if filled[s] != ic:
                    bad.append(("issuer reads a slot holding another tile", ic, filled[s]))
                iss_done = max(now, iss_done) + rng.randint(1, 30)
                events.append((iss_done, "mma", s))
                ic += 1
                progressed = True
        if not progressed:
            if not events:
                break
            events.sort(key=lambda e: e[0])
            t0, kind, x = events.pop(0)
            now = max(now, t0)
            if kind == "load":
                s, j = x
                filled[s] = j
                full[s].arrive()
            else:
                empty[x].arrive()
    if not bad and ic < ntiles:
        bad.append(("stalled", ic, lj))
    return bad


@pytest.mark.parametrize("S", [2, 3, 4, 5, 6])
def test_two_loaders_never_pass_a_wait_early(S):
    """Loader w at tile j already waited, at its previous tile j - 2, for the
    commit of tile j - 2 - S; the issuer consumes in order, so every tile up
    to j - 2 - S -- among them j - 2S, the previous fill of slot j % S that
    this loader made -- is consumed.  So with S >= 2 slots no loader waits
    more than one phase ahead of a slot, odd or even S alike."""
    rng = random.Random(S)
    for _ in range(40):
        assert simulate_two_loaders(S, rng.randint(1, 80), rng) == []


def test_two_loaders_one_slot_does_pass_a_wait_early():
    """With a single slot the argument fails (j - 2 - S < j - 2S), and the
    loaders do overtake: the launcher never runs two loaders on one slot."""
    rng = random.Random(5)
    assert any(simulate_two_loaders(1, 60, rng) for _ in range(60))
