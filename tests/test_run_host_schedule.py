"""The schedule of the overlapped host run (culbm_run_host, culbm_b200/csrc/sim.cu
run_host_overlapped / run_slab_steps), checked on the CPU.

The model restates the slab geometry (slab_z0, slab_lo), the task list and its
submission order (anti-diagonal d = j + t', then t'), the stream of each slab
(j mod 4) and the events a task waits for (step t-1 of slab j-1), and the
joins around the whole-domain steps of long runs.  From these it derives
happens-before and checks, at the level of z-planes per buffer:

* every step reads the state of the previous step from tasks that happen
  before it (its own region and one plane on each side);
* no two tasks that may run at the same time conflict (a write against a read
  or a write of the same plane of the same buffer), except steps of one
  in-place time step, whose cells touch disjoint locations by construction of
  the AA pattern (each location belongs to one cell per step);
* the dumps cover the domain, and a dump region's copy-out follows its dump.

Access sets per task, by plane (a cell touches only its own plane and the two
next to it):
* pull step t: reads buffer t%2 on its region +-1, writes buffer (t+1)%2 on its
  region;
* in-place odd kernel (t even): reads and writes its region +-1 (pulls from
  and pushes to neighbours); even kernel (t odd): its own region;
* dump after step T-1: reads the state on its region +-1 in pull mode and in
  the in-place layout A (T even), its own region in layout B (T odd); writes
  the fields of its region;
* every step and dump reads the op bytes and fields of its own region, which
  the slab's op-byte task and input copy wrote.
"""
import pytest

KSTREAMS = 4


def run_slabs(nx, ny, nz, nsteps, requested=0):
    n = nx * ny * nz
    want = requested if requested > 0 else (min(64, n >> 18) if nsteps <= 40 else min(32, n >> 19))
    return max(1, min(want, nz // 2))


def slab_z0(nz, ns, j):
    return j * nz // ns


def slab_lo(nz, ns, j, shift):
    if j <= 0:
        return 0
    if j >= ns:
        return nz
    return max(0, slab_z0(nz, ns, j) - shift)


def schedule(nz, T, ns, nst=KSTREAMS):
    """Tasks in submission order: (kind, t, j, shift) with kind in
    'build', 'step', 'dump', 'plain' (whole-domain steps, a full barrier)."""
    nst = min(ns, nst)

    def phase(t0, t1, build, dump):
        ts = []
        for j in range(ns):
            for t in range(t0 - 1 if build else t0, (t1 if dump else t1 - 1) + 1):
                ts.append((j + max(t - t0, 0), t, j))
        ts.sort(key=lambda x: (x[0], x[1]))
        out = []
        for d, t, j in ts:
            kind = "build" if t < t0 else ("dump" if t == t1 else "step")
            out.append((kind, t, j, max(t - t0, 0), t0))
        return out

    if T <= 2 * ns:
        return phase(0, T, True, True), nst
    ta, tb = ns, T - ns
    return phase(0, ta, True, False) + [("plain", ta, -1, 0, tb)] + phase(tb, T, False, True), nst


def check(nz, T, pull, ns):
    tasks, nst = schedule(nz, T, ns)
    n = len(tasks)
    anc = [set() for _ in range(n)]
    last_on_stream, step_task, barrier = {}, {}, None
    for i, (kind, t, j, sh, t0) in enumerate(tasks):
        pred = set()
        if kind == "plain":
            pred = set(range(i))            # join of every slab stream
            barrier = i
        else:
            st = j % nst
            if st in last_on_stream:
                pred.add(last_on_stream[st])
            if barrier is not None:
                pred.add(barrier)           # fork after the whole-domain steps
            if kind in ("step", "dump") and t > t0 and j > 0 and (j - 1) % nst != j % nst:
                pred.add(step_task[(t - 1, j - 1)])
            last_on_stream[st] = i
        if kind == "step":
            step_task[(t, j)] = i
        for p in pred:
            anc[i] |= anc[p] | {p}

    def region(j, sh):
        return slab_lo(nz, ns, j, sh), slab_lo(nz, ns, j + 1, sh)

    def accesses(k):
        kind, t, j, sh, _ = tasks[k]
        out = []
        if kind == "plain":
            return [(r, z, "w") for z in range(nz) for r in (("P", 0), ("P", 1), "mac")]
        if kind == "build":
            for z in range(slab_z0(nz, ns, j), slab_z0(nz, ns, j + 1)):
                out += [("in", z, "w"), ("ops", z, "w")]
            return out
        a, b = region(j, sh)
        if b <= a:
            return out
        near = range(max(0, a - 1), min(nz, b + 1))
        own = range(a, b)
        out += [("in", z, "r") for z in own] + [("ops", z, "r") for z in own]
        if kind == "dump":
            buf = ("P", T % 2) if pull else ("P", 0)
            zs = near if (pull or T % 2 == 0) else own
            return out + [(buf, z, "r") for z in zs] + [("mac", z, "w") for z in own]
        out += [("mac", z, "r") for z in own]
        if pull:
            return out + [(("P", t % 2), z, "r") for z in near] + [(("P", (t + 1) % 2), z, "w") for z in own]
        zs = near if t % 2 == 0 else own
        return out + [(("P", 0), z, "rw") for z in zs]

    acc = [accesses(k) for k in range(n)]
    problems = []
    for x in range(n):
        ax = {(r, z): m for r, z, m in acc[x]}
        for y in range(x + 1, n):
            if x in anc[y] or y in anc[x]:
                continue
            same_inplace_step = (not pull and tasks[x][0] == tasks[y][0] == "step" and tasks[x][1] == tasks[y][1])
            for r, z, m in acc[y]:
                m2 = ax.get((r, z))
                if m2 is None or (m == "r" and m2 == "r"):
                    continue
                if same_inplace_step and r == ("P", 0):
                    continue
                problems.append(("race", tasks[x][:3], tasks[y][:3], r, z))

    # Reads of the previous step's state, and of the op bytes / inputs.
    def writer_of(t, z):
        for k, (kind, tt, j, sh, _) in enumerate(tasks):
            if kind == "step" and tt == t:
                a, b = region(j, sh)
                if a <= z < b:
                    return k
        for k, (kind, tt, j, sh, tb) in enumerate(tasks):
            if kind == "plain" and tt <= t < tb:
                return k
        raise AssertionError(("no writer", t, z))

    for k, (kind, t, j, sh, _) in enumerate(tasks):
        if kind not in ("step", "dump"):
            continue
        a, b = region(j, sh)
        if b <= a:
            continue
        if t > 0:
            for z in range(max(0, a - 1), min(nz, b + 1)):
                w = writer_of(t - 1, z)
                if w != k and w not in anc[k]:
                    problems.append(("stale read", tasks[k][:3], tasks[w][:3], z))
        for z in range(a, b):
            jb = next(jj for jj in range(ns) if slab_z0(nz, ns, jj) <= z < slab_z0(nz, ns, jj + 1))
            wb = next(i for i, tk in enumerate(tasks) if tk[0] == "build" and tk[2] == jb)
            if wb not in anc[k]:
                problems.append(("inputs not in", tasks[k][:3], z))

    # The dump regions partition the domain.
    covered = []
    for kind, t, j, sh, _ in tasks:
        if kind == "dump":
            covered += list(range(*region(j, sh)))
    if sorted(covered) != list(range(nz)):
        problems.append(("dumps do not partition the domain",))
    return problems


@pytest.mark.parametrize("pull", [True, False])
@pytest.mark.parametrize("nz,T", [(1, 3), (3, 2), (5, 7), (9, 8), (16, 1), (16, 7), (37, 8), (40, 20),
                                  (40, 41), (9, 30), (280, 20), (280, 70), (280, 41)])
def test_schedule_has_no_race_and_no_stale_read(nz, T, pull):
    ns = run_slabs(288, 272, nz, T, requested=16 if nz < 280 else 0)
    assert ns == 1 or all(slab_z0(nz, ns, j + 1) - slab_z0(nz, ns, j) >= 2 for j in range(ns))
    problems = check(nz, T, pull, ns)
    assert not problems, problems[:5]


def test_automatic_slab_count():
    assert run_slabs(288, 272, 280, 20) == 64       # 21.9 M cells, a short run: 64 slabs of 2^18 or more
    assert run_slabs(288, 272, 280, 100) == 32      # a long run: 32 slabs of 2^19 or more
    assert run_slabs(128, 64, 160, 12) == 5         # 1.3 M cells
    assert run_slabs(128, 64, 160, 41) == 2
    assert run_slabs(48, 20, 44, 20) == 1
    assert run_slabs(512, 512, 256, 100) == 32
    assert run_slabs(288, 272, 3, 20, requested=16) == 1
