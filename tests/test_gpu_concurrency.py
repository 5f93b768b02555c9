"""Two contexts on one device used from two host threads at once: each keeps its own Krylov workspace,
scalars and graph cache, so concurrent solves of different systems give bitwise the results of the
same solves run one after the other."""
import threading

import numpy as np
import pytest

from conftest import load_package

pytestmark = pytest.mark.gpu


def five_point(rsd, ctx, N, shift):
    n = N * N
    rows, cols, vals = [], [], []
    for j in range(N):
        for i in range(N):
            r = j * N + i
            k = 1.0 + 0.5 * np.sin(0.37 * i + shift) * np.cos(0.23 * j)
            ent = []
            if j:
                ent.append((r - N, -k))
            if i:
                ent.append((r - 1, -k))
            ent.append((r, 4.0 * k + 0.01))
            if i + 1 < N:
                ent.append((r + 1, -k))
            if j + 1 < N:
                ent.append((r + N, -k))
            for c, v in ent:
                rows.append(r); cols.append(c); vals.append(v)
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, np.array(rows) + 1, 1)
    rp = np.cumsum(rp)
    return rsd.CSR.from_host(ctx, rp, np.array(cols, np.int64), np.array(vals))


def test_two_contexts_two_threads_match_serial():
    rsd = load_package()
    cases = []
    for t, (N, prec) in enumerate(((160, rsd.FP64), (140, rsd.MIXED))):
        ctx = rsd.Context(0)
        A = five_point(rsd, ctx, N, 0.3 * t)
        b = ctx.to_device(np.sin(np.arange(N * N) * (0.01 + 0.003 * t)) + 0.5)
        cases.append((ctx, A, b, rsd.SolverConfig.make(tol=1e-10, max_iters=20000, precision=prec)))

    def run(case, out, idx, reps):
        ctx, A, b, cfg = case
        x = ctx.array(A.n)
        res = []
        for _ in range(reps):
            x.zero()
            rep = rsd.solve(ctx, A, b, x, cfg)
            res.append((x.download(), rep["iterations"]))
        out[idx] = res

    serial = [None, None]
    for i, c in enumerate(cases):
        run(c, serial, i, 1)
    conc = [None, None]
    th = [threading.Thread(target=run, args=(c, conc, i, 5)) for i, c in enumerate(cases)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i in range(2):
        for x, its in conc[i]:
            assert its == serial[i][0][1]
            assert np.array_equal(x, serial[i][0][0])
    for ctx, A, b, _ in cases:
        del A, b
        ctx.close()
