"""The L-BFGS step of the GPU Dimer (walkers.cu, lbfgs_translate) runs Nocedal's two-loop
recursion on coefficients: the step is a combination of the stored s_j, y_j and g, and the
loops read only the Gram entries s_i.y_j, y_i.y_j (kept per walker by ring slot, one row and
column added per stored pair) and g.s_j, g.y_j, g.g of the step.  This restates that
bookkeeping in numpy and checks it against the vector two-loop of oracle/walkers.py step by
step, through convex-region restarts, a full ring and its wraparound."""
import types

import numpy as np

from oracle.walkers import _Lbfgs


class VectorFree:
    """The coefficient form, slot by slot as the kernel keeps it."""

    def __init__(self, mem, box):
        self.mem, self.box = mem, np.asarray(box, dtype=np.float64)
        self.head = self.count = self.prev = 0
        self.rho = np.zeros(mem)
        self.SY = np.zeros((mem, mem))
        self.YY = np.zeros((mem, mem))
        self.S = [None] * mem
        self.Y = [None] * mem
        self.xp = self.gp = None

    def step(self, x, F0, N, fn, C, p):
        mem = self.mem
        if not C < 0.0:
            self.count = self.prev = 0
            return (1.0 if fn <= 0.0 else -1.0) * p.convex_step * N
        g = -(F0 - 2.0 * fn * N)
        h = self.head
        push = bool(self.prev)
        nold = min(self.count, mem - 1) if push else 0
        old = [(h - j) % mem for j in range(1, nold + 1)]        # stored pairs, newest first
        if push:
            s = x - self.xp
            s -= self.box * np.rint(s / self.box)
            y = g - self.gp
            sy = float(np.sum(s * y))
        self.xp, self.gp = x.copy(), g.copy()
        count = self.count
        gS, gY = {}, {}
        if push:
            if sy > 1e-12:
                self.S[h], self.Y[h] = s, y
                self.rho[h] = 1.0 / sy
                self.SY[h, h], self.YY[h, h] = sy, float(np.sum(y * y))
                for sj in old:
                    self.SY[h, sj] = float(np.sum(s * self.Y[sj]))
                    self.SY[sj, h] = float(np.sum(self.S[sj] * y))
                    self.YY[h, sj] = self.YY[sj, h] = float(np.sum(y * self.Y[sj]))
                self.head = (h + 1) % mem
                count = nold + 1
            else:
                count = 0
        ages = [(self.head - 1 - j) % mem for j in range(count)]  # slot of each stored pair, newest first
        for sl in ages:
            gS[sl], gY[sl] = float(np.sum(g * self.S[sl])), float(np.sum(g * self.Y[sl]))
        gg = float(np.sum(g * g))
        # q = qg g + sum qa_l y_l;  r = rg g + sum ra_l y_l + rb_l s_l
        qa = {sl: 0.0 for sl in ages}
        qg = 1.0
        al = {}
        for sj in ages:                                            # newest first
            sq = qg * gS[sj] + sum(qa[sl] * self.SY[sj, sl] for sl in ages)
            al[sj] = self.rho[sj] * sq
            qa[sj] -= al[sj]
        gam = (1.0 / self.rho[ages[0]]) / self.YY[ages[0], ages[0]] if count > 0 else 0.01
        ra = {sl: gam * qa[sl] for sl in ages}
        rg = gam * qg
        rb = {sl: 0.0 for sl in ages}
        for sj in reversed(ages):                                  # oldest first
            yr = rg * gY[sj] + sum(rb[sl] * self.SY[sl, sj] + ra[sl] * self.YY[sl, sj] for sl in ages)
            rb[sj] += al[sj] - self.rho[sj] * yr
        rgd = rg * gg + sum(rb[sl] * gS[sl] + ra[sl] * gY[sl] for sl in ages)
        self.prev = 1
        if not (-rgd < 0.0):                                       # not downhill: steepest descent
            self.count = 0
            return -0.01 * g
        self.count = count
        st = -rg * g
        for sl in ages:
            st = st - rb[sl] * self.S[sl] - ra[sl] * self.Y[sl]
        return st


def test_vector_free_steps_match_the_two_loop():
    rng = np.random.default_rng(5)
    n, box = 40, np.array([9.0, 10.0, 11.0])
    p = types.SimpleNamespace(convex_step=0.05, max_step=1e9)      # no cap: compare raw steps
    # a quadratic surface with one negative direction, seen through the modified force
    Q = rng.normal(0.0, 1.0, (3 * n, 3 * n))
    H = Q @ Q.T / (3 * n) + np.eye(3 * n)
    for mem in (3, 8):
        a, b = _Lbfgs(mem, box), VectorFree(mem, box)
        x = rng.uniform(0.0, 1.0, (n, 3)) * box
        N = rng.normal(0.0, 1.0, (n, 3))
        N /= np.linalg.norm(N)
        checked, full = 0, 0
        for it in range(60):
            F0 = -(H @ (x.reshape(-1) - 0.5 * box.repeat(1)[0])).reshape(n, 3) + rng.normal(0.0, 0.01, (n, 3))
            fn = float(np.sum(F0 * N))
            C = 1.0 if it in (7, 31) else -0.5                      # two convex-region restarts
            sa = a.step(x, F0, N, fn, C, p)
            sb = b.step(x, F0, N, fn, C, p)
            assert np.allclose(sa, sb, rtol=1e-10, atol=1e-12 * np.abs(sa).max()), (mem, it)
            checked += 1
            full += len(a.S) == mem == b.count
            x = x + sa
            x -= box * np.floor(x / box)                            # positions wrapped in place
        assert checked == 60
        assert full >= 3                                            # steps taken on a full ring
