"""Operation count of the reference's analytic assembly, per ordered fiber pair.

Test and measurement infrastructure (not shipped, not on the product path):
a scalar restatement of the reference formulas run on a counting number type,
so that the algorithmic work of one assembly is a counted figure rather than
an estimate.  It follows
  * Int_analytical.f90:83-207   b, c, ue, ub, d and the I/J/S moments
                                 (forward recursion for c < 10, backward from
                                 n = 27 otherwise, the d < 1e-14 branch);
  * Int_analytical.f90:213-288, 735-746   Legendre combinations L11..L24 and
                                 the Stokeslet + doublet tensor G_l, l = 0..N;
  * matrix_assembly.f90:534, 551-615   target point, projection
                                 theta^k_l = sum_q w_q P_k(s_q) G_l(q) and the
                                 3x3 block entries for k, l = 1..N;
  * matrix_assembly.f90:874-899  right-hand side from theta^k_0.
One FMA counts as two flops (it is never formed here: every operation is a
separate add or multiply); divisions, square roots and logarithms are counted
apart.  The item cost depends on which recursion runs, so the per-pair figure
is reported for both and mixed with a fraction of near items.

    python oracle/count_flops.py [near_fraction]
"""
import math
import sys


class Counter:
    add = mul = div = sqrt = log = 0

    @classmethod
    def reset(cls):
        cls.add = cls.mul = cls.div = cls.sqrt = cls.log = 0


class F:
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v.v if isinstance(v, F) else float(v)

    def __add__(self, o):
        Counter.add += 1
        return F(self.v + F(o).v)

    __radd__ = __add__

    def __sub__(self, o):
        Counter.add += 1
        return F(self.v - F(o).v)

    def __rsub__(self, o):
        Counter.add += 1
        return F(F(o).v - self.v)

    def __mul__(self, o):
        Counter.mul += 1
        return F(self.v * F(o).v)

    __rmul__ = __mul__

    def __truediv__(self, o):
        Counter.div += 1
        return F(self.v / F(o).v)

    def __rtruediv__(self, o):
        Counter.div += 1
        return F(F(o).v / self.v)

    def __neg__(self):
        return F(-self.v)

    def __lt__(self, o):
        return self.v < F(o).v


def fsqrt(x):
    Counter.sqrt += 1
    return F(math.sqrt(x.v))


def flog(x):
    Counter.log += 1
    return F(math.log(abs(x.v)))


LEG = {0: {0: 1}, 1: {1: 1}, 2: {2: 3, 0: -1}, 3: {3: 5, 1: -3}, 4: {4: 35, 2: -30, 0: 3},
       5: {5: 63, 3: -70, 1: 15}}
SCALE = {0: 1, 1: 1, 2: 0.5, 3: 0.5, 4: 0.125, 5: 0.125}


def moments(b, c, K):
    I, J, S = [F(0)] * K, [F(0)] * K, [F(0)] * K
    ue = fsqrt(1 + b + c)
    ub = fsqrt(1 - b + c)
    te = 1 + 0.5 * b
    tb = -1 + 0.5 * b
    d = c - 0.25 * b * b
    I[0] = flog(2 + b + 2 * ue) - flog(-2 + b + 2 * ub)
    I[1] = ue - ub - 0.5 * b * I[0]
    J[0] = te / (d * ue) - tb / (d * ub)
    J[1] = -1 / ue + 1 / ub - b * 0.5 * J[0]
    d6 = 6 * d
    ue3, ub3 = ue * ue * ue, ub * ub * ub
    S[0] = (2 + b) / (d6 * ue3) - (-2 + b) / (d6 * ub3) + 2 / (3 * d) * J[0]
    S[1] = -(b + 2 * c) / (d6 * ue3) + (-b + 2 * c) / (d6 * ub3) - b / (3 * d) * J[0]
    if c < 10:
        for n in range(2, K):
            nn = n + 1.0
            om = 1 - nn
            sbp = 1.0 if n % 2 == 1 else -1.0
            I[n] = sbp * ub / om - ue / om - (0.5 - (nn - 1)) * b / om * I[n - 1] + (nn - 2) * c / om * I[n - 2]
            J[n] = I[n - 2] - b * J[n - 1] - c * J[n - 2]
            S[n] = J[n - 2] - b * S[n - 1] - c * S[n - 2]
    else:
        i1 = i2 = j1 = j2 = s1 = s2 = F(0)
        for n in range(27, 1, -1):
            a0, r2, cb = (n + 2.0) / (n + 1.0), 1.0 / (n + 2.0), (1 - 2 * (n + 2.0)) / (2 * (n + 2.0))
            sbp = 1.0 if (n + 1) % 2 == 0 else -1.0
            i_ = a0 / c * (ue * r2 - sbp * ub * r2 + cb * b * i1 - i2)
            j_ = (i_ - b * j1 - j2) / c
            s_ = (j_ - b * s1 - s2) / c
            if n < K:
                I[n], J[n], S[n] = i_, j_, s_
            i2, i1, j2, j1, s2, s1 = i1, i_, j1, j_, s1, s_
    return I, J, S


def item(R0, p, N, eps2):
    """G_l (6 components), l = 0..N, at one target point for one source."""
    b = -2 * (p[0] * R0[0] + p[1] * R0[1] + p[2] * R0[2])
    c = R0[0] * R0[0] + R0[1] * R0[1] + R0[2] * R0[2]
    I, J, S = moments(b, c, N + 3)
    ia, ib = (0, 1, 2, 0, 0, 1), (0, 1, 2, 1, 2, 2)
    rr = [R0[x] * R0[y] for x, y in zip(ia, ib)]
    pr = [p[x] * R0[y] + R0[x] * p[y] for x, y in zip(ia, ib)]
    pp = [p[x] * p[y] for x, y in zip(ia, ib)]
    G = []
    for m in range(N + 1):
        L = [F(0)] * 7
        for pw, a in LEG[m].items():
            for t, v in enumerate((I[pw], J[pw], J[pw + 1], J[pw + 2], S[pw], S[pw + 1], S[pw + 2])):
                L[t] = L[t] + a * v
        L = [SCALE[m] * v for v in L]
        e2 = 2 * F(eps2)
        cI = L[0] + e2 * L[1]
        cRR = L[1] - 3 * e2 * L[4]
        cPR = -L[2] + 3 * e2 * L[5]
        cPP = L[3] - 3 * e2 * L[6]
        G.append([cRR * rr[k] + cPR * pr[k] + cPP * pp[k] + (cI if k < 3 else 0) for k in range(6)])
    return G


def pair_cost(c_value, N=5, LQ=24):
    """Counted operations of one ordered pair whose 24 items all take the recursion of c_value."""
    Counter.reset()
    dist = math.sqrt(c_value)
    p = [F(0.0), F(0.0), F(1.0)]
    t = [F(1.0), F(0.0), F(0.0)]
    xi = [F(0.0), F(dist), F(0.0)]
    xj = [F(0.0), F(0.0), F(0.0)]
    theta = [[[F(0)] * 6 for _ in range(N + 1)] for _ in range(N + 1)]
    for q in range(LQ):
        s = -1.0 + (2.0 * q + 1.0) / LQ
        xbar = [xi[a] + s * t[a] for a in range(3)]           # matrix_assembly.f90:534
        R0 = [xbar[a] - xj[a] for a in range(3)]
        G = item(R0, p, N, 1e-6)
        w = [0.08 * (k + 1) for k in range(N + 1)]          # w_q P_k(s_q): table values
        for k in range(N + 1):
            for l in range(N + 1):
                for cc in range(6):
                    theta[k][l][cc] = theta[k][l][cc] + w[k] * G[l][cc]
    for k in range(1, N + 1):                               # block entries, matrix_assembly.f90:551-615
        for l in range(1, N + 1):
            th = theta[k][l]
            Q = [th[0] * t[0] + th[3] * t[1] + th[4] * t[2], th[3] * t[0] + th[1] * t[1] + th[5] * t[2],
                 th[4] * t[0] + th[5] * t[1] + th[2] * t[2]]
            for a in range(3):
                for bb in range(3):
                    if k == 1:
                        _ = 0.75 * t[a] * Q[bb]
                    else:
                        _ = 1.1 * (th[0] - 0.3 * t[a] * Q[bb])
    for k in range(N + 1):                                  # right-hand side from theta^k_0
        th = theta[k][0]
        _ = [th[0] * 0.5 + th[3] * 0.5 + th[4] * 0.5 for _ in range(3)]
    return dict(add=Counter.add, mul=Counter.mul, div=Counter.div, sqrt=Counter.sqrt, log=Counter.log)


def main():
    near = float(sys.argv[1]) if len(sys.argv) > 1 else 0.116
    fwd, bwd = pair_cost(4.0), pair_cost(40.0)
    print("per ordered pair, all items forward recursion (c < 10):", fwd)
    print("per ordered pair, all items backward recursion (c >= 10):", bwd)
    mix = {k: near * fwd[k] + (1 - near) * bwd[k] for k in fwd}
    flops = mix["add"] + mix["mul"]
    print(f"mixed with {near:.3f} forward items: {flops:.0f} add+mul flops, {mix['div']:.0f} div, "
          f"{mix['sqrt']:.0f} sqrt, {mix['log']:.0f} log per ordered pair")
    M = 4000
    print(f"M = {M}: {flops * M * (M - 1) / 1e12:.3f} Tflop (add+mul) per assembly, "
          f"{(mix['div'] + mix['sqrt'] + mix['log']) * M * (M - 1) / 1e9:.1f} G div/sqrt/log")


if __name__ == "__main__":
    main()
