"""The exact solution of the 1D Riemann problem of an ideal gas (Toro 2009, ch. 4: the pressure function, Newton's method
for p*, the wave pattern sampled at x / t), without vacuum; cell averages by midpoint sub-samples, as the reference's
test helper takes them (src/test/exact_riemann.hpp). Test infrastructure."""
import math

import numpy as np


class ExactRiemann:
    def __init__(self, left, right, gamma):
        self.L, self.R, self.g = tuple(map(float, left)), tuple(map(float, right)), float(gamma)
        g = self.g
        self.cL = math.sqrt(g * self.L[2] / self.L[0])
        self.cR = math.sqrt(g * self.R[2] / self.R[0])
        p = max(1e-12, 0.5 * (self.L[2] + self.R[2]))
        for _ in range(100):
            fL, dL = self._f(p, self.L, self.cL)
            fR, dR = self._f(p, self.R, self.cR)
            nxt = max(1e-14, p - (fL + fR + self.R[1] - self.L[1]) / (dL + dR))
            done = 2 * abs(nxt - p) / (nxt + p) < 1e-15
            p = nxt
            if done:
                break
        self.p = p
        fL, _ = self._f(p, self.L, self.cL)
        fR, _ = self._f(p, self.R, self.cR)
        self.u = 0.5 * (self.L[1] + self.R[1] + fR - fL)

    def _f(self, p, K, c):
        g = self.g
        if p > K[2]:
            A, B = 2 / ((g + 1) * K[0]), (g - 1) / (g + 1) * K[2]
            q = math.sqrt(A / (p + B))
            return (p - K[2]) * q, q * (1 - 0.5 * (p - K[2]) / (B + p))
        return 2 * c / (g - 1) * ((p / K[2]) ** ((g - 1) / (2 * g)) - 1), 1 / (K[0] * c) * (p / K[2]) ** (-(g + 1) / (2 * g))

    def sample(self, s):
        """(rho, u, p) at s = (x - x0) / t."""
        g, p, u = self.g, self.p, self.u
        if s <= u:
            K, c, sign = self.L, self.cL, 1
        else:
            K, c, sign = self.R, self.cR, -1
        if p > K[2]:  # a shock
            S = K[1] - sign * c * math.sqrt((g + 1) / (2 * g) * p / K[2] + (g - 1) / (2 * g))
            if (s <= S) if sign > 0 else (s >= S):
                return K
            r, k = p / K[2], (g - 1) / (g + 1)
            return (K[0] * (r + k) / (k * r + 1), u, p)
        head = K[1] - sign * c
        cs = c * (p / K[2]) ** ((g - 1) / (2 * g))
        tail = u - sign * cs
        if (s <= head) if sign > 0 else (s >= head):
            return K
        if (s >= tail) if sign > 0 else (s <= tail):
            return (K[0] * (p / K[2]) ** (1 / g), u, p)
        cf = 2 / (g + 1) * (c + sign * (g - 1) / 2 * (K[1] - s))
        uf = 2 / (g + 1) * (sign * c + (g - 1) / 2 * K[1] + s)
        return (K[0] * (cf / c) ** (2 / (g - 1)), uf, K[2] * (cf / c) ** (2 * g / (g - 1)))

    def average(self, a, b, x0, t, samples=256):
        """The conservative average over [a, b] at time t with the jump at x0, as primitives."""
        g = self.g
        m = mom = e = 0.0
        for k in range(samples):
            x = a + (b - a) * (k + 0.5) / samples
            rho, u, p = self.sample((x - x0) / t)
            m += rho
            mom += rho * u
            e += p / (g - 1) + 0.5 * rho * u * u
        m, mom, e = m / samples, mom / samples, e / samples
        u = mom / m if m > 0 else 0.0
        return np.array([m, u, (g - 1) * (e - 0.5 * m * u * u)])
