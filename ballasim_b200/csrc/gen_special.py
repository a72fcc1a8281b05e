"""Generates the fp32 constants of special.cuh from their published constructions, in 60-digit decimal arithmetic:

- Weideman (1994), "Computation of the complex error function", SIAM J. Numer. Anal. 31(5): erfcx(x) = w(ix) =
  2 p(Z) / (L + x)^2 + 1 / (sqrt(pi) (L + x)), Z = (L - x) / (L + x), with L = sqrt(N / sqrt 2) and p the degree
  N - 1 polynomial whose coefficients are the FFT (M = 2N nodes, 2M samples) of f(t) = e^{-t^2} (L^2 + t^2) at
  t_k = L tan(k pi / (2M)); N = 24 for fp32. This one is evaluated as the paper's published program does, in
  double with an FFT (numpy's): its rounding is part of the constants the reference's erfcx uses (the two
  highest-degree coefficients, ~1e-10, differ from the exact ones in their last float bits).
- Rybicki (1989), Dawson's integral by the exponentially convergent sum with step h = 1/4: the weights
  c_i = e^{-((2i + 1) h)^2}, i = 0..12.
- 8-point Gauss-Legendre on [0, 1]: the node pairs u = (1 -+ xi) / 2 and the halved weights.

Each value is rounded to the nearest double first and then to float, as a double constant cast to float in
fp32 code is; the fp32 kernels see only the float. Run `python gen_special.py` to print the constants."""
from decimal import Decimal as D, getcontext

import numpy as np

getcontext().prec = 60


def pi() -> D:
    getcontext().prec += 4
    three = D(3)
    lasts, t, s, n, na, d, da = 0, three, 3, 1, 0, 0, 24
    while s != lasts:
        lasts = s
        n, na = n + na, na + 8
        d, da = d + da, da + 32
        t = (t * n) / d
        s += t
    getcontext().prec -= 4
    return +s


def cos(x: D) -> D:
    getcontext().prec += 4
    i, lasts, s, fact, num, sign = 0, 0, D(1), 1, D(1), 1
    while s != lasts:
        lasts = s
        i += 2
        fact *= i * (i - 1)
        num *= x * x
        sign *= -1
        s += num / fact * sign
    getcontext().prec -= 4
    return +s


def sin(x: D) -> D:
    getcontext().prec += 4
    i, lasts, s, fact, num, sign = 1, 0, x, 1, x, 1
    while s != lasts:
        lasts = s
        i += 2
        fact *= i * (i - 1)
        num *= x * x
        sign *= -1
        s += num / fact * sign
    getcontext().prec -= 4
    return +s


def to_f32(v) -> float:
    """Nearest double, then nearest float (a double literal cast to float)."""
    return float(np.float32(float(v)))


def weideman(n: int) -> tuple[float, list[float]]:
    """L and the coefficients of p, highest degree first (Horner order), by the published program in double."""
    m = 2 * n
    k = np.arange(-m + 1, m, dtype=np.float64)
    L = np.sqrt(n / np.sqrt(2.0))
    t = L * np.tan(k * np.pi / m / 2)
    f = np.concatenate([[0.0], np.exp(-t ** 2) * (L ** 2 + t ** 2)])
    a = np.real(np.fft.fft(np.fft.fftshift(f))) / (2 * m)
    return float(L), [float(v) for v in np.flipud(a[1:n + 1])]


def rybicki() -> list[D]:
    h = D(1) / D(4)
    return [(-(((2 * i + 1) * h) ** 2)).exp() for i in range(13)]


def legendre8() -> list[tuple[D, D]]:
    """Positive nodes of P_8 (Newton from the Chebyshev guesses) and their weights, ascending."""
    P = pi()
    out = []
    for i in range(1, 5):
        x = cos(P * (D(i) - D(1) / D(4)) / (D(8) + D(1) / D(2)))
        for _ in range(100):
            p0, p1 = D(1), x
            for k in range(2, 9):
                p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
            dp = 8 * (x * p1 - p0) / (x * x - 1)
            dx = p1 / dp
            x -= dx
            if abs(dx) < D(10) ** -55:
                break
        p0, p1 = D(1), x
        for k in range(2, 9):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        dp = 8 * (x * p1 - p0) / (x * x - 1)
        w = D(2) / ((1 - x * x) * dp * dp)
        out.append((x, w))
    return sorted(out)


def constants() -> dict:
    L, p24 = weideman(24)
    P = pi()
    gl = []
    for xi, w in legendre8():
        xd = float(xi)
        # (0.5 -+ 0.5 xi) formed in double from the double node, then cast to float
        gl.append((float(np.float32(0.5 - 0.5 * xd)), float(np.float32(0.5 + 0.5 * xd)), to_f32(w / 2)))
    return {
        "weideman_L24": to_f32(L),
        "weideman_p24": [to_f32(c) for c in p24],
        "inv_sqrt_pi": to_f32(1 / P.sqrt()),
        "half_sqrt_pi": to_f32(P.sqrt() / 2),
        "rybicki": [to_f32(c) for c in rybicki()],
        "gl8": gl,
    }


def hexf(v: float) -> str:
    return float(v).hex().replace("0000000p", "p") + "f" if v != 0 else "0.0f"


if __name__ == "__main__":
    c = constants()
    for k, v in c.items():
        if isinstance(v, list):
            print(k, [hexf(x) if not isinstance(x, tuple) else tuple(hexf(y) for y in x) for x in v])
        else:
            print(k, hexf(v))
