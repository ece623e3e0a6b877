"""Coefficients of cos_turns (so_kerr.cuh; the oracle repeats them): a near-minimax polynomial of
degree 8 in z = g^2 for cos(2 pi g) on |g| <= 1/4 turn, from Chebyshev interpolation of
cos(2 pi sqrt(z)) on [0, 1/16] at 60-digit precision, printed as C hex-float literals (ascending
powers of z).  Run: python fit_cos_turns.py"""
import mpmath as mp

mp.mp.dps = 60
poly, err = mp.chebyfit(lambda z: mp.cos(2 * mp.pi * mp.sqrt(z)), [mp.mpf(0), mp.mpf(1) / 16], 9, error=True)
coef = [mp.mpf(c) for c in reversed(poly)]
# error of the double-rounded coefficients on a fine grid of g
worst = max(abs(sum(mp.mpf(float(c)) * (g * g) ** j for j, c in enumerate(coef)) - mp.cos(2 * mp.pi * g))
            for g in (mp.mpf(k) / 4096 / 4 for k in range(0, 4097)))
print(f"// max abs error: exact-coefficient fit {mp.nstr(err, 3)}, double coefficients {mp.nstr(worst, 3)}")
print("{" + ", ".join(float(c).hex() for c in coef) + "}")
