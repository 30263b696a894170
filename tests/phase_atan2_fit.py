"""Coefficients of ``phase_atan2`` (qssb_device.cuh): atan(t) = t P(t^2) on
[0, 1], P of degree 8 with P(0) = 1, fitted by iteratively reweighted least
squares towards the minimax (equal-ripple) error. Prints the float32
coefficients and the error of a float32 evaluation (fused multiply-adds
emulated in float64, rounded to float32 at every step) of the whole atan2
against numpy.arctan2.

    python tests/phase_atan2_fit.py
"""
import numpy as np

N_TERMS = 9


def fit(n_terms: int, iters: int = 60) -> np.ndarray:
    t = np.concatenate([np.cos(np.linspace(0, np.pi, 4000)) * 0.5 + 0.5, np.linspace(0, 1, 4000)])
    t = t[t > 1e-6]
    u = t * t
    f = np.arctan(t) / t - 1.0
    a = np.stack([u ** k for k in range(1, n_terms)], 1)
    w = np.ones_like(t)
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(a * w[:, None], f * w, rcond=None)
        err = np.abs(a @ c - f)
        w = w * (1 + 10 * err / err.max())
        w /= w.mean()
    return np.concatenate([[1.0], c]).astype(np.float32)


def f32(x):
    return np.asarray(x, np.float64).astype(np.float32)


def fma32(a, b, c):
    return f32(np.float64(a) * np.float64(b) + np.float64(c))


PIO2_HI, PIO2_LO = np.float32(1.5707963705062866), np.float32(-4.371139000186243e-08)
PI_HI, PI_LO = np.float32(3.1415927410125732), np.float32(-8.742278000372485e-08)


def phase_atan2_f32(y, x, c):
    y, x = f32(y), f32(x)
    ax, ay = np.abs(x), np.abs(y)
    mx, mn = np.maximum(ax, ay), np.minimum(ax, ay)
    with np.errstate(invalid="ignore", divide="ignore"):
        t = np.where(mx > 0, f32(mn / mx), np.float32(0))
    u = f32(t * t)
    p = np.full_like(u, c[-1])
    for k in range(len(c) - 2, -1, -1):
        p = fma32(p, u, c[k])
    r = f32(t * p)
    r = np.where(ay > ax, f32(f32(PIO2_HI - r) + PIO2_LO), r)
    r = np.where(np.signbit(x), f32(f32(PI_HI - r) + PI_LO), r)
    return np.copysign(r, y)


if __name__ == "__main__":
    c = fit(N_TERMS)
    print("coefficients:", ", ".join(f"{v:.9e}f" for v in c))
    rng = np.random.default_rng(0)
    y = rng.standard_normal(4_000_000) * 10.0 ** rng.uniform(-3, 6, 4_000_000)
    x = rng.standard_normal(4_000_000) * 10.0 ** rng.uniform(-3, 6, 4_000_000)
    err = np.abs(phase_atan2_f32(y, x, c).astype(np.float64) - np.arctan2(f32(y), f32(x)))
    print(f"max |error| {err.max():.3g} rad, rms {np.sqrt(np.mean(err ** 2)):.3g} rad")
