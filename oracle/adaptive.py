"""TEST INFRASTRUCTURE ONLY — numpy restatement of the reference's per-pixel
sample loop with adaptive stopping and NFOR accumulation.

Follows src/renderer/Threads.cpp of the Luz reference:
  cleanColor                 :122-137
  sampleLuminance            :139-148  (ColorManagement::luminance, ColorManagement.cpp:313-320)
  sampleMeanVariance         :150-161
  confidenceInterval95       :163-172
  channelConverged           :174-180
  darkMinimumSamples         :182-192
  adaptiveSampleConverged    :194-265
  adaptiveSamplingCanStop    :267-273
  addDenoiseFeatureSample    :274-290
  storeDenoisePixel          :343-372
  _threadRender              :551-641

It is fed per-sample path colours (and primary features) and reproduces the
stored pixel, the samples used and the NFOR buffers. Pixels are processed in
lockstep over samples with elementwise float64 numpy operations, so every sum
is the same IEEE sequence the reference forms one pixel at a time.
Only tests/ use it, as the checker.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

LUM = (0.2722287168, 0.6740817658, 0.0536895174)


def clean(c: np.ndarray) -> np.ndarray:
    return np.where(np.isfinite(c), c, 0.0)


def mean_variance(s, q, count: int):
    if count <= 1:
        return np.zeros_like(s)
    n = float(count)
    with np.errstate(all="ignore"):
        v = ((q - (s * s / n)) / (n - 1.0)) / n
    return np.where(0.0 < v, v, 0.0)          # std::max(0.0, v): NaN -> 0


def ci95(s, q, count: int):
    mv = mean_variance(s, q, count)
    with np.errstate(all="ignore"):
        return np.where(np.isfinite(mv), 1.96 * np.sqrt(mv), np.inf)


def channel_converged(mean, ci, threshold: float):
    am = np.abs(mean)
    with np.errstate(invalid="ignore"):
        target = threshold * np.where(am < 0.02, 0.02, am)
        return ci <= target


def dark_minimum(spp: int, min_s: int, interval: int) -> int:
    return min(spp, max(min_s, max(256, min_s + 3 * interval)))


def render_pixels(colors: np.ndarray, adaptive: Optional[dict] = None,
                  features: Optional[np.ndarray] = None):
    """colors: (P, S, 3) per-sample path colours (before cleanColor) in sample order;
    features: (P, S, 11) primary features or None (no denoise buffers).
    Returns rgb (P, 3), used (P,) and the NFOR buffers (dict) or None."""
    P, S, _ = colors.shape
    can_stop = bool(adaptive) and adaptive["min_samples"] < S
    min_s = min(adaptive["min_samples"], S) if adaptive else S
    interval = adaptive["check_interval"] if adaptive else 1
    thr = adaptive["threshold"] if adaptive else 1.0
    dark = dark_minimum(S, min_s, interval)

    csum = np.zeros((P, 3))
    csq = np.zeros((P, 3))
    lsum = np.zeros(P)
    lsq = np.zeros(P)
    lmax = np.zeros(P)
    nf = features is not None
    if nf:
        F = features.shape[2]
        ha_c, hb_c = np.zeros((P, 3)), np.zeros((P, 3))
        ha_n, hb_n = np.zeros(P, np.int64), np.zeros(P, np.int64)
        ha_f, hb_f = np.zeros((P, F)), np.zeros((P, F))
        fs, fq = np.zeros((P, F)), np.zeros((P, F))
    used = np.zeros(P, np.int64)
    active = np.ones(P, bool)
    for s in range(S):
        a = active
        c = clean(colors[a, s].astype(np.float64))
        if nf:
            f = features[a, s].astype(np.float64)
            if s % 2 == 0:
                ha_c[a] += c
                ha_n[a] += 1
                ha_f[a] += f
            else:
                hb_c[a] += c
                hb_n[a] += 1
                hb_f[a] += f
            fs[a] += f
            fq[a] += f * f
        csum[a] += c
        csq[a] += c * c
        lum = c[:, 0] * LUM[0] + c[:, 1] * LUM[1] + c[:, 2] * LUM[2]
        lum = np.where(np.isfinite(lum), lum, 0.0)
        lsum[a] += lum
        lsq[a] += lum * lum
        lmax[a] = np.where(lmax[a] < lum, lum, lmax[a])
        m = s + 1
        used[a] = m
        if m >= S:
            break
        if not can_stop or m < min_s or (m - min_s) % interval != 0 or m <= 1:
            continue
        n = float(m)
        idx = np.nonzero(a)[0]
        ok = ~((lmax[idx] < 0.02) & (m < dark))
        conv = ok & channel_converged(lsum[idx] / n, ci95(lsum[idx], lsq[idx], m), thr)
        for k in range(3):
            conv &= channel_converged(csum[idx, k] / n, ci95(csum[idx, k], csq[idx, k], m), thr)
        active[idx[conv]] = False
        if not active.any():
            break
    n = used.astype(np.float64)[:, None]
    rgb = clean(csum / n)
    bufs = None
    if nf:
        fb_c = csum / n
        fb_f = fs / n
        with np.errstate(all="ignore"):
            bufs = {
                "color_a": np.where(ha_n[:, None] > 0, ha_c / np.maximum(ha_n, 1)[:, None], fb_c),
                "color_b": np.where(hb_n[:, None] > 0, hb_c / np.maximum(hb_n, 1)[:, None], fb_c),
                "features_a": np.where(ha_n[:, None] > 0, ha_f / np.maximum(ha_n, 1)[:, None], fb_f),
                "features_b": np.where(hb_n[:, None] > 0, hb_f / np.maximum(hb_n, 1)[:, None], fb_f),
            }
        cv = np.zeros(P)
        fv = np.zeros((P, features.shape[2]))
        for u in np.unique(used):
            sel = used == u
            cv[sel] = (mean_variance(csum[sel, 0], csq[sel, 0], int(u)) + mean_variance(csum[sel, 1], csq[sel, 1], int(u))
                       + mean_variance(csum[sel, 2], csq[sel, 2], int(u))) / 3.0
            fv[sel] = mean_variance(fs[sel], fq[sel], int(u))
        bufs["color_variance"] = cv
        bufs["feature_variance"] = fv
    return rgb, used, bufs
