"""Independent numpy restatement of the reference's OpenCL stereo kernels (test infrastructure).

Follows src/main/java/sgm/GpuStereo.java:706-769 (``costs``, ``paths``, ``winners``) and the host
``select`` (GpuStereo.java:631-687) in the resident, unstreamed configuration.  Structure differs
on purpose from the C oracle (which follows the CPU loops of CensusSgm.match): lines are processed
in vectorized batches and costs come from whole-volume array expressions.  The reference's own
regressions assert that its CPU and GPU implementations agree bit for bit; tests assert the same
of these two restatements.
"""
from __future__ import annotations

import math

import numpy as np

DIRS = [(1, 0), (-1, 0), (0, 1), (0, -1), (1, 1), (-1, 1), (1, -1), (-1, -1)]


def costs(a_words, b_words, ta, tb, ga, gb, w, h, D, md, reverse, rx, ry, mode, weight, adcap,
          gradcap, wx, wy):
    """``costs`` kernel: uint16 volume [n][D], 512 = invalid."""
    n = w * h
    ys, xs = np.divmod(np.arange(n), w)
    ks = np.arange(D)
    disp = md + ks
    target = xs[:, None] + (disp[None, :] if reverse else -disp[None, :])
    inside = ((xs >= rx) & (xs < w - rx) & (ys >= ry) & (ys < h - ry) & (ta != 0))[:, None]
    valid = inside & (target >= rx) & (target < w - rx)
    q = ys[:, None] * w + np.clip(target, 0, w - 1)
    valid &= tb[q] != 0
    p = np.broadcast_to(np.arange(n)[:, None], (n, D))
    ham = np.zeros((n, D), np.int64)
    for j in range(a_words.shape[0]):
        ham += np.bitwise_count(a_words[j][p] ^ b_words[j][q]).astype(np.int64)
    value = ham.copy()
    bits = wx * wy - 1
    gai, gbi = ga.astype(np.int64), gb.astype(np.int64)
    if mode in (1, 2):
        if mode == 1:
            difference = np.abs(gai[p] - gbi[q])
            cap = adcap
        else:
            pp, qq = np.clip(p, w + 1, n - w - 2), np.clip(q, w + 1, n - w - 2)
            ax = gai[pp + 1] - gai[pp - 1]
            ay = gai[pp + w] - gai[pp - w]
            bx = gbi[qq + 1] - gbi[qq - 1]
            by = gbi[qq + w] - gbi[qq - w]
            difference = np.abs(ax - bx) + np.abs(ay - by)
            cap = gradcap
        den = 1000 * cap
        value = (weight * ham * cap + (1000 - weight) * np.minimum(difference, cap) * bits
                 + den // 2) // den
    if mode == 3:
        count = wx * wy
        sa = np.zeros((n, D), np.int64)
        sb, saa, sbb, sab = sa.copy(), sa.copy(), sa.copy(), sa.copy()
        pc = np.clip(p, 0, n - 1)
        for dy in range(-ry, ry + 1):
            for dx in range(-rx, rx + 1):
                off = dy * w + dx
                av = gai[np.clip(pc + off, 0, n - 1)]
                bv = gbi[np.clip(q + off, 0, n - 1)]
                sa += av
                sb += bv
                saa += av * av
                sbb += bv * bv
                sab += av * bv
        va = count * saa - sa * sa
        vb = count * sbb - sb * sb
        with np.errstate(invalid="ignore", divide="ignore"):
            corr = (count * sab - sa * sb).astype(np.float64) / np.sqrt(
                va.astype(np.float64) * vb.astype(np.float64))
            z = np.floor((1 - np.fmax(-1.0, np.fmin(1.0, corr))) * .5 * bits + .5)
        value = np.where((va <= 0) | (vb <= 0), 512, np.nan_to_num(z, nan=512).astype(np.int64))
    return np.where(valid, value, 512).astype(np.int64)


def paths(cost, valid, gray, w, h, D, directions, p1, p2, edge_scale, sum_bytes):
    """``paths`` kernel over every direction, resident mode: returns the aggregate (int64)."""
    C = cost.reshape(h, w, D)
    S = np.zeros((h, w, D), np.int64)
    vmask = valid.reshape(h, w) != 0
    g = gray.reshape(h, w).astype(np.int64)
    big = np.int64(2**40)

    def step(prev_vals, has, cur_cost, gcur, gprev):
        # prev_vals [..., D]; has [...]
        minimum = np.where(has, prev_vals.min(axis=-1), 0)
        lp2 = np.full(has.shape, p2, np.int64)
        if edge_scale > 0:
            diff = np.abs(gcur - gprev)
            lp2 = np.where(has, np.maximum(p1 + 1, (p2 * edge_scale) // (edge_scale + diff)), p2)
        t = np.minimum(prev_vals, (minimum + lp2)[..., None])
        dn = np.concatenate([np.full(prev_vals.shape[:-1] + (1,), big), prev_vals[..., :-1] + p1], -1)
        up = np.concatenate([prev_vals[..., 1:] + p1, np.full(prev_vals.shape[:-1] + (1,), big)], -1)
        t = np.minimum(np.minimum(t, dn), up)
        return np.where(has[..., None], cur_cost + t - minimum[..., None], cur_cost)

    for dx, dy in DIRS[:directions]:
        L = np.zeros((h, w, D), np.int64)
        if dy == 0:
            xs = range(w) if dx > 0 else range(w - 1, -1, -1)
            for x in xs:
                px = x - dx
                if 0 <= px < w:
                    has = vmask[:, px]
                    L[:, x] = step(L[:, px], has, C[:, x], g[:, x], g[:, px])
                else:
                    L[:, x] = C[:, x]
        else:
            ys = range(h) if dy > 0 else range(h - 1, -1, -1)
            for y in ys:
                py = y - dy
                if not 0 <= py < h:
                    L[y] = C[y]
                    continue
                px = np.arange(w) - dx
                inb = (px >= 0) & (px < w)
                pxc = np.clip(px, 0, w - 1)
                has = inb & vmask[py, pxc]
                L[y] = step(L[py, pxc], has, C[y], g[y], g[py, pxc])
        S += L
        if sum_bytes == 2:
            S &= 0xFFFF  # ushort SUM storage in the kernel
    return S.reshape(h * w, D)


def winners(cost, S, w, h, D, rx, ry):
    """``winners`` kernel: int32 [n][6]."""
    n = w * h
    out = np.zeros((n, 6), np.int64)
    out[:, 0] = -1
    out[:, 1] = 2**31 - 1
    out[:, 2] = 2**31 - 1
    out[:, 3] = -1
    out[:, 4] = -1
    ys, xs = np.divmod(np.arange(n), w)
    region = (xs >= rx) & (xs < w - rx) & (ys >= ry) & (ys < h - ry)
    validc = cost != 512
    key = np.where(validc, S, np.int64(2**40))
    best = key.argmin(axis=1)
    has = region & validc.any(axis=1)
    ks = np.arange(D)
    far = np.abs(ks[None, :] - best[:, None]) > 1
    second = np.where(far & validc, S, np.int64(2**31 - 1)).min(axis=1)
    rows = np.arange(n)
    bm = np.clip(best - 1, 0, D - 1)
    bp = np.clip(best + 1, 0, D - 1)
    before = np.where((best > 0) & validc[rows, bm], S[rows, bm], -1)
    after = np.where((best + 1 < D) & validc[rows, bp], S[rows, bp], -1)
    out[has, 0] = best[has]
    out[has, 1] = S[rows, best][has]
    out[has, 2] = second[has]
    out[has, 3] = before[has]
    out[has, 4] = after[has]
    out[:, 5] = (cost[:, 0] != 512).astype(np.int64) | ((cost[:, D - 1] != 512).astype(np.int64) << 1)
    return out


def select(summary, D, md, uniqueness):
    """Host ``select`` (GpuStereo.java:644-686): float disparities and the six counters."""
    n = summary.shape[0]
    result = np.full(n, np.nan, np.float32)
    st = dict(full=0, boundary=0, lower=0, upper=0, ambiguous=0, selected=0)
    for j in range(n):
        best, value, second, before, after, flags = (int(v) for v in summary[j])
        if best < 0:
            continue
        full = flags == 3
        if full:
            st["full"] += 1
        if best == 0 or best == D - 1:
            st["boundary"] += 1
            if full and best == 0:
                st["lower"] += 1
            if full and best == D - 1:
                st["upper"] += 1
            continue
        if second != 2**31 - 1 and float(second - value) <= max(1.0, value * uniqueness):
            st["ambiguous"] += 1
            continue
        offset = 0.0
        if before >= 0 and after >= 0:
            curvature = float(before) + after - 2.0 * value
            if curvature > 0:
                offset = max(-.5, min(.5, .5 * (before - float(after)) / curvature))
        result[j] = np.float32(md + best + offset)
        st["selected"] += 1
    return result, st


def match(prm, a, b, ga, gb, ta, tb, w, h, reverse):
    """One view through the four kernel stages; returns (cost, S, summary, disp, stats)."""
    words = a.size // (w * h)
    A = a.reshape(words, w * h)
    B = b.reshape(words, w * h)
    rx, ry = prm.window_x // 2, prm.window_y // 2
    cost = costs(A, B, ta, tb, ga, gb, w, h, prm.disparities, prm.min_disparity, reverse, rx, ry,
                 prm.cost_mode, prm.census_weight_milli, prm.ad_truncation,
                 prm.gradient_truncation, prm.window_x, prm.window_y)
    S = paths(cost, ta, ga, w, h, prm.disparities, prm.directions, prm.p1, prm.p2,
              prm.edge_scale, prm.aggregate_bytes)
    summary = winners(cost, S, w, h, prm.disparities, rx, ry)
    disp, st = select(summary, prm.disparities, prm.min_disparity, prm.uniqueness)
    return cost, S, summary, disp, st
