"""NumPy model of the tile kernel's index arithmetic (test infrastructure).

It replays, element by element, what sip_b200/csrc/fft_tile.cu does for one
transform — the Stockham stage gather/scatter positions, the stage twiddle
index r*(j mod Ns)*tstep, the multi-pass load/store addressing with the
column-block jump, and the R2C/C2R pack twiddles — in complex128.  The CPU
tests compare it with the oracle so that an indexing mistake is caught
without a GPU.
"""
from __future__ import annotations

import numpy as np


def factor_radices(n: int) -> list[int]:
    """Same decomposition as planner.cpp factor_radices(): powers of two in balanced
    stages of <= 16, odd primes with pairs of 3 as 9, a single 3 or 5 merged into a
    power-of-two radix (12, 6, 10) when there is one."""
    m, twos = n, 0
    while m % 2 == 0:
        m //= 2
        twos += 1
    out = []
    if twos:
        s = (twos + 3) // 4
        base, extra = divmod(twos, s)
        out += [1 << (base + (1 if i < extra else 0)) for i in range(s)]
    odd = []
    for p in (13, 11, 7, 5):
        while m % p == 0:
            odd.append(p)
            m //= p
    while m % 9 == 0:
        odd.append(9)
        m //= 9
    if m % 3 == 0:  # a single 3 joins a radix 4 (-> 12) or 2 (-> 6)
        m //= 3
        for want in (4, 2):
            if want in out:
                out[out.index(want)] *= 3
                break
        else:
            odd.append(3)
    for i, r in enumerate(odd):  # a 5 joins a radix 2 (-> 10)
        if r == 5 and 2 in out:
            out[out.index(2)] = 10
            odd[i] = 1
    out += [r for r in odd if r > 1]
    if m != 1:
        raise ValueError(f"{n} has a prime factor above 13")
    return out


def table(denom: int, count: int, forward: bool, mult: int = 1) -> np.ndarray:
    m = (np.arange(count, dtype=np.int64) * mult) % denom
    w = np.exp(-2j * np.pi * m / denom)
    return w if forward else np.conj(w)


def dft_small(a: np.ndarray, forward: bool) -> np.ndarray:
    r = a.shape[-1]
    k = np.arange(r)
    w = np.exp((-2j if forward else 2j) * np.pi * np.outer(k, k) / r)
    return a @ w.T


def smem_fft(row: np.ndarray, forward: bool, tw: np.ndarray, tw_mul: int) -> np.ndarray:
    """Stockham stages exactly as stage_read/stage_write index them."""
    n = row.shape[0]
    x = row.astype(np.complex128).copy()
    ns = 1
    for r in factor_radices(n) if n > 1 else []:
        nbf = n // r
        tstep = (n // (ns * r)) * tw_mul
        j = np.arange(nbf)
        v = np.stack([x[j + q * nbf] for q in range(r)], axis=1)
        if ns > 1:
            step = (j % ns) * tstep
            for q in range(1, r):
                v[:, q] *= tw[q * step]
        v = dft_small(v, forward)
        k = j % ns
        base = (j - k) * r + k
        y = np.empty_like(x)
        for q in range(r):
            y[base + q * ns] = v[:, q]
        x = y
        ns *= r
    return x


def multipass(x: np.ndarray, passes: list[int], forward: bool) -> np.ndarray:
    """Multi-pass Stockham over HBM: pass p reads columns j (stride F/Rp),
    applies W_F^(r*(j mod Ns)*F/(Ns*Rp)), runs an Rp-point FFT and stores at
    j + (j//Ns)*Ns*(Rp-1) + r*Ns."""
    F = x.shape[0]
    wF = table(F, F, forward)
    cur = x.astype(np.complex128)
    ns = 1
    for rp in passes:
        cols = F // rp
        nxt = np.empty_like(cur)
        twr = table(rp, rp, forward)
        for c in range(cols):
            e = np.arange(rp)
            v = cur[c + e * cols]
            if ns > 1:
                v = v * wF[e * (c % ns) * (F // (ns * rp))]
            v = smem_fft(v, forward, twr, 1)
            nxt[c + (c // ns) * ns * (rp - 1) + e * ns] = v
        cur = nxt
        ns *= rp
    return cur


def r2c_packed(x: np.ndarray, forward: bool) -> np.ndarray:
    n = x.shape[0]
    m = n // 2
    tw = table(n, n, forward)
    z = smem_fft(x[0::2] + 1j * x[1::2], forward, tw, 2)
    out = np.empty(m + 1, np.complex128)
    for k in range(m // 2 + 1):
        zk = z[k]
        zm = np.conj(z[0 if k == 0 else m - k])
        e = 0.5 * (zk + zm)
        t = zk - zm
        od = -0.5j * t
        wo = tw[k] * od
        out[k] = e + wo
        if 2 * k != m:
            out[m - k] = np.conj(e - wo)
    return out


def c2r_packed(xh: np.ndarray, n: int, forward: bool) -> np.ndarray:
    m = n // 2
    tw = table(n, n, forward)
    z = np.empty(m, np.complex128)
    for k in range(m // 2 + 1):
        xk, xm = xh[k], xh[m - k]
        if k == 0:
            xk, xm = xk.real + 0j, xm.real + 0j
        e = xk + np.conj(xm)
        od = (xk - np.conj(xm)) * tw[k]
        z[k] = e + 1j * od
        if k != 0 and 2 * k != m:
            z[m - k] = np.conj(e) + 1j * np.conj(od)
    y = smem_fft(z, forward, tw, 2)
    out = np.empty(n)
    out[0::2] = y.real
    out[1::2] = y.imag
    return out


def fused_c2r_first_stage(xh: np.ndarray, m: int, R: int, forward: bool) -> np.ndarray:
    """static_fft.cu FusedC2R::gather: thread `lane` (NBF/2 threads, NBF = m/R)
    owns butterflies j0 = lane and j1 = NBF - lane (lane 0: 0 and NBF/2) and
    builds their packed inputs Z[j + r NBF] pairwise; lane 0 runs the common
    loop with selected inputs and twiddles, then moves its results into
    butterfly order.  Returns Z (length m) assembled from every thread's
    registers."""
    nbf = m // R
    G = (R + 1) // 2
    w = np.exp((-1 if forward else 1) * 2j * np.pi * np.arange(m + 1) / (2 * m))

    def pair(xk, xm, tw):
        ev = xk + np.conj(xm)
        od = (xk - np.conj(xm)) * tw
        return ev + 1j * od, np.conj(ev) + 1j * np.conj(od)

    def lane0_slot(k):
        if k >= R:
            return k - R if k - R < G else k
        return G - 1 + k if k <= R - G else R - G + k

    Z = np.full(m, np.nan, dtype=complex)
    for lane in range(nbf // 2):
        z = lane == 0
        j0 = lane
        j1 = nbf // 2 if z else nbf - lane
        a0 = nbf // 2 if z else j0
        wa = w[a0]
        wb = 1.0 if z else wa
        u = [None] * (2 * R)
        for r in range(R):
            if r < G:
                e = a0 + r * nbf
                tw = wa if r == 0 else wa * w[r * nbf]
            else:
                p = r - G + 1
                e = p * nbf if z else j0 + r * nbf
                tw = wb * w[(p if z else r) * nbf]
            u[r], u[2 * R - 1 - r] = pair(xh[e], xh[m - e], tw)
        v = [u[lane0_slot(k)] if z else u[k] for k in range(2 * R)]
        if z:
            x0, xn = xh[0].real + 0j, xh[m].real + 0j
            v[0] = pair(x0, xn, 1.0)[0]
        for r in range(R):
            Z[j0 + r * nbf] = v[r]
            Z[j1 + r * nbf] = v[R + r]
    return Z


def fused_r2c_last_stage(Z: np.ndarray, R: int, forward: bool) -> np.ndarray:
    """static_fft.cu FusedR2C::run after the last stage's butterflies: the
    thread that owns butterflies j0, j1 = NBF - j0 (lane 0: 0, NBF/2) holds
    Z[j + r NBF] and writes the m+1 bins X[k] = S/2 + w^k U/2,
    X[m-k] = conj(S/2 - w^k U/2) through the common pair loop (lane 0 with
    its operands selected).  Returns X (length m + 1)."""
    m = len(Z)
    nbf = m // R
    G = (R + 1) // 2
    w = np.exp((-1 if forward else 1) * 2j * np.pi * np.arange(m + 1) / (2 * m))

    def pair(zk, zm, tw):
        s = zk + np.conj(zm)
        u = -1j * (zk - np.conj(zm))
        return s / 2 + tw * u / 2, np.conj(s / 2 - tw * u / 2)

    X = np.full(m + 1, np.nan, dtype=complex)
    for lane in range(nbf // 2):
        z = lane == 0
        j0 = lane
        j1 = nbf // 2 if z else nbf - lane
        v = [Z[j0 + r * nbf] for r in range(R)] + [Z[j1 + r * nbf] for r in range(R)]
        u = [None] * (2 * R)
        for r in range(R):
            if r < G:
                u[r] = v[R + r] if z else v[r]
                u[2 * R - 1 - r] = v[2 * R - 1 - r]
            else:
                p = r - G + 1
                u[r] = v[p] if z else v[r]
                u[2 * R - 1 - r] = v[R - p] if z else v[2 * R - 1 - r]
        a0 = nbf // 2 if z else j0
        wa = w[a0]
        wb = 1.0 if z else wa
        for r in range(R):
            if r < G:
                o1, o2 = a0 + r * nbf, j1 + (R - 1 - r) * nbf
                tw = wa if r == 0 else wa * w[r * nbf]
            else:
                p = r - G + 1
                o1 = p * nbf if z else j0 + r * nbf
                o2 = (R - p) * nbf if z else j1 + (R - 1 - r) * nbf
                tw = wb * w[(p if z else r) * nbf]
            X[o1], X[o2] = pair(u[r], u[2 * R - 1 - r], tw)
        if z:
            X[0], X[m] = pair(v[0], v[0], 1.0)
    return X
