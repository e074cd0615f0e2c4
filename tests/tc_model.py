"""NumPy model of the tensor-core FFT kernel (sip_b200/csrc/tc_fft.cu), test infrastructure.

It replays one tile of tc_fft_kernel: the four-step split n = N1 * N2, the
real 2x2 expansion of the complex DFT matrices, the K-major operand layout
(tc_desc.cuh umma_offset), the hi/lo split in FP16 (with the per-tile
power-of-two scale) or BF16, the three products hi*hi + hi*lo + lo*hi, the
inner twiddles W_n^(k1 n2) and the transposed hand-off between the stages.
The CPU tests compare it with the oracle (error of each precision form) and
check that every shared-memory and tensor-memory index stays inside the
regions the kernel reserves.
"""
from __future__ import annotations

import numpy as np

CONFIGS = {256: (16, 16, 8), 1024: (32, 32, 4), 2048: (64, 32, 2), 4096: (64, 64, 1)}
SMEM_LIMIT = 227 * 1024
TMEM_COLS = 128


def umma_offset(row, k, K):
    return (row >> 3) * (K * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2


def round_sig(v: np.ndarray, bits: int) -> np.ndarray:
    """Round to `bits` significant bits, ties to even (BF16: 8)."""
    m, e = np.frexp(v)
    return np.ldexp(np.round(m * (1 << bits)) / (1 << bits), e)


def to_fmt(v: np.ndarray, fmt: int) -> np.ndarray:
    v = np.asarray(v, np.float64)
    if fmt == 0:
        return v.astype(np.float16).astype(np.float64)
    return round_sig(v, 8)


def split(v: np.ndarray, fmt: int, src32: bool = True):
    """hi = fmt(v), lo = fmt(v - hi); src32: v is an FP32 value (kernel operands)."""
    if src32:
        v = np.asarray(v, np.float32).astype(np.float64)
        hi = to_fmt(v, fmt)
        lo = to_fmt((v - hi).astype(np.float32), fmt)
    else:
        hi = to_fmt(v, fmt)
        lo = to_fmt(v - hi, fmt)
    return hi, lo


def range_scale(maxabs: float, fmt: int) -> float:
    if fmt != 0 or not (maxabs > 0) or not np.isfinite(maxabs):
        return 1.0
    _, e = np.frexp(maxabs)
    return float(np.ldexp(1.0, 14 - int(e)))


def dft_matrix(N: int, forward: bool, fmt: int):
    """128 x 2N real matrix (rows m = 2k + co, cols 2n + ci) split hi/lo, as tc_matrix_kernel builds it."""
    K = 2 * N
    a = np.zeros((128, K))
    k = np.arange(N)[:, None]
    n = np.arange(N)[None, :]
    th = 2 * np.pi * ((k * n) % N) / N
    c, s = np.cos(th), np.sin(th)
    wi = -s if forward else s
    a[0:2 * N:2, 0::2] = c
    a[0:2 * N:2, 1::2] = -wi
    a[1:2 * N:2, 0::2] = wi
    a[1:2 * N:2, 1::2] = c
    return split(a, fmt, src32=False)


def smem_layout(n: int):
    """Offsets of the kernel's shared-memory regions (TcShape)."""
    N1, N2, TB = CONFIGS[n]
    KA, KB, CA, CB, M = 2 * N1, 2 * N2, TB * N2, TB * N1, 128
    pitch = ((n - 1) + ((n - 1) >> 4) + 1) | 1
    a_bytes, b_bytes = M * KA * 2, M * KB * 2
    u1 = max(KA * CA * 2 * 2, TB * n * 8)
    u2 = max(TB * pitch * 8, KB * CB * 2 * 2)
    off_aa = 128
    off_ab = off_aa + 2 * a_bytes
    off_u1 = off_ab + 2 * b_bytes
    off_u2 = off_u1 + (u1 + 127) // 128 * 128
    total = off_u2 + (u2 + 127) // 128 * 128
    return dict(N1=N1, N2=N2, TB=TB, KA=KA, KB=KB, CA=CA, CB=CB, pitch=pitch, a_bytes=a_bytes, b_bytes=b_bytes,
                U1=u1, U2=u2, off_aa=off_aa, off_ab=off_ab, off_u1=off_u1, off_u2=off_u2, total=total)


def pad(i):
    return i + (i >> 4)


def check_bounds(n: int) -> None:
    """Every index the kernel forms stays inside its region; raises AssertionError otherwise."""
    L = smem_layout(n)
    N1, N2, TB, KA, KB, CA, CB = (L[k] for k in ("N1", "N2", "TB", "KA", "KB", "CA", "CB"))
    assert L["total"] <= SMEM_LIMIT
    assert CA <= TMEM_COLS and CB <= TMEM_COLS and CA % 16 == 0 and CB % 16 == 0
    assert 2 * N1 <= 128 and 2 * N2 <= 128
    # X tile (float2) in U2: t * pitch + pad(e)
    t = np.arange(TB)[:, None]
    e = np.arange(n)[None, :]
    xi = t * L["pitch"] + pad(e)
    assert xi.max() * 8 + 8 <= L["U2"] and xi.min() >= 0
    # stage-A operand (hi then lo) in U1: rows j < CA, k < KA
    j = np.arange(CA)[:, None]
    kk = np.arange(0, KA, 8)[None, :]
    off = umma_offset(j, kk, KA)
    assert off.max() + 16 + KA * CA * 2 <= L["U1"]
    # MMA reads of the B operand: 3 passes, K blocks of 16 -> last byte of the last core matrix
    last = umma_offset(CA - 1, KA - 1, KA) + 2
    assert last <= KA * CA * 2
    last = umma_offset(127, KA - 1, KA) + 2
    assert last <= L["a_bytes"]
    # Y (float) in U1: ((t*N2 + n2)*N1 + k1)*2 + c
    assert ((TB - 1) * N2 + N2 - 1) * N1 * 2 + (N1 - 1) * 2 + 1 < L["U1"] // 4
    # stage-B operand in U2
    j = np.arange(CB)[:, None]
    kk = np.arange(0, KB, 8)[None, :]
    off = umma_offset(j, kk, KB)
    assert off.max() + 16 + KB * CB * 2 <= L["U2"]
    assert umma_offset(127, KB - 1, KB) + 2 <= L["b_bytes"]
    # inner twiddle index k1 * n2 < n
    assert (N1 - 1) * (N2 - 1) < n


def tc_tile(x: np.ndarray, forward: bool, fmt: int) -> np.ndarray:
    """One tile (TB transforms of length n, complex) through the kernel's arithmetic."""
    n = x.shape[-1]
    N1, N2, TB = CONFIGS[n]
    x = np.asarray(x, np.complex64).reshape(-1, n)
    ntr = x.shape[0]
    assert ntr <= TB
    xs = np.zeros((TB, n), np.complex64)
    xs[:ntr] = x
    a_hi, a_lo = dft_matrix(N1, forward, fmt)
    b_hi, b_lo = dft_matrix(N2, forward, fmt)
    # stage A
    s1 = range_scale(float(np.max(np.abs(np.concatenate([xs.real.ravel(), xs.imag.ravel()])))), fmt)
    v = xs.reshape(TB, N1, N2)  # [t][n1][n2]
    B = np.empty((TB, N2, 2 * N1), np.float32)  # row j = (t, n2), k = 2 n1 + ci
    B[:, :, 0::2] = (v.real * np.float32(s1)).transpose(0, 2, 1)
    B[:, :, 1::2] = (v.imag * np.float32(s1)).transpose(0, 2, 1)
    B = B.reshape(TB * N2, 2 * N1)
    bh, bl = split(B, fmt)
    D = (a_hi @ bh.T + a_hi @ bl.T + a_lo @ bh.T).astype(np.float32)  # FP32 accumulator, rows m, cols j
    D = D / np.float32(s1)
    z = (D[0:2 * N1:2] + 1j * D[1:2 * N1:2]).reshape(N1, TB, N2)  # [k1][t][n2]
    k1 = np.arange(N1)[:, None]
    n2 = np.arange(N2)[None, :]
    w = np.exp(-2j * np.pi * (k1 * n2) / n).astype(np.complex64)
    if not forward:
        w = np.conj(w)
    y = (z * w[:, None, :]).astype(np.complex64)  # Y[k1][t][n2]
    s2 = range_scale(float(np.max(np.abs(np.concatenate([y.real.ravel(), y.imag.ravel()])))), fmt)
    # stage B: row j' = (t, k1), k = 2 n2 + ci
    B2 = np.empty((TB, N1, 2 * N2), np.float32)
    B2[:, :, 0::2] = (y.real * np.float32(s2)).transpose(1, 0, 2)
    B2[:, :, 1::2] = (y.imag * np.float32(s2)).transpose(1, 0, 2)
    B2 = B2.reshape(TB * N1, 2 * N2)
    bh, bl = split(B2, fmt)
    D2 = (b_hi @ bh.T + b_hi @ bl.T + b_lo @ bh.T).astype(np.float32) / np.float32(s2)
    X = (D2[0:2 * N2:2] + 1j * D2[1:2 * N2:2]).reshape(N2, TB, N1)  # [k2][t][k1]
    out = X.transpose(1, 0, 2)  # [t][k2][k1] -> index k1 + N1 k2 needs [t][k2*N1 + k1]
    return out.reshape(TB, n)[:ntr].astype(np.complex64)


# ---------------------------------------------------------------------------- row pipeline (tc_rows.cu)
ROWS_CONFIGS = {1024: (32, 32, 4), 2048: (64, 32, 4), 4096: (64, 64, 2)}


def umma_offset_mn(m, k, sbo):
    return (m >> 3) * sbo + (k >> 3) * 128 + (k & 7) * 16 + (m & 7) * 2


def rows_layout(n: int):
    """TcRowShape of tc_rows.cu."""
    N1, N2, TB = ROWS_CONFIGS[n]
    KA, KB, RA, RB = 2 * N1, 2 * N2, TB * N2, TB * N1
    CHA, CHB = RA // 128, RB // 128
    DC = CHA * KA
    SBO_A, SBO_B = KA * 16 + 1024 // N2, KB * 16 + 1024 // N1
    A1, A2 = 16 * SBO_A, 16 * SBO_B
    FA, FB = KA * KA * 2, KB * KB * 2
    off_fa = 1024
    off_fb = off_fa + 2 * FA
    off_a1 = off_fb + (0 if N1 == N2 else 2 * FB)
    off_a2 = off_a1 + 2 * CHA * A1
    total = off_a2 + 2 * CHB * A2
    return dict(N1=N1, N2=N2, TB=TB, KA=KA, KB=KB, RA=RA, RB=RB, CHA=CHA, CHB=CHB, DC=DC, SBO_A=SBO_A,
                SBO_B=SBO_B, A1_CHUNK=A1, A2_CHUNK=A2, FA=FA, FB=FB, off_a1=off_a1, off_a2=off_a2, total=total,
                tmem_cols=4 * DC)


def check_rows_bounds(n: int) -> None:
    L = rows_layout(n)
    N1, N2, TB, KA, KB = L["N1"], L["N2"], L["TB"], L["KA"], L["KB"]
    assert L["RA"] % 128 == 0 and L["RB"] % 128 == 0
    assert L["CHA"] * KA == L["CHB"] * KB == L["DC"] and L["DC"] in (64, 128)
    assert L["tmem_cols"] <= 512 and L["total"] <= SMEM_LIMIT and L["total"] > 0
    # header (TcHeader: 12 x 8 + 4 + 4 + 16 + 64 bytes) fits before the matrices
    assert 12 * 8 + 8 + 16 + 64 <= 1024
    # loader: element pair (e, e+1), e even, of transform t -> rows r = t N2 + n2 (+1), K n1 and N1 + n1
    q = np.arange(TB * n // 2)
    t, e = q // (n // 2), 2 * (q % (n // 2))
    n1, n2 = e // N2, e % N2
    r = t * N2 + n2
    ch, m = r >> 7, r & 127
    assert ch.max() < L["CHA"]
    for k in (n1, N1 + n1):
        off = ch * L["A1_CHUNK"] + umma_offset_mn(m, k, L["SBO_A"])
        assert off.min() >= 0 and (off + 4).max() <= L["CHA"] * L["A1_CHUNK"]
        assert np.all((m & 7) % 2 == 0)  # 4-byte stores stay inside their 16-byte core-matrix row
    # stage-A epilogue: row r = ch*128 + m, 8 bins per 16 columns -> A2 rows t N1 + 8 c16 (8 rows), K n2 / N2 + n2
    for chn in range(L["CHA"]):
        mm = np.arange(128)
        rr = chn * 128 + mm
        tt, nn2 = rr // N2, rr % N2
        for c16 in range(KA // 16):
            r2 = tt * N1 + c16 * 8
            cb, m2 = r2 >> 7, r2 & 127
            assert cb.max() < L["CHB"] and np.all(m2 % 8 == 0)
            for k in (nn2, N2 + nn2):
                off = cb * L["A2_CHUNK"] + umma_offset_mn(m2, k, L["SBO_B"])
                assert (off + 16).max() <= L["CHB"] * L["A2_CHUNK"]
            assert (c16 * 8 + 7) * (N2 - 1) < n  # twiddle index k1 n2
    # MMA reads: last byte of a 128-row chunk, and of the DFT matrices
    assert umma_offset_mn(127, KA - 1, L["SBO_A"]) + 2 <= L["A1_CHUNK"]
    assert umma_offset_mn(127, KB - 1, L["SBO_B"]) + 2 <= L["A2_CHUNK"]
    assert umma_offset(KA - 1, KA - 1, KA) + 2 <= L["FA"]
    assert umma_offset(KB - 1, KB - 1, KB) + 2 <= L["FB"]
    # stage-B epilogue: rows t N1 + k1 -> output k1 + N1 k2 < n
    assert (N1 - 1) + N1 * (N2 - 1) < n


def tc_rows_tile(x: np.ndarray, forward: bool, fmt: int) -> np.ndarray:
    """One tile of tc_rows_kernel: tile-max scale before stage A (FP16), fixed 2^-(log2 N1 + 1) before stage B."""
    n = x.shape[-1]
    N1, N2, TB = ROWS_CONFIGS[n]
    x = np.asarray(x, np.complex64).reshape(-1, n)
    ntr = x.shape[0]
    xs = np.zeros((TB, n), np.complex64)
    xs[:ntr] = x
    s1 = range_scale(float(np.max(np.abs(np.concatenate([xs.real.ravel(), xs.imag.ravel()])))), fmt)
    sb = 1.0 / (2 * N1) if fmt == 0 else 1.0
    v = xs.reshape(TB, N1, N2)
    A = np.concatenate([(v.real * np.float32(s1)).transpose(0, 2, 1),
                        (v.imag * np.float32(s1)).transpose(0, 2, 1)], axis=2).reshape(TB * N2, 2 * N1)
    ah, al = split(A, fmt)
    fh, fl = dft_matrix(N1, forward, fmt)  # rows (k1, c), cols (n1, ci) interleaved
    # reorder the matrix columns to (ci, n1) blocks, as the B operand stores them
    perm = np.concatenate([np.arange(0, 2 * N1, 2), np.arange(1, 2 * N1, 2)])
    fh, fl = fh[:2 * N1][:, perm], fl[:2 * N1][:, perm]
    D = (ah @ fh.T + ah @ fl.T + al @ fh.T).astype(np.float32)  # rows (t, n2), cols (k1, c)
    z = (D[:, 0::2] + 1j * D[:, 1::2]).reshape(TB, N2, N1)  # [t][n2][k1]
    k1 = np.arange(N1)[None, :]
    n2 = np.arange(N2)[:, None]
    w = np.exp(-2j * np.pi * (k1 * n2) / n).astype(np.complex64)
    if not forward:
        w = np.conj(w)
    y = (z * w[None] * np.float32(sb)).astype(np.complex64)  # [t][n2][k1]
    B = np.concatenate([y.real.transpose(0, 2, 1), y.imag.transpose(0, 2, 1)], axis=2).reshape(TB * N1, 2 * N2)
    bh, bl = split(B, fmt)
    gh, gl = dft_matrix(N2, forward, fmt)
    perm2 = np.concatenate([np.arange(0, 2 * N2, 2), np.arange(1, 2 * N2, 2)])
    gh, gl = gh[:2 * N2][:, perm2], gl[:2 * N2][:, perm2]
    D2 = (bh @ gh.T + bh @ gl.T + bl @ gh.T).astype(np.float32) / np.float32(s1 * sb)  # rows (t, k1), cols (k2, c)
    X = (D2[:, 0::2] + 1j * D2[:, 1::2]).reshape(TB, N1, N2)  # [t][k1][k2] -> index k1 + N1 k2
    return X.transpose(0, 2, 1).reshape(TB, n)[:ntr].astype(np.complex64)


def tc_fft_rows(x: np.ndarray, forward: bool, fmt: int) -> np.ndarray:
    n = x.shape[-1]
    TB = ROWS_CONFIGS[n][2]
    x = np.asarray(x).reshape(-1, n)
    return np.concatenate([tc_rows_tile(x[i:i + TB], forward, fmt) for i in range(0, x.shape[0], TB)])


def tc_fft(x: np.ndarray, forward: bool, fmt: int) -> np.ndarray:
    n = x.shape[-1]
    TB = CONFIGS[n][2]
    x = np.asarray(x).reshape(-1, n)
    return np.concatenate([tc_tile(x[i:i + TB], forward, fmt) for i in range(0, x.shape[0], TB)])
