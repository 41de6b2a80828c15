"""CPU models of the index arithmetic and update orders the device kernels
rely on.  Each test restates a formula of a kernel in numpy / Python and
checks the property the kernel needs; the kernels themselves are checked on
the GPU against the oracle (test_gpu_*.py).

* oz_digit_kernel (imcom_b200/csrc/ozaki.cu): for 4 <= S <= 7 slices the
  balanced base-256 digits are taken from N = 2^24 H + L in 32-bit pieces;
  they must equal the 64-bit recursion of the CPU model (oracle/split_oracle.py).
* trd_panel_kernel (imcom_b200/csrc/eigen_dc.cu), phase A/B: the closed-form
  decode of the lower-triangle tiles visits every tile on or below the
  diagonal exactly once, and the per-row ranges of row and column partial
  sums in phase B add up to the trailing product A22 x.
* jacobi_kernel (imcom_b200/csrc/eigen_jacobi.cu): the round-robin rounds
  pair every two columns exactly once per sweep, each round with disjoint
  pairs.
* stacks_kernel (imcom_b200/csrc/solve.cu): every (column, stack) of H is
  written by exactly one lane, every read stays inside T and the stacks, and
  the zero-filled chunks sum to T^T I.
* trd_tail_kernel (imcom_b200/csrc/eigen_dc.cu): the distributed row layout
  and the lazy update order (column j's update applied to row j+1 before its
  reflector and to the other rows in the next pass) give a tridiagonal form
  Q^T A Q = T.
"""
import itertools
import math

import numpy as np
import pytest

# -- split digits ----------------------------------------------------------


def digits_64(N, S):
    d = [0] * S
    for s in range(S - 1, 0, -1):
        q = ((N + 128) & 255) - 128
        d[s] = q
        N = (N - q) >> 8
    d[0] = N
    return d


def digits_32(N, S):
    d = [0] * S
    c, hi = N & 0xFFFFFF, N >> 24
    for s in range(S - 1, 0, -1):
        if s >= S - 3:
            q = ((c + 128) & 255) - 128
            d[s] = q
            c = (c - q) >> 8
            if s == S - 3:
                hi += c
        else:
            q = ((hi + 128) & 255) - 128
            d[s] = q
            hi = (hi - q) >> 8
    d[0] = hi
    return d


@pytest.mark.parametrize("S", [4, 5, 6, 7])
def test_digit_split_matches_64bit_recursion(S):
    rng = np.random.default_rng(S)
    lim = 2 ** (7 + 8 * (S - 1) - 1)  # |N| < 2^(6 + 8(S-1)) for rows scaled below 1/2
    Ns = [int(v) for v in rng.integers(-lim, lim, 20000)]
    Ns += [lim - 1, -lim, 0, 1, -1, 2 ** 24, -(2 ** 24), 2 ** 24 - 1, 128, -128, 127, -129]
    for N in Ns:
        d = digits_32(N, S)
        assert d == digits_64(N, S)
        assert all(-128 <= x <= 127 for x in d[1:]) and abs(d[0]) <= 65


def test_digit_recursion_is_the_oracle_digits():
    from oracle import split_oracle as SO
    rng = np.random.default_rng(1)
    X = rng.standard_normal((6, 40)) * np.logspace(-3, 3, 40)
    for S in (4, 7):
        planes, scale = SO.digits(X, S)
        _, e = SO.row_scales(X)
        for r in range(X.shape[0]):
            for k in range(X.shape[1]):
                N = int(np.rint(np.ldexp(np.ldexp(X[r, k], -int(e[r])), 7 + 8 * (S - 1))))
                assert digits_32(N, S) == [int(p[r, k]) for p in planes]


# -- lower-triangle tiles of the panel kernel --------------------------------

CW, TR = 16, 64
CPB = TR // CW


def tile_geometry(n, j):
    rbase = (j + 1) & ~1
    R = n - (j + 1)
    RB = (n - rbase + TR - 1) // TR
    NC = (R + CW - 1) // CW
    rbc = min(RB, max(0, (NC - 1) // CPB))
    tri = CPB * rbc * (rbc + 1) // 2
    return rbase, RB, NC, rbc, tri, tri + (RB - rbc) * NC


def decode(tile, tri, rbc, NC):
    if tile < tri:
        q = int((math.sqrt(np.float32(1.0) + np.float32(8.0) * np.float32(tile) / CPB) - 1.0) * 0.5)
        while CPB * (q + 1) * (q + 2) // 2 <= tile:
            q += 1
        while q > 0 and CPB * q * (q + 1) // 2 > tile:
            q -= 1
        return q, tile - CPB * q * (q + 1) // 2
    return rbc + (tile - tri) // NC, (tile - tri) % NC


@pytest.mark.parametrize("n,j", [(40, 0), (41, 0), (100, 3), (130, 64), (257, 100), (300, 17),
                                 (199, 196), (70, 66), (640, 0), (1000, 1)])
def test_panel_tiles_cover_lower_triangle_and_sum_to_product(n, j):
    rng = np.random.default_rng(n + j)
    M = rng.standard_normal((n, n))
    A = M + M.T
    x = np.zeros(n)
    x[j + 1:] = rng.standard_normal(n - j - 1)
    rbase, RB, NC, rbc, tri, ntiles = tile_geometry(n, j)
    seen = set()
    ypart = np.full((NC, n), np.nan)
    ycol = np.full((RB, n), np.nan)
    for t in range(ntiles):
        rb, ch = decode(t, tri, rbc, NC)
        assert 0 <= rb < RB and 0 <= ch < NC and (rb, ch) not in seen
        seen.add((rb, ch))
        c0, c1 = j + 1 + ch * CW, min(n, j + 1 + ch * CW + CW)
        r0, r1 = rbase + rb * TR, min(n, rbase + rb * TR + TR)
        blk = A[r0:r1, c0:c1]
        rows = np.arange(r0, r1)[:, None]
        cols = np.arange(c0, c1)[None, :]
        low = np.where(rows >= cols, blk, 0.0)      # row sums: on or below the diagonal
        strict = np.where(rows > cols, blk, 0.0)    # column sums: strictly below
        rs = low @ x[c0:c1]
        keep = np.arange(r0, r1) >= j + 1
        ypart[ch, r0:r1][keep] = rs[keep]
        ycol[rb, c0:c1] = strict.T @ x[r0:r1]
    for rb in range(RB):
        for ch in range(NC):
            lower = rbase + rb * TR + TR - 1 >= j + 1 + ch * CW
            assert ((rb, ch) in seen) == lower
    y = np.zeros(n)
    for r in range(j + 1, n):
        ncr = min(NC, CPB * ((r - rbase) // TR + 1))
        rb0 = (r - (j + 1)) // CW // CPB
        parts = np.concatenate([ypart[:ncr, r], ycol[rb0:RB, r]])
        assert not np.isnan(parts).any()
        y[r] = parts.sum()
    ref = A[j + 1:, j + 1:] @ x[j + 1:]
    assert np.max(np.abs(y[j + 1:] - ref)) <= 1e-12 * max(1.0, np.max(np.abs(ref)))


# -- Jacobi round-robin ------------------------------------------------------


def jacobi_rounds(n):
    npl = n + (n & 1)
    m = npl - 1
    for s in range(m):
        pairs = []
        for k in range(npl // 2):
            p, q = (s, m) if k == 0 else ((s + k) % m, (s - k + m) % m)
            p, q = min(p, q), max(p, q)
            if q < n:
                pairs.append((p, q))
        yield pairs


@pytest.mark.parametrize("n", [2, 3, 7, 8, 31, 64, 112])
def test_jacobi_rounds_pair_every_two_columns_once(n):
    seen = []
    for pairs in jacobi_rounds(n):
        flat = [c for pq in pairs for c in pq]
        assert len(flat) == len(set(flat))
        seen += pairs
    assert sorted(seen) == sorted(itertools.combinations(range(n), 2))


# -- cluster tail ------------------------------------------------------------


def tail_lazy(A, ctas):
    n = A.shape[0]
    S, rpc = n, (n + ctas - 1) // ctas
    Lw = np.tril(A)  # only the lower triangle is valid in global memory
    rows = [np.full((max(0, min(rpc, S - q * rpc)), S), np.nan) for q in range(ctas)]
    for q in range(ctas):  # phase 1: row r right of the diagonal = column r of the lower part
        for i in range(rows[q].shape[0]):
            r = q * rpc + i
            rows[q][i, r:] = Lw[r:, r]
    for q in range(ctas):  # phase 2: left of the diagonal, from the owner of row c
        for i in range(rows[q].shape[0]):
            r = q * rpc + i
            for c in range(r):
                o = c // rpc
                rows[q][i, c] = rows[o][c - o * rpc, r]
    d, e, tau = np.zeros(n), np.zeros(n - 1), np.zeros(n - 1)
    V = np.zeros((n, n))
    vb, pb = [np.zeros(S), np.zeros(S)], [np.zeros(S), np.zeros(S)]
    a2 = 0.0
    for jl in range(S - 1):
        par = jl & 1
        vq, pq = vb[par ^ 1], pb[par ^ 1]
        o = jl // rpc
        row = rows[o][jl - o * rpc]
        if jl > 0:
            vr = vq[jl]
            wr = pq[jl] + a2 * vr
            row[jl:] -= vr * (pq[jl:] + a2 * vq[jl:]) + wr * vq[jl:]
        xn2 = np.sum(row[jl + 2:] ** 2)
        alpha = row[jl + 1]
        if xn2 == 0:
            t, beta, scl = 0.0, alpha, 0.0
        else:
            beta = -math.copysign(math.sqrt(alpha * alpha + xn2), alpha)
            t, scl = (beta - alpha) / beta, 1.0 / (alpha - beta)
        v = np.zeros(S)
        v[jl + 1] = 1.0
        v[jl + 2:] = row[jl + 2:] * scl
        V[:, jl], d[jl], e[jl], tau[jl] = v, row[jl], beta, t
        newp, ptv = np.zeros(S), 0.0
        for q in range(ctas):
            for i in range(rows[q].shape[0]):
                rr = q * rpc + i
                if rr <= jl:
                    continue
                R = rows[q][i]
                if jl > 0:
                    vr = vq[rr]
                    wr = pq[rr] + a2 * vr
                    R[jl:] -= vr * (pq[jl:] + a2 * vq[jl:]) + wr * vq[jl:]
                newp[rr] = t * (R[jl + 1:] @ v[jl + 1:])
                ptv += newp[rr] * v[rr]
        vb[par], pb[par] = v, newp
        a2 = -0.5 * t * ptv
    par = (S - 2) & 1
    vr = vb[par][S - 1]
    wr = pb[par][S - 1] + a2 * vr
    oq = (S - 1) // rpc
    d[S - 1] = rows[oq][S - 1 - oq * rpc][S - 1] - 2.0 * vr * wr
    return d, e, tau, V


@pytest.mark.parametrize("n,ctas", [(2, 16), (3, 16), (37, 16), (64, 8), (70, 16)])
def test_cluster_tail_order_tridiagonalises(n, ctas):
    rng = np.random.default_rng(n)
    M = rng.standard_normal((n, n))
    A = M + M.T
    d, e, tau, V = tail_lazy(A, ctas)
    Q = np.eye(n)
    for j in range(n - 1):
        Q = Q @ (np.eye(n) - tau[j] * np.outer(V[:, j], V[:, j]))
    T = np.diag(d) + np.diag(e, -1) + np.diag(e, 1)
    assert np.linalg.norm(Q.T @ A @ Q - T) <= 1e-13 * np.linalg.norm(A)


# -- many-stack streaming kernel ---------------------------------------------

STK_WARPS, STK_CPW, STK_KC = 4, 4, 128


def stacks_model(T, I, SG):
    """stacks_kernel (imcom_b200/csrc/solve.cu) restated loop for loop:
    returns H and the number of writes of each element."""
    n, m = T.shape
    S = I.shape[1]
    H = np.full((m, S), np.nan)
    writes = np.zeros((m, S), dtype=int)
    gx = (m + STK_WARPS * STK_CPW - 1) // (STK_WARPS * STK_CPW)
    gy = (S + SG - 1) // SG
    for by in range(gy):
        s0 = by * SG
        sg = min(SG, S - s0)
        assert sg >= 1
        for bx in range(gx):
            acc = np.zeros((STK_WARPS, 32, STK_CPW, SG))
            for k0 in range(0, n, STK_KC):
                Is = np.zeros(SG * STK_KC)
                for e in range(SG * STK_KC):
                    s, kk = divmod(e, STK_KC)
                    k = k0 + kk
                    if s < sg and k < n:
                        Is[e] = I[k, s0 + s]
                for w in range(STK_WARPS):
                    a0 = (bx * STK_WARPS + w) * STK_CPW
                    for lane in range(32):
                        for j in range(STK_KC // 32):
                            k = k0 + lane + 32 * j
                            kk = lane + 32 * j
                            for c in range(STK_CPW):
                                t = T[k, a0 + c] if (a0 + c < m and k < n) else 0.0
                                for s in range(SG):
                                    acc[w, lane, c, s] += t * Is[s * STK_KC + kk]
            for w in range(STK_WARPS):
                a0 = (bx * STK_WARPS + w) * STK_CPW
                tot = acc[w].sum(axis=0)  # the butterfly leaves the sum in every lane
                for lane in range(32):
                    for c in range(STK_CPW):
                        for s in range(SG):
                            if (c * SG + s) % 32 == lane and a0 + c < m and s < sg:
                                H[a0 + c, s0 + s] = tot[c, s]
                                writes[a0 + c, s0 + s] += 1
    return H, writes


@pytest.mark.parametrize("n,m,S,SG", [(1, 1, 1, 1), (130, 17, 3, 4), (257, 33, 8, 8),
                                      (100, 16, 19, 8), (64, 5, 2, 2)])
def test_stacks_kernel_covers_each_output_once(n, m, S, SG):
    rng = np.random.default_rng(n * m + S)
    T = rng.standard_normal((n, m))
    I = rng.standard_normal((n, S))
    H, writes = stacks_model(T, I, SG)
    assert np.all(writes == 1)
    assert np.allclose(H, T.T @ I, rtol=1e-13, atol=1e-13)


def test_stacks_launch_choice():
    """The launch picks 1, 2, 4 or 8 stacks per pass: one pass up to 8
    stacks, ceil(S / 8) passes (grid rows) beyond."""
    def sg(S):
        return 1 if S == 1 else 2 if S == 2 else 4 if S <= 4 else 8
    for S in range(1, 70):
        g, passes = sg(S), -(-S // sg(S))
        assert g in (1, 2, 4, 8) and g * passes >= S
        assert passes == (1 if S <= 8 else -(-S // 8))


# -- fused, pruned table FFT ---------------------------------------------------


def fft_radices(L):
    """The factorisation table_fft.cu uses: fours first, then 2, 3, 5, 7, 11, 13."""
    out = []
    while L % 4 == 0:
        out.append(4)
        L //= 4
    for r in (2, 3, 5, 7, 11, 13):
        while L % r == 0:
            out.append(r)
            L //= r
    return out if L == 1 else None


def stockham(x, tw):
    """One line of the kernel's in-place Stockham stages (sign +, natural
    order out): per stage of radix R and span Ns, butterfly j reads
    x[j + r L/R], twiddles by tw[k r L/(Ns R)] (k = j mod Ns), and writes
    x[(j div Ns) Ns R + k + r Ns]."""
    L = len(x)
    Ns = 1
    for R in fft_radices(L):
        per = L // R
        v = [[x[j + r * per] for r in range(R)] for j in range(per)]  # all reads first
        for j in range(per):
            k = j % Ns
            vv = [v[j][0]] + [v[j][r] * tw[k * r * (L // (Ns * R))] for r in range(1, R)]
            base = (j // Ns) * Ns * R + k
            for r in range(R):
                x[base + r * Ns] = sum(vv[s] * tw[((r * s) % R) * (L // R)] for s in range(R))
        Ns *= R
    return x


def cshift_src(i1, s, n):
    return 1 + ((i1 - 1 + s) % n + n) % n


def table_model(Gt, Gammat, pairs, nps, L, isB):
    """table_fft.cu's two passes: pass 1 transforms the nps non-zero lines
    of the embedded grid along p into W (nps x L per table); pass 2
    scatters W's columns into zero lines along q, transforms them and
    writes the shifted, scaled real table."""
    s = L // 2
    nmin = (L - nps) // 2 + 1
    tw = np.exp(2j * np.pi * np.arange(L) / L)
    tabs = []
    for pr in pairs:
        W = np.zeros((nps, L), complex)
        for u in range(nps):
            sj = cshift_src(u + 1, nps // 2, nps)
            line = np.zeros(L, complex)
            for p0 in range(L):
                sp = cshift_src(p0 + 1, s, L)
                if nmin <= sp < nmin + nps:
                    si = cshift_src(sp - nmin + 1, nps // 2, nps)
                    if pr[1] > 0:  # A: conj(Gt_e) Gt_f
                        a, b = Gt[si - 1, sj - 1, pr[0] - 1], Gt[si - 1, sj - 1, pr[1] - 1]
                    else:  # B: conj(Gammat) Gt_e
                        a, b = Gammat[si - 1, sj - 1], Gt[si - 1, sj - 1, pr[0] - 1]
                    line[p0] = np.conj(a) * b
            W[u] = stockham(line, tw)
        tab = np.full((L, L), np.nan)  # tab[p-1, q-1]
        for k1 in range(L):
            col = np.zeros(L, complex)
            for u in range(nps):
                q0 = (nmin + u - 1 - s) % L  # the line of grid row sq = nmin + u
                col[q0] = W[u, k1]
            F = stockham(col, tw)
            for k2 in range(L):
                v = F[k2].real
                if isB:
                    v = -2.0 * v
                tab[(k1 - s) % L, (k2 - s) % L] = v / nps / nps
        tabs.append(tab)
    return tabs


def table_reference(Gt, Gammat, pairs, nps, L, isB):
    """The cuFFT path restated: embed_kernel, an unnormalised inverse 2-D
    FFT, shift_scale_kernel."""
    s = L // 2
    nmin, nmax = (L - nps) // 2 + 1, (L + nps) // 2
    tabs = []
    for pr in pairs:
        grid = np.zeros((L, L), complex)  # grid[p-1, q-1]
        for q in range(1, L + 1):
            for p in range(1, L + 1):
                sp, sq = cshift_src(p, s, L), cshift_src(q, s, L)
                if nmin <= sp <= nmax and nmin <= sq <= nmax:
                    si = cshift_src(sp - nmin + 1, nps // 2, nps)
                    sj = cshift_src(sq - nmin + 1, nps // 2, nps)
                    if pr[1] > 0:
                        a, b = Gt[si - 1, sj - 1, pr[0] - 1], Gt[si - 1, sj - 1, pr[1] - 1]
                    else:
                        a, b = Gammat[si - 1, sj - 1], Gt[si - 1, sj - 1, pr[0] - 1]
                    grid[p - 1, q - 1] = np.conj(a) * b
        F = np.fft.ifft2(grid) * L * L
        tab = np.empty((L, L))
        for q in range(1, L + 1):
            for p in range(1, L + 1):
                v = F[cshift_src(p, s, L) - 1, cshift_src(q, s, L) - 1].real
                tab[p - 1, q - 1] = (-2.0 * v if isB else v) / nps / nps
        tabs.append(tab)
    return tabs


@pytest.mark.parametrize("nps,npad", [(2, 3), (4, 3), (6, 3), (10, 3), (4, 5), (6, 2)])
def test_pruned_table_fft_matches_embed_fft_shift(nps, npad):
    L = nps * npad
    if fft_radices(L) is None:
        pytest.skip("size outside the kernel's radices")
    rng = np.random.default_rng(nps * 10 + npad)
    E = 2
    Gt = rng.standard_normal((nps, nps, E)) + 1j * rng.standard_normal((nps, nps, E))
    Gammat = rng.standard_normal((nps, nps)) + 1j * rng.standard_normal((nps, nps))
    for isB, pairs in ((0, [(1, 1), (1, 2), (2, 2)]), (1, [(1, 0), (2, 0)])):
        got = table_model(Gt, Gammat, pairs, nps, L, isB)
        ref = table_reference(Gt, Gammat, pairs, nps, L, isB)
        for g, r in zip(got, ref):
            assert not np.isnan(g).any()
            assert np.max(np.abs(g - r)) <= 1e-12 * max(1.0, np.max(np.abs(r)))


def test_fft_radices_cover_the_workload_sides():
    assert fft_radices(1728) == [4, 4, 4, 3, 3, 3]  # nps 576 (n = 4096 workload)
    assert fft_radices(3 * 2 * 11) == [2, 3, 11]
    assert fft_radices(3 * 2 * 17) is None  # a factor 17: cuFFT keeps such sizes
    for L in range(1, 400):
        r = fft_radices(L)
        if r is not None:
            assert int(np.prod(r)) == L


@pytest.mark.parametrize("R", [3, 5, 7, 11, 13])
def test_symmetric_pair_dft_is_the_dft(R):
    """dft_store's odd radices: y_r, y_{R-r} = v_0 + sum_s a_s cos(2 pi r s/R)
    +- i sum_s b_s sin(2 pi r s/R), a_s = v_s + v_{R-s}, b_s = v_s - v_{R-s}."""
    rng = np.random.default_rng(R)
    v = rng.standard_normal(R) + 1j * rng.standard_normal(R)
    H = (R - 1) // 2
    a = {s: v[s] + v[R - s] for s in range(1, H + 1)}
    b = {s: v[s] - v[R - s] for s in range(1, H + 1)}
    y = np.empty(R, complex)
    y[0] = v[0] + sum(a.values())
    for r in range(1, H + 1):
        A = v[0] + sum(a[s] * np.cos(2 * np.pi * r * s / R) for s in a)
        B = sum(b[s] * np.sin(2 * np.pi * r * s / R) for s in b)
        y[r], y[R - r] = A + 1j * B, A - 1j * B
    assert np.allclose(y, np.fft.ifft(v) * R, atol=1e-13)


FFT_THREADS = 512
FFT_CAP = {4: 8192, 2: 8192, 3: 6144, 5: 5120, 7: 3584, 11: 5632, 13: 6656}


def fft_plan(L):
    """make_plan (table_fft.cu): odd line stride, lines per block from the
    smallest cap of the plan's radices."""
    r = fft_radices(L)
    LS = L + 1 if L % 2 == 0 else L
    if r is None or LS > 8192:
        return None
    cap = min([FFT_CAP[x] for x in r] + [8192])
    TP = min(8, cap // LS)
    return (LS, TP, r) if TP >= 1 else None


def test_fft_plan_keeps_every_stage_in_its_registers():
    for L in list(range(1, 700)) + [1728, 2304, 3456, 5120, 6144, 8190]:
        plan = fft_plan(L)
        if plan is None:
            continue
        LS, TP, radices = plan
        assert LS % 2 == 1 and LS >= L and TP * LS <= 8192
        for R in set(radices):
            JM = FFT_CAP[R] // (R * FFT_THREADS)
            assert JM * R * FFT_THREADS == FFT_CAP[R]
            assert TP * (L // R) <= JM * FFT_THREADS  # butterflies fit the register array
    assert fft_plan(1728)[:2] == (1729, 3)  # radix 3 caps the block at 6144 values


# -- learned-kappa band segments ------------------------------------------------


def band_segments(bidx):
    """band_segments_kernel (imcom_b200/csrc/kappa.cu) restated thread for
    thread: seg[k] = first p with bidx[p] >= k (seg[8] = n), seg[9] = 1 where
    the index decreases; returns seg and the writes of each seg[k]."""
    n = len(bidx)
    seg = [0] * 10
    writes = [0] * 9
    for p in range(n):
        b = int(bidx[p])
        prev = int(bidx[p - 1]) if p > 0 else -1
        if b < prev:
            seg[9] = 1
            continue
        for k in range(prev + 1, b + 1):
            seg[k] = p
            writes[k] += 1
        if p == n - 1:
            for k in range(b + 1, 9):
                seg[k] = n
                writes[k] += 1
    return seg, writes


def band_index(lam):
    lmax = lam[0]
    out = []
    for v in lam:
        r = v / lmax if (v > 0 and lmax > 0) else 0.0
        b = int(np.floor(-np.log10(r) * 0.5)) if r > 0 else 7
        out.append(min(max(b, 0), 7))
    return np.array(out)


@pytest.mark.parametrize("seed", range(6))
def test_band_segments_are_the_bands(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 300))
    lam = np.sort(10.0 ** rng.uniform(-18, 0, n))[::-1]
    if seed % 2:
        lam[-min(5, n):] = -np.abs(lam[-min(5, n):])  # tiny negative eigenvalues: band 7
    bidx = band_index(lam)
    assert np.all(np.diff(bidx) >= 0)  # descending eigenvalues give a monotone band index
    seg, writes = band_segments(bidx)
    assert seg[9] == 0 and writes == [1] * 9 and seg[8] == n
    P = rng.standard_normal(n)
    for b in range(8):
        assert np.array_equal(np.arange(seg[b], seg[b + 1]), np.nonzero(bidx == b)[0])
        assert np.isclose(np.sum(P[seg[b]:seg[b + 1]] ** 2), np.sum(P[bidx == b] ** 2))


def test_band_segments_flag_a_decreasing_index():
    seg, _ = band_segments(np.array([0, 0, 2, 1, 3]))
    assert seg[9] == 1
    seg, writes = band_segments(np.array([5]))
    assert seg[:9] == [0, 0, 0, 0, 0, 0, 1, 1, 1] and writes == [1] * 9


def dft_store(v, R, tw, L, y, base, Ns):
    """dft_store (table_fft.cu) as written: radix 2 and 4 butterflies, odd
    radices in the symmetric-pair form, outputs stored to y[base + r Ns]."""
    if R == 2:
        y[base], y[base + Ns] = v[0] + v[1], v[0] - v[1]
    elif R == 4:
        s0, d0, s1, d1 = v[0] + v[2], v[0] - v[2], v[1] + v[3], v[1] - v[3]
        y[base] = s0 + s1
        y[base + 2 * Ns] = s0 - s1
        y[base + Ns] = d0 + 1j * d1
        y[base + 3 * Ns] = d0 - 1j * d1
    else:
        H, step = (R - 1) // 2, L // R
        v = list(v)
        y0 = v[0]
        for s in range(1, H + 1):
            a, b = v[s] + v[R - s], v[s] - v[R - s]
            v[s], v[R - s] = a, b
            y0 += a
        y[base] = y0
        for r in range(1, H + 1):
            A, B = v[0], 0j
            for s in range(1, H + 1):
                w = tw[((r * s) % R) * step]
                A += v[s] * w.real
                B += v[R - s] * w.imag
            y[base + r * Ns] = A + 1j * B
            y[base + (R - r) * Ns] = A - 1j * B


def run_stages_block(buf, L, LS, TP, tw):
    """run_stages over a block's TP lines at stride LS: every butterfly's
    inputs are read before any output is written (the stage's barrier)."""
    Ns = 1
    for R in fft_radices(L):
        per = L // R
        B = TP * per
        v = [[buf[(b // per) * LS + (b % per) + r * per] for r in range(R)] for b in range(B)]
        tstep = L // (Ns * R)
        for b in range(B):
            line, j = divmod(b, per)
            k = j % Ns
            vv = [v[b][0]] + [v[b][r] * tw[k * r * tstep] if Ns > 1 else v[b][r]
                              for r in range(1, R)]
            dft_store(vv, R, tw, L, buf, line * LS + (j // Ns) * Ns * R + k, Ns)
        Ns *= R


def table_kernels(Gt, Gammat, pairs, nps, L, isB):
    """table_fft_pass1 and table_fft_pass2 emulated block by block with the
    plan's line stride and lines per block."""
    LS, TP, _ = fft_plan(L)
    s, nmin = L // 2, (L - nps) // 2 + 1
    tw = np.exp(2j * np.pi * np.arange(L) / L)
    W = np.full((len(pairs), nps, L), np.nan + 0j)
    tab = np.full((len(pairs), L * L), np.nan)
    for t, pr in enumerate(pairs):
        for bx in range(-(-nps // TP)):
            u0 = bx * TP
            buf = np.full(TP * LS, np.nan + 0j)
            for e in range(TP * L):
                line, p0 = divmod(e, L)
                u = u0 + line
                v = 0j
                if u < nps:
                    sp = cshift_src(p0 + 1, s, L)
                    if nmin <= sp < nmin + nps:
                        si = cshift_src(sp - nmin + 1, nps // 2, nps)
                        sj = cshift_src(u + 1, nps // 2, nps)
                        if pr[1] > 0:
                            a, b = Gt[si - 1, sj - 1, pr[0] - 1], Gt[si - 1, sj - 1, pr[1] - 1]
                        else:
                            a, b = Gammat[si - 1, sj - 1], Gt[si - 1, sj - 1, pr[0] - 1]
                        v = np.conj(a) * b
                buf[line * LS + p0] = v
            run_stages_block(buf, L, LS, TP, tw)
            for e in range(TP * L):
                line, k1 = divmod(e, L)
                if u0 + line < nps:
                    W[t, u0 + line, k1] = buf[line * LS + k1]
        for bx in range(-(-L // TP)):
            c0 = bx * TP
            buf = np.full(TP * LS, np.nan + 0j)
            for e in range(TP * L):
                line, q0 = divmod(e, L)
                buf[line * LS + q0] = 0j
            for e in range(nps * TP):
                u, c = divmod(e, TP)
                if c0 + c < L:
                    buf[c * LS + (nmin + u - 1 - s) % L] = W[t, u, c0 + c]
            run_stages_block(buf, L, LS, TP, tw)
            for e in range(TP * L):
                k2, c = divmod(e, TP)
                k1 = c0 + c
                if k1 < L:
                    v = buf[c * LS + k2].real
                    if isB:
                        v = -2.0 * v
                    tab[t, ((k2 - s) % L) * L + (k1 - s) % L] = v / nps / nps
    return [tt.reshape(L, L).T for tt in tab]  # tab[t][(q-1) L + (p-1)] as (p, q)


@pytest.mark.parametrize("nps,npad", [(2, 3), (4, 3), (10, 3), (14, 3), (4, 5), (6, 2),
                                      (22, 3), (26, 2)])
def test_table_kernels_as_written_match_embed_fft_shift(nps, npad):
    L = nps * npad
    if fft_plan(L) is None:
        pytest.skip("size outside the kernel's radices")
    rng = np.random.default_rng(nps + 100 * npad)
    E = 2
    Gt = rng.standard_normal((nps, nps, E)) + 1j * rng.standard_normal((nps, nps, E))
    Gammat = rng.standard_normal((nps, nps)) + 1j * rng.standard_normal((nps, nps))
    for isB, pairs in ((0, [(1, 1), (1, 2), (2, 2)]), (1, [(1, 0), (2, 0)])):
        got = table_kernels(Gt, Gammat, pairs, nps, L, isB)
        ref = table_reference(Gt, Gammat, pairs, nps, L, isB)
        for g, r in zip(got, ref):
            assert not np.isnan(g).any()
            assert np.max(np.abs(g - r)) <= 1e-12 * max(1.0, np.max(np.abs(r)))


# -- the PSF spectra's own real-to-complex transform ------------------------------


def r2c_kernels(images):
    """r2c_pass1 and r2c_pass2 (table_fft.cu) emulated block by block: the
    half spectra half[b][j][k] (k fastest, n/2 + 1 per row) of n x n real
    images stored x fastest."""
    count, n = images.shape[0], images.shape[1]
    LS, TP, _ = fft_plan(n)
    nh = n // 2 + 1
    tw = np.exp(2j * np.pi * np.arange(n) / n)
    src = [im.T.ravel() for im in images]  # element (k, j) at j n + k
    H = np.full((count, nh, n), np.nan + 0j)
    half = np.full((count, n, nh), np.nan + 0j)
    for b in range(count):
        for bx in range(-(-n // TP)):
            j0 = bx * TP
            buf = np.full(TP * LS, np.nan + 0j)
            for e in range(TP * n):
                line, k = divmod(e, n)
                j = j0 + line
                buf[line * LS + k] = src[b][j * n + k] if j < n else 0.0
            run_stages_block(buf, n, LS, TP, tw)
            for e in range(TP * nh):
                k, line = divmod(e, TP)
                if j0 + line < n:
                    H[b, k, j0 + line] = np.conj(buf[line * LS + k])
        for bx in range(-(-nh // TP)):
            k0 = bx * TP
            buf = np.full(TP * LS, np.nan + 0j)
            for e in range(TP * n):
                line, j = divmod(e, n)
                k = k0 + line
                buf[line * LS + j] = np.conj(H[b, k, j]) if k < nh else 0j
            run_stages_block(buf, n, LS, TP, tw)
            for e in range(TP * n):
                j, line = divmod(e, TP)
                if k0 + line < nh:
                    half[b, j, k0 + line] = np.conj(buf[line * LS + j])
    return half


@pytest.mark.parametrize("n", [4, 6, 12, 18, 20, 24, 28])
def test_r2c_kernels_as_written_match_rfft2(n):
    """The half spectrum imcom_ft_r2c keeps (FFTW's r2c: the first axis
    halved), as numpy's rfft along the first axis and fft along the second."""
    rng = np.random.default_rng(n)
    images = rng.standard_normal((2, n, n))  # images[b][x][y], x the first axis
    got = r2c_kernels(images)
    for b in range(2):
        ref = np.fft.fft(np.fft.rfft(images[b], axis=0), axis=1)  # (nh, n): [k][j]
        assert not np.isnan(got[b]).any()
        assert np.max(np.abs(got[b].T - ref)) <= 1e-12 * np.max(np.abs(ref))


# -- Lagrange weights of the PSF rotation ------------------------------------------


def lagrange_weights(t, x0, m):
    """lagrange_weights (tables.cu) as written: prefix/suffix products over
    16 slots and the integer denominators (-1)^(m-1-k) k! (m-1-k)!."""
    sv = [t - (x0 + j) if j < m else 1.0 for j in range(16)]
    node = any(j < m and sv[j] == 0.0 for j in range(16))
    pre, acc = [], 1.0
    for j in range(16):
        pre.append(acc)
        acc *= sv[j]
    w, acc = [0.0] * 16, 1.0
    for k in range(15, -1, -1):
        den = float(np.prod(np.arange(2, k + 1), dtype=float)) * float(
            np.prod(np.arange(2, m - k), dtype=float))
        if (m - 1 - k) % 2:
            den = -den
        w[k] = pre[k] * acc / den if k < m else 0.0
        acc *= sv[k]
    if node:
        w = [1.0 if (k < m and sv[k] == 0.0) else 0.0 for k in range(16)]
    return np.array(w)


@pytest.mark.parametrize("m", [1, 2, 5, 7, 8, 9, 16])
def test_lagrange_weights_reproduce_polynomials(m):
    """Weights on m consecutive integer nodes reproduce every polynomial of
    degree < m (so they interpolate as Neville's tableau does), also at a node."""
    rng = np.random.default_rng(m)
    x0 = 17
    nodes = x0 + np.arange(m)
    coef = rng.standard_normal(m)
    vals = np.polyval(coef, nodes - x0 - 0.5 * (m - 1))
    for t in [x0 + 0.37 * (m - 1), x0 + m - 1.0, x0 + 0.5, float(x0)]:
        w = lagrange_weights(t, x0, m)
        ref = np.polyval(coef, t - x0 - 0.5 * (m - 1))
        assert abs(w[:m] @ vals - ref) <= 1e-9 * max(1.0, np.abs(vals).max())
        assert np.all(w[m:] == 0.0)


# ---- seq_abs2_sum_kernel (tables.cu): the sequential sum by binades ----------

SQ_CHUNK, SQ_SUB = 4096, 32
TINY = 2.0 ** -1021


def seq_sum_by_binades(t):
    """The kernel's algorithm: per chunk of SQ_CHUNK terms, the rounded
    quotients rint(t / u) (u the running sum's ulp) of the whole chunk at
    once when the sum stays in its binade and no quotient is a tie; else per
    sub-chunk of SQ_SUB terms, adding term by term only where a sub-chunk
    crosses a binade or holds a tie (and recomputing the later quotients after
    a crossing)."""
    S, N = 0.0, len(t)
    for base in range(0, N, SQ_CHUNK):
        ch = np.zeros(SQ_CHUNK)
        part = t[base:base + SQ_CHUNK]
        ch[:len(part)] = part
        start = 0
        while True:
            normal = S >= TINY
            if normal:
                E = math.frexp(S)[1]
                x = np.ldexp(ch, 53 - E)
                q, tie = np.rint(x), (x - np.floor(x)) == 0.5
            else:
                E, q, tie = None, np.zeros(SQ_CHUNK), np.ones(SQ_CHUNK, bool)
            q[:start * SQ_SUB] = 0.0
            tie[:start * SQ_SUB] = False
            wq = q.reshape(-1, SQ_SUB).sum(1)
            wt = tie.reshape(-1, SQ_SUB).any(1)
            M = math.ldexp(S, 53 - E) if normal else 0.0
            if normal and not wt.any() and M + wq.sum() < 2.0 ** 53:
                S = math.ldexp(M + wq.sum(), E - 53)
                break
            restart, Sw, nw = None, S, normal
            for idx in range(start, SQ_CHUNK // SQ_SUB):
                if nw and not wt[idx] and M + wq[idx] < 2.0 ** 53:
                    M += wq[idx]
                    continue
                if nw:
                    Sw = math.ldexp(M, E - 53)
                for v in ch[idx * SQ_SUB:(idx + 1) * SQ_SUB]:
                    Sw = Sw + float(v)
                if Sw >= TINY:
                    E2 = math.frexp(Sw)[1]
                    if not nw or E2 != E:
                        if idx + 1 < SQ_CHUNK // SQ_SUB:
                            restart = idx + 1
                        nw = False
                        break
                    M = math.ldexp(Sw, 53 - E)
                else:
                    nw = False
            S = math.ldexp(M, E - 53) if nw else Sw
            if restart is None:
                break
            start = restart
    return S


def _sequential(t):
    s = 0.0
    for v in t.tolist():
        s = s + v
    return s


@pytest.mark.parametrize("case", ["spectrum", "lognormal", "half_ulp_ties", "zeros_first",
                                  "subnormal"])
def test_sum_by_binades_is_the_sequential_sum(case):
    """Bit-identical to the sequential loop of imcom_calc_C on |FFT|^2 terms,
    terms spanning 20 decades, exact half-ulp ties, leading zeros and sums
    that start subnormal."""
    rng = np.random.default_rng(11)
    if case == "spectrum":
        G = np.fft.fft2(rng.random((160, 160)) / 160 ** 2 * 4)
        t = (G.real * G.real + G.imag * G.imag).reshape(-1, order="F")
    elif case == "lognormal":
        t = np.exp(rng.normal(0.0, 8.0, 30000))
    elif case == "half_ulp_ties":
        t = np.full(20000, 2.0 ** -53)
        t[0] = 1.0
        t[100::7] = 3 * 2.0 ** -54
    elif case == "zeros_first":
        t = np.concatenate([np.zeros(5000), rng.random(9000)])
    else:
        t = rng.random(12000) * 1e-310
    assert seq_sum_by_binades(t) == _sequential(t)


# ---- the register path of the table FFT (table_fft.cu, fx_pass1/2) ---------

def _w(n, k):
    return np.exp(2j * np.pi * (np.asarray(k) % n) / n)


def _dft3p(a, b, c):
    t1, t2 = b + c, (b - c) * (1j * math.sqrt(3) / 2)
    m = a - 0.5 * t1
    return a + t1, m + t2, m - t2


def _dft9p(z):
    z = list(z)
    for r in range(3):
        z[r], z[r + 3], z[r + 6] = _dft3p(z[r], z[r + 3], z[r + 6])
    z[4] *= _w(9, 1); z[7] *= _w(9, 2); z[5] *= _w(9, 2); z[8] *= _w(9, 4)
    for s in range(3):
        z[3 * s], z[3 * s + 1], z[3 * s + 2] = _dft3p(z[3 * s], z[3 * s + 1], z[3 * s + 2])
    return z  # output s + 3 t at z[3 s + t]


def _dft576_warp(v):
    """dft576_warp as written: lane L holds v[32 n1 + L]; returns X."""
    reg = np.array([[v[32 * n1 + L] for n1 in range(18)] for L in range(32)])
    for L in range(32):
        e, o = _dft9p(reg[L][0::2]), _dft9p(reg[L][1::2])
        y = np.zeros(18, complex)
        for k in range(9):
            at = 3 * (k % 3) + k // 3
            t = o[at] * _w(18, k)
            y[k], y[k + 9] = e[at] + t, e[at] - t
        reg[L] = y * _w(576, L * np.arange(18))
    for h in (16, 8, 4, 2, 1):
        new = reg.copy()
        for L in range(32):
            upper = bool(L & h)
            r = (-1.0 if upper else 1.0) * reg[L] + reg[L ^ h]
            new[L] = r * (_w(2 * h, L % h) if upper else 1.0)
        reg = new
    X = np.zeros(576, complex)
    for L in range(32):
        j0 = 18 * int(f"{L:05b}"[::-1], 2)
        X[j0:j0 + 18] = reg[L]
    return X


def test_register_dft576_model():
    """The register path's line transform (DFT-18 per lane, lane twiddles,
    DFT-32 across lanes, output k1 + 18 bitrev5(lane)) and its k = 3 j + b
    split of the zero-padded length-1728 transform, against direct DFTs."""
    rng = np.random.default_rng(3)
    v = rng.standard_normal(576) + 1j * rng.standard_normal(576)
    n = np.arange(576)
    ref = np.array([np.sum(v * _w(576, n * k)) for k in range(576)])
    assert np.abs(_dft576_warp(v) - ref).max() <= 1e-15 * np.abs(ref).max() * 10
    m = np.where(n < 288, n, n - 576)
    F_ref = np.array([np.sum(v * _w(1728, m * k)) for k in range(1728)])
    F = np.zeros(1728, complex)
    for b in range(3):
        F[3 * n + b] = _dft576_warp(v * _w(1728, m * b))
    assert np.abs(F - F_ref).max() <= 1e-14 * np.abs(F_ref).max()


# ---- the deflation scan's parallel path (eigen_dc.cu, dc_deflate_kernel) ---

def _fma(a, b, c):
    """a b + c rounded once (the device fma)."""
    from fractions import Fraction
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def _deflate_scan(d, z, perm, rho, tol):
    """The sequential scan as written (LAPACK dlaed2's tests), returning the
    non-deflated (d, z, column), deflated (d, column) lists and rotations."""
    dl, dd, rot = [], [], 0
    have, dp, zp, pp = False, 0.0, 0.0, 0
    for dj, zj, pj in zip(d, z, perm):
        if rho * abs(zj) <= tol:
            dd.append((dj, pj))
            continue
        if not have:
            have, dp, zp, pp = True, dj, zj, pj
            continue
        t = dj - dp
        far = 4.0 * tol * _fma(zj, zj, zp * zp)
        rotate = False
        if not (far >= 2.2250738585072014e-308 and abs(t * zj * zp) > far):
            tau = math.hypot(zj, zp)
            c, s = zj / tau, -zp / tau
            rotate = abs(t * c * s) <= tol
        if rotate:
            rot += 1
            dd.append((dp * c * c + dj * s * s, pp))
            dp, zp, pp = dp * s * s + dj * c * c, tau, pj
        else:
            dl.append((dp, zp, pp))
            dp, zp, pp = dj, zj, pj
    if have:
        dl.append((dp, zp, pp))
    return dl, dd, rot


def _deflate_parallel(d, z, perm, rho, tol, threads=256):
    """The fast path as written: per-thread chunks, the cheap test against
    the raw previous entry, prefix offsets; None when a pair needs the scan."""
    nm = len(d)
    per = -(-nm // threads)
    chunks = [(min(nm, u * per), min(nm, u * per + per)) for u in range(threads)]
    zdef = [rho * abs(x) <= tol for x in z]
    prev = -1
    for a0, a1 in chunks:
        for q in range(a0, a1):
            if zdef[q]:
                continue
            if prev >= 0:
                far = 4.0 * tol * _fma(z[q], z[q], z[prev] * z[prev])
                if not (far >= 2.2250738585072014e-308 and abs((d[q] - d[prev]) * z[q] * z[prev]) > far):
                    return None
            prev = q
    dl = [(d[q], z[q], perm[q]) for q in range(nm) if not zdef[q]]
    dd = [(d[q], perm[q]) for q in range(nm) if zdef[q]]
    return dl, dd, 0


@pytest.mark.parametrize("seed", range(6))
def test_deflation_fast_path_is_the_scan(seed):
    """Wherever the parallel path applies it gives the scan's lists; it
    declines exactly when some pair needs the exact test."""
    rng = np.random.default_rng(seed)
    nm = int(rng.integers(1, 3000))
    d = np.sort(rng.standard_normal(nm) * 10.0 ** rng.integers(-2, 3))
    if seed % 2:  # clusters: some pairs close enough to rotate
        d[1::7] = d[0::7][: len(d[1::7])] + 1e-17
        d = np.sort(d)
    z = rng.standard_normal(nm)
    z[rng.random(nm) < 0.2] *= 1e-20  # z-deflated entries
    perm = rng.permutation(nm)
    rho = 1.3
    tol = 8.0 * 2.0 ** -53 * max(np.abs(d).max(), rho * np.abs(z).max())
    fast = _deflate_parallel(list(d), list(z), list(perm), rho, tol)
    slow = _deflate_scan(list(d), list(z), list(perm), rho, tol)
    if fast is not None:
        assert fast == slow
    else:
        assert seed % 2  # only the clustered cases need the scan


# ---- the trailing update's lower-tile enumeration (dgemm.cu) ---------------

def _lower_tile(b):
    """lower_update_kernel's (ti, tj) from the linear index b: a float32
    square root as the first guess, corrected by integer steps."""
    ti = int((np.sqrt(np.float32(8.0) * np.float32(b) + np.float32(1.0)) - np.float32(1.0))
             * np.float32(0.5))
    while (ti + 1) * (ti + 2) // 2 <= b:
        ti += 1
    while ti > 0 and ti * (ti + 1) // 2 > b:
        ti -= 1
    return ti, b - ti * (ti + 1) // 2


@pytest.mark.parametrize("nt", [1, 2, 3, 10, 64, 254, 700])
def test_lower_tiles_enumerate_the_lower_triangle(nt):
    """Linear indices 0 .. nt(nt+1)/2 - 1 map one to one onto the tiles
    (ti, tj) with tj <= ti < nt (nt = 254 is n = 16200 in 64-row tiles)."""
    tiles = [_lower_tile(b) for b in range(nt * (nt + 1) // 2)]
    assert len(set(tiles)) == len(tiles)
    assert all(0 <= tj <= ti < nt for ti, tj in tiles)


def test_persistent_tile_loops_cover_each_tile_once():
    """dgemm_persist_kernel and dc_gemm_kernel: CTA b takes tiles b, b + grid,
    ... of gm x gn x nkz (row blocks fastest); every tile exactly once."""
    for gm, gn, nkz, grid in [(32, 32, 1, 24), (2, 32, 9, 18), (5, 3, 1, 148), (1, 1, 4, 3)]:
        seen = []
        for b in range(grid):
            for tile in range(b, gm * gn * nkz, grid):
                xy = tile % (gm * gn)
                seen.append((xy % gm, xy // gm, tile // (gm * gn)))
        assert sorted(seen) == sorted((x, y, z) for z in range(nkz) for y in range(gn)
                                      for x in range(gm))


def table_register_model(Gt, Gammat, pairs, nps, isB):
    """fx_pass1/2's composition for npad = 3 (L = 3 nps): along each axis
    three length-nps transforms of copies pre-twiddled by exp(2 pi i m(u) b / L)
    (m(u) the signed frequency of spectrum index u) give outputs 3 j + b; W is
    kept as W[k1][u2]; pass 2 writes the real part through both cshifts."""
    L, s = 3 * nps, 3 * nps // 2
    u = np.arange(nps)
    m = np.where(u < nps // 2, u, u - nps)
    tabs = []
    for pr in pairs:
        if pr[1] > 0:
            X = np.conj(Gt[:, :, pr[0] - 1]) * Gt[:, :, pr[1] - 1]  # X[u1, u2]
        else:
            X = np.conj(Gammat) * Gt[:, :, pr[0] - 1]
        W = np.zeros((L, nps), complex)
        for b in range(3):
            tw = np.exp(2j * np.pi * ((m * b) % L) / L)
            W[3 * u + b, :] = np.fft.ifft(X * tw[:, None], axis=0) * nps
        tab = np.empty((L, L))
        p0 = (np.arange(L) - s) % L
        for b in range(3):
            tw = np.exp(2j * np.pi * ((m * b) % L) / L)
            v = (np.fft.ifft(W * tw[None, :], axis=1) * nps).real  # [k1][j]
            v = (-2.0 * v if isB else v) / nps / nps
            tab[np.ix_(p0, (3 * u + b - s) % L)] = v
        tabs.append(tab)
    return tabs


@pytest.mark.parametrize("nps", [4, 6, 12, 20])
def test_register_table_path_matches_embed_fft_shift(nps):
    """The register path's layout and shifts against the embed, FFT and
    shift of the cuFFT path (npad = 3; the kernels take nps = 576)."""
    rng = np.random.default_rng(nps)
    E = 2
    Gt = rng.standard_normal((nps, nps, E)) + 1j * rng.standard_normal((nps, nps, E))
    Gammat = rng.standard_normal((nps, nps)) + 1j * rng.standard_normal((nps, nps))
    for isB, pairs in ((0, [(1, 1), (1, 2), (2, 2)]), (1, [(1, 0), (2, 0)])):
        got = table_register_model(Gt, Gammat, pairs, nps, isB)
        ref = table_reference(Gt, Gammat, pairs, nps, 3 * nps, isB)
        for g, r in zip(got, ref):
            assert np.max(np.abs(g - r)) <= 1e-12 * max(1.0, np.max(np.abs(r)))
