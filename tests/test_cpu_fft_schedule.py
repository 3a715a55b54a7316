"""The ring FFT pass schedule of csrc/rings.cu, checked on the CPU.

Restates `Radices` (small radix last in decimation-in-frequency order, the
first warp-local pass p0 = 1) and `for_butterflies` (CTA-wide passes:
thread t takes butterfly t >> lg of lane t & (lanes - 1), stepping by the
CTA size; warp-local passes: warp w takes the contiguous blocks
[w k, (w + 1) k) of 2^wl points of every lane), then checks for every
transform length and lane count a ring CTA can have:
  * every (butterfly, lane) of a pass runs exactly once;
  * a warp-local pass reads only points its own warp wrote in the pass
    before (or that a CTA-wide pass, ending in a CTA barrier, wrote), so
    warp barriers suffice between them -- in both the DIF order (synthesis,
    Bluestein forward) and the reverse DIT order (analysis, Bluestein
    inverse).
"""
import pytest

WARPS, THREADS, RADIX_LOG, BUFFER = 16, 512, 4, 8192


def radices(M):
    lgM = M.bit_length() - 1
    r0 = lgM % RADIX_LOG
    n = lgM // RADIX_LOG + (1 if r0 else 0)
    r = [(1 << r0) if (r0 and p == n - 1) else 16 for p in range(n)]
    lgl = [lgM - RADIX_LOG * p for p in range(n)]
    wl = [lgl[1] if (1 <= p < n) else 0 for p in range(n)]
    return n, r, lgl, wl


def butterflies(M, lg, R, lglen, wl):
    """(thread, butterfly, lane, points) of one pass."""
    LR = R.bit_length() - 1
    lq = lglen - LR
    gm = (1 << lg) - 1
    out = []

    def pts(b):
        j = b & ((1 << lq) - 1)
        base = ((b >> lq) << lglen) + j
        return [base + (i << lq) for i in range(R)]

    if wl == 0:
        nbf = (M >> LR) << lg
        for t in range(nbf):
            out.append((t % THREADS, t >> lg, t & gm, pts(t >> lg)))
    else:
        k = (M >> wl) // WARPS
        lp = wl - LR + lg
        for w in range(WARPS):
            for i in range(k << lp):
                B = w * k + (i >> lp)
                u = i & ((1 << lp) - 1)
                b = (B << (wl - LR)) + (u >> lg)
                out.append((w * 32 + (i % 32), b, u & gm, pts(b)))
    return out


def cases():
    for lgM in range(1, 14):
        M = 1 << lgM
        for lg in range(0, 5):
            if (M << lg) <= BUFFER:
                yield M, lg


@pytest.mark.parametrize("order", ["dif", "dit"])
def test_every_butterfly_once_and_warp_local_reads_own_writes(order):
    for M, lg in cases():
        n, r, lgl, wl = radices(M)
        assert sum(x.bit_length() - 1 for x in r) == M.bit_length() - 1
        seq = list(range(n)) if order == "dif" else list(range(n - 1, -1, -1))
        writer = {}  # (point, lane) -> warp of the last write, None after a CTA barrier
        for p in seq:
            bfs = butterflies(M, lg, r[p], lgl[p], wl[p])
            seen = {(b, g) for _, b, g, _ in bfs}
            assert len(seen) == len(bfs) == (M // r[p]) << lg, (M, lg, p)
            for thread, b, g, pts in bfs:
                w = thread // 32
                if wl[p]:
                    for x in pts:
                        prev = writer.get((x, g), None)
                        assert prev is None or prev == w, (M, lg, order, p, x, g, prev, w)
            new = {}
            for thread, b, g, pts in bfs:
                for x in pts:
                    new[(x, g)] = thread // 32 if wl[p] else None
            writer = new
            if wl[p] == 0:
                writer = {key: None for key in writer}


def test_warp_local_blocks_cover_the_cta_evenly():
    for M, lg in cases():
        n, r, lgl, wl = radices(M)
        for p in range(n):
            if wl[p]:
                assert (M >> wl[p]) % WARPS == 0 and (M >> wl[p]) >= WARPS
                assert lgl[p] <= wl[p]
