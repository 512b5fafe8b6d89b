"""Model-based tuner of the register-resident FFT passes (csrc/fast.cuh).

For a line of N samples held by T lanes of E samples each, every radix stage
but the last ends with an exchange through the line's shared memory: each lane
stores its E outputs and loads the next stage's E inputs.  How many shared-memory
wavefronts those 8-byte accesses take depends on where sample p is placed.  This
module counts them with a model of the bank rule (one 128-byte wavefront per
half-warp request when the 16 lanes hit 16 distinct 8-byte bank pairs, one more
for every extra distinct word on the same pair; the counts agree with ncu's
shared-memory conflict counters on the passes they were checked on) and picks,
per exchange, the placement p ^ (((p >> a) * m) & mask) that needs the fewest,
among those that permute 0 .. N-1.  It also ranks orders of the radix stages by
the same count.  The placements it prints are the XSw<...> lists in
csrc/fast_<N>.cu; tests/test_fft_tuning.py checks that they agree.

    python -m pyfwix_b200.tune_fft            # every plan's placements
    python -m pyfwix_b200.tune_fft 384 12     # radix orders of one (N, E), ranked
"""
from __future__ import annotations

import sys


def wavefronts(addrs):
    """Wavefronts of one warp-wide 8-byte shared-memory access (addresses in
    8-byte words, one per lane)."""
    tot = 0
    for half in (addrs[:16], addrs[16:]):
        banks = {}
        for a in half:
            banks.setdefault(a % 16, set()).add(a)
        tot += max(len(v) for v in banks.values()) if banks else 0
    return tot


def exchanges(N, E, radices):
    """Per exchange (forward stages first, then the inverse's reversed order):
    (direction, stage, warp store address lists, warp load address lists, ideal
    wavefront count), addresses as (line of the warp, sample) pairs, following
    the stage loop of fast.cuh (stages / lpos)."""
    T = N // E
    out = []
    for rev in (False, True):
        rs = list(radices[::-1]) if rev else list(radices)
        spans = [1]
        for r in rs[:-1]:
            spans.append(spans[-1] * r)
        for S in range(len(rs) - 1):
            R, Ns, R2 = rs[S], spans[S], rs[S + 1]
            B = E // R
            stores = []
            for b in range(B):
                for r in range(R):
                    row = []
                    for lane in range(32):
                        g, t = lane // T, lane % T
                        j = t + T * b
                        row.append((g, (j // Ns) * Ns * R + (j % Ns) + r * Ns))
                    stores.append(row)
            loads = [[(lane // T, lane % T + T * (e // R2) + (e % R2) * (N // R2)) for lane in range(32)]
                     for e in range(E)]
            out.append(((rev, S), stores, loads, 2 * B * R + 2 * E))
    return out


def cost(ex, f, line):
    _, st, ld, _ = ex
    return sum(wavefronts([g * line + f(p) for g, p in row]) for row in st + ld)


def _xor_default(p):
    return p ^ ((p >> 3) & 15)


def placements(N):
    """Candidate placements: name -> (code, function), in a fixed order; only
    permutations of 0 .. N-1.  Code -1 is the default XOR placement, 0 the
    identity, else a | m << 4 | mask << 8."""
    fs = {"id": (0, lambda p: p)}
    for a in range(1, 8):
        for mask in (7, 15, 31):
            if N % (mask + 1):
                continue
            for m in (1, 3, 5, 7, 9, 11, 13, 15):
                f = (lambda a, m, mask: (lambda p: p ^ (((p >> a) * m) & mask)))(a, m, mask)
                if sorted(f(p) for p in range(N)) == list(range(N)):
                    fs[f"x{a}m{m}k{mask}"] = (a | m << 4 | mask << 8, f)
    return fs


def lines(N, E):
    """Line strides of the row and column passes (RowGeo / ColGeo LINE)."""
    T = N // E
    lx = 8 * (32 // T)
    return N + (8 if T < 32 else 0), N + (2 if lx == 8 else 5)


def best_placements(N, E, radices):
    """(codes, wavefronts, ideal): per exchange the placement with the fewest
    wavefronts summed over the row and the column line stride (ties to the
    identity, then to the default XOR placement)."""
    row, col = lines(N, E)
    fs = placements(N)
    codes, total, ideal = [], 0, 0
    for ex in exchanges(N, E, radices):
        name, (code, f) = min(fs.items(), key=lambda kv: (cost(ex, kv[1][1], row) + cost(ex, kv[1][1], col),
                                                          kv[0] != "id"))
        cb = cost(ex, f, row) + cost(ex, f, col)
        cx = cost(ex, _xor_default, row) + cost(ex, _xor_default, col)
        if cx <= cb:
            code, cb = -1, cx
        codes.append(code)
        total += cb
        ideal += 2 * ex[3]
    return codes, total, ideal


def radix_orders(N, E, allowed=(2, 3, 4, 5, 7, 8, 12, 16, 20)):
    """Stage radix sequences of product N whose radices divide E, fewest stages
    first, largest radix first within a stage count."""
    cands = [r for r in allowed if E % r == 0]
    found = set()

    def rec(rest, seq):
        if rest == 1:
            found.add(tuple(seq))
            return
        if len(seq) >= 6:
            return
        for r in cands:
            if rest % r == 0:
                rec(rest // r, seq + [r])

    rec(N, [])
    return sorted(found, key=lambda s: (len(s), [-r for r in s]))


def code_text(c):
    if c < 1:
        return str(c)
    return f"fwix::fast::xs({c & 15}, {(c >> 4) & 15}, {c >> 8})"


# (N, E, radices) of the plans with their own exchange placements (csrc/fast_<N>.cu;
# for 256 the column plan: the rows place samples at p + (p >> 4) instead)
PLANS = {96: (12, (12, 4, 2)), 128: (8, (8, 4, 4)), 160: (20, (20, 4, 2)), 192: (12, (12, 4, 4)),
         256: (16, (16, 16)), 320: (20, (20, 4, 4)), 384: (12, (12, 4, 4, 2)), 512: (16, (8, 8, 8)),
         640: (20, (20, 4, 4, 2)), 64: (8, (8, 8))}


def main(argv):
    if len(argv) >= 2:
        N, E = int(argv[0]), int(argv[1])
        rows = []
        for rad in radix_orders(N, E)[:12]:
            codes, tot, ideal = best_placements(N, E, rad)
            rows.append((len(rad), tot, rad, ideal))
        for ns, tot, rad, ideal in sorted(rows):
            print(f"{N} E={E} radices {rad}: {ns} stages, exchange wavefronts {tot} (conflict-free {ideal})")
        return
    for N, (E, rad) in sorted(PLANS.items()):
        codes, tot, ideal = best_placements(N, E, rad)
        xs = ", ".join(code_text(c) for c in codes)
        print(f"{N:4d} E={E:2d} {rad}: wavefronts {tot} (conflict-free {ideal})  XSw<{xs}>")


if __name__ == "__main__":
    main(sys.argv[1:])
