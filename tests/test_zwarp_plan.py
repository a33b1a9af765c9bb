"""The index arithmetic of the warp-resident z-row transforms (``zwarp.cuh``),
restated on the CPU: the exchange slots, the middle-stage butterfly tables
(read from the header), the twiddle table layout and the post-processing
partner of every supported half length H = Nz/2.  For each H the three-stage
plan (two stages at H = 32) of every lane is run with numpy on one row and
compared with numpy's FFT, and every exchange access of a half warp is
checked to hit 16 distinct 8-byte bank pairs -- the property the kernels'
shared-memory throughput rests on.  No GPU is needed."""

import os
import re

import numpy as np
import pytest

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "3dhit_b200", "csrc", "zwarp.cuh")
TWN = 2048


def _table(name):
    src = open(HDR).read()
    body = re.search(name + r"\[64\] = \{([^}]*)\}", src).group(1)
    return [int(x) for x in body.replace("\n", " ").split(",") if x.strip()]


def slot(H, p):
    return p + (p >> 3) if H <= 64 else p + (p >> 4)


class Plan:
    def __init__(self, H):
        self.H = H
        self.LPR = H // 8
        self.ROWS = 256 // H if H <= 256 else 1
        self.R1 = H // 64
        self.NB0 = H // 8
        self.XS = H + H // 8 if H <= 64 else H + H // 16
        self.LR = 4 if H == 32 else 8
        self.LP = H // self.LR
        self.TW2 = (self.R1 - 1) * 8 if self.R1 > 1 else 0
        self.TWZ = self.TW2 + (self.LR - 1) * self.LP
        tw = np.exp(-2j * np.pi * np.arange(TWN) / TWN)
        n = (self.TWZ + H + 1 + 1) // 2 * 2
        self.tws = np.zeros(n, complex)
        for e in range(n):  # zw_fill_twiddles
            m = 0
            if e < self.TW2:
                r, k = e // 8 + 1, e % 8
                m = r * k * (TWN // (8 * self.R1))
            elif e < self.TWZ:
                r, k = (e - self.TW2) // self.LP + 1, (e - self.TW2) % self.LP
                m = r * k * (TWN // H)
            elif e - self.TWZ <= H:
                m = (e - self.TWZ) * (TWN // (2 * H))
            self.tws[e] = tw[m]
        self.t256 = _table("kZwMid256")
        self.t512 = _table("kZwMid512")

    def mid(self, b):
        """ZwMid: (k, ld, st) of the lane's middle-stage butterflies."""
        C1 = 8 // self.R1 if self.R1 > 1 else 1
        out = []
        for i in range(C1):
            if self.H == 256:
                b1 = self.t256[32 * i + b]
            elif self.H == 512:
                b1 = self.t512[b]
            else:
                b1 = b + self.LPR * i
            k = b1 & 7
            out.append((b1, k, slot(self.H, b1), slot(self.H, (b1 - k) * self.R1 + k)))
        return out


def dft(v, inv):
    R = len(v)
    s = 1 if inv else -1
    n = np.arange(R)
    return np.exp(s * 2j * np.pi * np.outer(n, n) / R) @ v


def run_plan(P, x, inv, log):
    """One row's transform as the lanes of zw_transform compute it; `log`
    collects (phase, lane, slot) of every exchange access."""
    H, L = P.H, P.LPR
    xch = np.full(P.XS, np.nan, complex)
    v = {b: dft(np.array([x[b + P.NB0 * r] for r in range(8)]), inv) for b in range(L)}
    for b in range(L):
        for r in range(8):
            s = slot(H, 8 * b + r)
            log.append(("st0", b, r, s))
            xch[s] = v[b][r]
    out = np.zeros(H, complex)
    if H == 32:
        for b in range(L):
            vv = [None] * 8
            for h in range(2):
                u = np.array([xch[slot(H, b + 4 * h + 8 * r)] for r in range(4)])
                for r in range(4):
                    log.append(("ld1", b, 4 * h + r, slot(H, b + 4 * h + 8 * r)))
                for r in range(1, 4):
                    w = P.tws[P.TW2 + (r - 1) * P.LP + b + 4 * h]
                    u[r] *= np.conj(w) if inv else w
                u = dft(u, inv)
                for r in range(4):
                    vv[h + 2 * r] = u[r]
            for r in range(8):
                out[b + P.NB0 * r] = vv[r]
        return out
    if P.R1 > 1:
        NB1 = H // P.R1
        xch2 = np.full(P.XS, np.nan, complex)
        for b in range(L):
            for i, (b1, k, ld, st) in enumerate(P.mid(b)):
                u = np.array([xch[ld + slot(H, NB1 * r)] for r in range(P.R1)])
                for r in range(P.R1):
                    assert ld + slot(H, NB1 * r) == slot(H, b1 + NB1 * r)  # additive offsets
                    log.append((f"ldm{i}", b, r, ld + slot(H, NB1 * r)))
                for r in range(1, P.R1):
                    w = P.tws[(r - 1) * 8 + k]
                    u[r] *= np.conj(w) if inv else w
                u = dft(u, inv)
                for r in range(P.R1):
                    s = st + slot(H, 8 * r)
                    assert s == slot(H, (b1 - k) * P.R1 + k + 8 * r)
                    log.append((f"stm{i}", b, r, s))
                    xch2[s] = u[r]
        xch = xch2
    for b in range(L):
        u = np.array([xch[slot(H, b + P.NB0 * r)] for r in range(8)])
        for r in range(8):
            log.append(("ld2", b, r, slot(H, b + P.NB0 * r)))
        assert not np.isnan(u).any()
        for r in range(1, 8):
            w = P.tws[P.TW2 + (r - 1) * P.NB0 + b]
            u[r] *= np.conj(w) if inv else w
        u = dft(u, inv)
        for r in range(8):
            out[b + P.NB0 * r] = u[r]
    return out


@pytest.mark.parametrize("H", [32, 64, 128, 256, 512])
def test_plan_matches_numpy_fft(H):
    P = Plan(H)
    rng = np.random.default_rng(H)
    x = rng.standard_normal(H) + 1j * rng.standard_normal(H)
    for inv in (False, True):
        y = run_plan(P, x, inv, [])
        ref = np.fft.ifft(x) * H if inv else np.fft.fft(x)
        assert np.abs(y - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("H", [32, 64, 128, 256, 512])
def test_exchange_accesses_are_bank_conflict_free(H):
    """Per phase and value index, the 16 lanes of every half warp (rows of a
    warp sit XS slots apart; at H = 512 the row's 64 lanes are the team's two
    warps) touch 16 distinct 8-byte bank pairs (slot mod 16).  The one
    exception is the middle stage's stores at H = 128: under the p + p/16
    padding their bank pairs (b1 % 8 + b1 / 8) mod 16 take only 15 values over
    the 64 butterflies, so no assignment of butterflies to lanes makes them
    conflict-free; they are at worst two-way."""
    P = Plan(H)
    log = []
    run_plan(P, np.ones(H, complex), False, log)
    per = {}
    for ph, b, r, s in log:
        per.setdefault((ph, r), {})[b] = s
    lanes = 32 if H <= 256 else 64
    for (ph, r), slots in per.items():
        for hw in range(lanes // 16):
            pairs = set()
            for t in range(16 * hw, 16 * hw + 16):
                q, b = (t // P.LPR, t % P.LPR) if H <= 256 else (0, t)
                pairs.add((q * P.XS + slots[b]) % 16)
            if H == 128 and ph.startswith("stm"):
                hits = [(q * P.XS + slots[b]) % 16 for t in range(16 * hw, 16 * hw + 16)
                        for q, b in [(t // P.LPR, t % P.LPR)]]
                assert max(hits.count(x) for x in hits) <= 2, (H, ph, r, hw)
                continue
            assert len(pairs) == 16, (H, ph, r, hw, sorted(pairs))


@pytest.mark.parametrize("H", [32, 64, 128, 256, 512])
def test_tables_and_post_processing_partner(H):
    P = Plan(H)
    if H in (256, 512):
        t = P.t256 if H == 256 else P.t512
        assert sorted(t) == list(range(64))  # every middle butterfly exactly once
    # r2c post-processing: Z[H - k] of k = b + (H/8) r sits with lane (LPR - b)
    # mod LPR as its value 7 - r (b = 0: the lane's own value (8 - r) mod 8)
    for b in range(P.LPR):
        for r in range(8):
            k = b + P.NB0 * r
            pb = (P.LPR - b) & (P.LPR - 1)
            kk = P.NB0 * ((8 - r) & 7) if b == 0 else pb + P.NB0 * (7 - r)
            assert kk == (H - k) % H
    # twiddle tables: the last stage's w_H^{r k} and e^{-2 pi i k / 2H}
    for e in range(P.TW2, P.TWZ):
        r, k = (e - P.TW2) // P.LP + 1, (e - P.TW2) % P.LP
        assert np.isclose(P.tws[e], np.exp(-2j * np.pi * r * k / H))
    for k in range(H + 1):
        assert np.isclose(P.tws[P.TWZ + k], np.exp(-2j * np.pi * k / (2 * H)))
