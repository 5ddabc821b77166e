"""CPU restatement of the reference's parallel M-series random-number
generator (test infrastructure: the checker of the device generator, never
part of the product path).

Follows, in the reference tree:
  RandomNumbers_Mseries::initset / delay3 / get
      src/lib/Tools/randomNumbers_Mseries.cpp:32-150, randomNumbers_Mseries.h:55-91
      (lagged XOR generator x_n = x_(n-521) ^ x_(n-32) on 31-bit words,
      output x_n * 2^-31, started by a polynomial jump of ndelay steps)
  RandomNumbers::gauss (Box-Muller, deviation 1/sqrt(2))
      src/lib/Tools/randomNumbers.cpp:53-75
  RandomNumbers_parallel<RandomNumbers_Mseries>::init_2d / set_lex_global_2d
      src/lib/Tools/randomNumbers_parallel-tmpl.h:160-252
      (one generator per (z, t) plane, seed (seed+1)*Lz*Lt + z + Lz*t, 1000
      discarded numbers, then per extra index j, per y, per x one block of
      Nin numbers from that plane's stream)
  get_gauss / get_uniform blocks
      src/lib/Tools/randomNumbers_parallel.h:102-145
      (uniform blocks hold one number: component 0 of a site, the rest 0)

Pinned against the reference corelib itself (tests/golden/mseries_parallel.npz,
made by tests/golden/make_golden.py through oracle/_ref/ref_harness rng).
"""
import math

import numpy as np

NP, NQ = 521, 32
FNORM = 4.656612870908988e-10
THERMALIZATION = 1000
SQ2R = 1.0 / math.sqrt(2.0)
PI2 = 2.0 * (4.0 * math.atan(1.0))


class Mseries:
    """One M-series stream (RandomNumbers_Mseries) started with ndelay."""

    def __init__(self, ndelay):
        self.w = np.zeros(NP, dtype=np.int64)
        self._initset(int(np.int32(np.int64(ndelay))))

    def _initset(self, ndelay):
        ib = np.zeros(NP, dtype=np.int64)
        ix = 1
        for i in range(NP):
            ix = (ix * 69069) & 0xFFFFFFFF
            ib[i] = ix >> 31
        jr, kr = 0, NP - NQ
        ibl = [int(v) for v in ib]
        w = []
        for _ in range(NP):
            iwork = 0
            for _ in range(32):
                iwork = ((iwork * 2) + ibl[jr]) & 0xFFFFFFFF
                ibl[jr] ^= ibl[kr]
                jr = jr + 1 if jr + 1 < NP else 0
                kr = kr + 1 if kr + 1 < NP else 0
            w.append(iwork >> 1)
        self.w = np.array(w, dtype=np.int64)
        self.jr, self.kr = jr, kr
        self._delay3(ndelay)

    def _delay3(self, ndelay):
        iwk = np.zeros(2 * NP - 1, dtype=np.int64)
        iwk[:NP] = self.w
        for i in range(NP, 2 * NP - 1):
            iwk[i] = iwk[i - NP] ^ iwk[i - NQ]
        mu = 40
        bits = [0] * mu
        m, nb = ndelay, mu - 1
        while m > NP - 1:
            nb += 1
            bits.append(m % 2)
            m //= 2
        c = np.zeros(2 * NP, dtype=np.int64)
        c[m] = 1
        for j in range(nb, -1, -1):
            b = bits[j]
            new = np.zeros(2 * NP, dtype=np.int64)
            new[2 * np.arange(NP) + b] = c[:NP]
            c = new
            for i in range(2 * NP - 1, NP - 1, -1):
                if c[i]:
                    c[i - NP] ^= 1
                    c[i - NQ] ^= 1
        sel = np.nonzero(c[:NP])[0]
        w = np.zeros(NP, dtype=np.int64)
        for j in range(NP):
            w[j] = np.bitwise_xor.reduce(iwk[j + sel]) if len(sel) else 0
        self.w = w

    def get(self):
        self.w[self.jr] ^= self.w[self.kr]
        r = float(self.w[self.jr]) * FNORM
        self.jr = self.jr + 1 if self.jr + 1 < NP else 0
        self.kr = self.kr + 1 if self.kr + 1 < NP else 0
        return r

    def gauss(self):
        r1, r2 = self.get(), self.get()
        slg = math.sqrt(-math.log(1.0 - r1) * 2.0) * SQ2R
        ang = PI2 * r2
        return slg * math.cos(ang), slg * math.sin(ang)


class MseriesParallel:
    """RandomNumbers_parallel<RandomNumbers_Mseries> on one process."""

    def __init__(self, lattice, seed):
        self.lattice = list(lattice)
        self.reset(seed)

    def reset(self, seed):
        lx, ly, lz, lt = self.lattice
        self.planes = []
        for t in range(lt):
            for z in range(lz):
                g = Mseries((seed + 1) * lz * lt + z + lz * t)
                for _ in range(THERMALIZATION):
                    g.get()
                self.planes.append(g)

    def _lex(self, nin, nex, block):
        lx, ly, lz, lt = self.lattice
        nvol = lx * ly * lz * lt
        v = np.zeros((nex, nvol, nin))
        for j in range(nex):
            for zt in range(lz * lt):
                g = self.planes[zt]
                for y in range(ly):
                    for x in range(lx):
                        v[j, x + lx * (y + ly * zt)] = block(g, nin)
        return v.reshape(-1)

    def gauss_lex_global(self, nin, nex):
        """Field(nin, Nvol, nex) in the corelib layout (nin even)."""
        def block(g, n):
            out = []
            for _ in range(n // 2):
                out.extend(g.gauss())
            return out
        return self._lex(nin, nex, block)

    def uniform_lex_global(self, nin, nex):
        def block(g, n):
            out = [0.0] * n
            out[0] = g.get()
            return out
        return self._lex(nin, nex, block)
