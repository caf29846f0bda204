"""Seeded synthetic molecular-like systems for the determinant-space path.

Integrals follow one recipe (used by every workload here):

* ``h1e`` is a symmetric FP64 matrix whose diagonal is drawn from U(-20, 0)
  and sorted ascending, with off-diagonal entries N(0, 0.05);
* the ERI tensor is built in Cholesky form, ``(pq|rs) = sum_K L^K_pq L^K_rs``
  with symmetric ``L^K`` of N(0, 0.1) entries, so it is positive
  semi-definite and 8-fold symmetric;
* the constant core energy is 9.0 Ha.

Arrays are returned in the packed layout of the reference integral store
(``csrc/detnqs/integral/integral_mo.hpp:30-49``): ``h1e[h1e_key(p,q)]`` with
``h1e_key(p,q) = P(P+1)/2 + Q`` (P = max, Q = min) and
``eri[h2e_key(p,q,r,s)] = eri[K(K+1)/2 + L]`` with K >= L the two pair keys.

Determinant sets are uint64[N, 2] (alpha mask, beta mask), bit i = orbital i,
matching ``Det`` (``csrc/detnqs/determinant/det.hpp:30-36``).
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

E_CORE = 9.0


@dataclass
class SyntheticSystem:
    n_orb: int
    n_alpha: int
    n_beta: int
    h1e: np.ndarray      # packed, n(n+1)/2
    eri: np.ndarray      # packed, n1e(n1e+1)/2
    e_core: float
    seed: int

    @property
    def n_elec(self) -> int:
        return self.n_alpha + self.n_beta

    def hf_det(self) -> np.ndarray:
        return hf_determinant(self.n_alpha, self.n_beta)


def pair_index(n: int) -> np.ndarray:
    """Matrix K[p, q] = h1e_key(p, q) (symmetric)."""
    p = np.arange(n)[:, None]
    q = np.arange(n)[None, :]
    hi = np.maximum(p, q)
    lo = np.minimum(p, q)
    return hi * (hi + 1) // 2 + lo


def make_integrals(n_orb: int, n_chol: int, seed: int,
                   e_core: float = E_CORE) -> tuple[np.ndarray, np.ndarray]:
    """Packed (h1e, eri) drawn with ``np.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    n = n_orb
    diag = np.sort(rng.uniform(-20.0, 0.0, size=n))
    off = rng.normal(0.0, 0.05, size=(n, n))
    h = np.triu(off, 1)
    h = h + h.T
    h[np.arange(n), np.arange(n)] = diag

    # Symmetric Cholesky vectors, drawn on the packed triangle.
    n1e = n * (n + 1) // 2
    L = rng.normal(0.0, 0.1, size=(n_chol, n1e))
    return _pack(h, L, n)


def _pack(h: np.ndarray, L: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Packed h1e from the dense symmetric h, packed ERIs from the Cholesky
    vectors L[K, pair key]."""
    n1e = n * (n + 1) // 2
    # G[k1, k2] = sum_K L[K, k1] L[K, k2]: one entry per unordered pair key.
    G = L.T @ L
    k1, k2 = np.tril_indices(n1e)
    eri = np.ascontiguousarray(G[k1, k2])   # row-major lower triangle = key order
    key = pair_index(n)
    h1e = np.empty(n1e)
    p, q = np.tril_indices(n)
    h1e[key[p, q]] = h[p, q]
    return h1e, eri


def scan_family(n_orb: int, n_alpha: int, n_beta: int, n_chol: int, seed: int,
                points: int = 10, amplitude: float = 0.02) -> list[SyntheticSystem]:
    """A bond-scan-like family: a seeded base (same recipe as
    :func:`make_integrals`) and ``points`` geometries whose h and Cholesky
    vectors are the base scaled element-wise by 1 + amplitude * t * xi, with
    t running evenly over [-1, 1] and xi ~ U(-1, 1) one seeded direction per
    family; neighbouring points differ smoothly and the end points by up to
    +-amplitude.  The ERIs stay positive semi-definite and 8-fold
    symmetric."""
    rng = np.random.default_rng(seed)
    n = n_orb
    diag = np.sort(rng.uniform(-20.0, 0.0, size=n))
    off = rng.normal(0.0, 0.05, size=(n, n))
    h = np.triu(off, 1)
    h = h + h.T
    h[np.arange(n), np.arange(n)] = diag
    n1e = n * (n + 1) // 2
    L = rng.normal(0.0, 0.1, size=(n_chol, n1e))
    xi_h = rng.uniform(-1.0, 1.0, size=(n, n))
    xi_h = np.triu(xi_h) + np.triu(xi_h, 1).T
    xi_L = rng.uniform(-1.0, 1.0, size=L.shape)
    out = []
    for k, t in enumerate(np.linspace(-1.0, 1.0, points)):
        h1e, eri = _pack(h * (1.0 + amplitude * t * xi_h), L * (1.0 + amplitude * t * xi_L), n)
        out.append(SyntheticSystem(n, n_alpha, n_beta, h1e, eri, E_CORE, seed * 100 + k))
    return out


def make_system(n_orb: int, n_alpha: int, n_beta: int, n_chol: int,
                seed: int) -> SyntheticSystem:
    h1e, eri = make_integrals(n_orb, n_chol, seed)
    return SyntheticSystem(n_orb, n_alpha, n_beta, h1e, eri, E_CORE, seed)


def write_fcidump(path: str, sysm: SyntheticSystem) -> None:
    """FCIDUMP with every value written as ``%.17e`` (exact round trip)."""
    n = sysm.n_orb
    key = pair_index(n)
    lines = [f" &FCI NORB={n},NELEC={sysm.n_elec},MS2={sysm.n_alpha - sysm.n_beta},",
             "  ORBSYM=" + "1," * n, "  ISYM=1,", " &END"]
    out = ["\n".join(lines)]
    pq = [(p, q) for p in range(n) for q in range(p + 1)]
    for a, (p, q) in enumerate(pq):
        for b in range(a + 1):
            r, s = pq[b]
            v = sysm.eri[a * (a + 1) // 2 + b]
            out.append(f"{v:.17e} {p + 1} {q + 1} {r + 1} {s + 1}")
    for p in range(n):
        for q in range(p + 1):
            out.append(f"{sysm.h1e[key[p, q]]:.17e} {p + 1} {q + 1} 0 0")
    out.append(f"{sysm.e_core:.17e} 0 0 0 0")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


def read_fcidump(path: str, n_orb: int) -> tuple[np.ndarray, np.ndarray, float]:
    """Parse an FCIDUMP into packed (h1e, eri, e_nuc) like the reference
    parser (``csrc/src/integral/integral_mo.cpp:48-182``): namelist skipped,
    ``D`` exponents accepted, 1-based indices, last assignment wins."""
    n = n_orb
    n1e = n * (n + 1) // 2
    h1e = np.zeros(n1e)
    eri = np.zeros(n1e * (n1e + 1) // 2)
    e_nuc = 0.0
    key = pair_index(n)
    with open(path) as f:
        for line in f:
            if not line.strip() or line[0] in "!*Cc#" or "&" in line:
                continue
            parts = line.replace("D", "E").replace("d", "E").split()
            if len(parts) < 5:
                continue
            try:
                v = float(parts[0])
                p, q, r, s = (int(x) for x in parts[1:5])
            except ValueError:
                continue
            if p == q == r == s == 0:
                e_nuc = v
            elif r == 0 and s == 0:
                h1e[key[p - 1, q - 1]] = v
            else:
                a = key[p - 1, q - 1]
                b = key[r - 1, s - 1]
                if a < b:
                    a, b = b, a
                eri[a * (a + 1) // 2 + b] = v
    return h1e, eri, e_nuc


def hf_determinant(n_alpha: int, n_beta: int) -> np.ndarray:
    a = (1 << n_alpha) - 1
    b = (1 << n_beta) - 1
    return np.array([[a, b]], dtype=np.uint64)


# ---------------------------------------------------------------------------
# Determinant sets
# ---------------------------------------------------------------------------

def _bits(mask: int, n: int) -> list[int]:
    return [i for i in range(n) if (mask >> i) & 1]


def singles_doubles(det: np.ndarray, n_orb: int) -> np.ndarray:
    """All single and double excitations of one determinant (sorted)."""
    a0, b0 = int(det[0]), int(det[1])
    out = set()
    for spin in (0, 1):
        m = a0 if spin == 0 else b0
        occ = _bits(m, n_orb)
        vir = [i for i in range(n_orb) if not (m >> i) & 1]
        for h in occ:
            for p in vir:
                mm = m ^ (1 << h) ^ (1 << p)
                out.add((mm, b0) if spin == 0 else (a0, mm))
        for i1 in range(len(occ)):
            for i2 in range(i1 + 1, len(occ)):
                for j1 in range(len(vir)):
                    for j2 in range(j1 + 1, len(vir)):
                        mm = m ^ (1 << occ[i1]) ^ (1 << occ[i2]) ^ (1 << vir[j1]) ^ (1 << vir[j2])
                        out.add((mm, b0) if spin == 0 else (a0, mm))
    occa, vira = _bits(a0, n_orb), [i for i in range(n_orb) if not (a0 >> i) & 1]
    occb, virb = _bits(b0, n_orb), [i for i in range(n_orb) if not (b0 >> i) & 1]
    for h in occa:
        for p in vira:
            na = a0 ^ (1 << h) ^ (1 << p)
            for hb in occb:
                for pb in virb:
                    out.add((na, b0 ^ (1 << hb) ^ (1 << pb)))
    arr = np.array(sorted(out), dtype=np.uint64).reshape(-1, 2)
    return arr


def hf_sd_space(n_orb: int, n_alpha: int, n_beta: int) -> np.ndarray:
    """HF followed by all its singles and doubles (sorted)."""
    hf = hf_determinant(n_alpha, n_beta)
    sd = singles_doubles(hf[0], n_orb)
    return np.ascontiguousarray(np.concatenate([hf, sd], axis=0))


def _popcount64(x: np.ndarray) -> np.ndarray:
    x = x.astype(np.uint64)
    c = np.zeros(x.shape, dtype=np.int64)
    for shift in range(0, 64, 8):
        c += _POP8[((x >> np.uint64(shift)) & np.uint64(0xFF)).astype(np.int64)]
    return c


_POP8 = np.array([bin(i).count("1") for i in range(256)], dtype=np.int64)


def _occ_table(masks: np.ndarray, n_orb: int, n_occ: int) -> np.ndarray:
    """Sorted occupied orbital indices per mask, shape (N, n_occ)."""
    bits = ((masks[:, None] >> np.arange(n_orb, dtype=np.uint64)[None, :])
            & np.uint64(1)).astype(bool)
    idx = np.nonzero(bits)[1].reshape(-1, n_occ)
    return idx


def heat_bath_sample(sysm: SyntheticSystem, n_dets: int, seed: int,
                     max_level: int = 4, batch: int = 1 << 18) -> np.ndarray:
    """Iterated heat-bath sampling of a determinant set.

    Starts from HF.  Each round draws parents uniformly from the set built
    so far and proposes one excitation per parent:

    * 1 in 16 proposals is a single (uniform hole, uniform virtual);
    * otherwise a double: an occupied pair is drawn uniformly (same-spin
      with probability 5/15) and the virtual pair with probability
      proportional to its heat-bath weight |<ij||ab>| (the weight of the
      reference table, ``csrc/src/integral/hb_table.cpp:102-138``),
      rejecting pairs that are occupied in the parent.

    Children whose excitation level from HF exceeds ``max_level`` are
    dropped; new unique determinants are appended in draw order until
    ``n_dets`` are collected (or no new determinant appears for 8 rounds,
    when the space is smaller).  Deterministic for a given ``seed``.
    """
    n = sysm.n_orb
    na, nb = sysm.n_alpha, sysm.n_beta
    rng = np.random.default_rng(seed)
    eri4 = unpack_eri(sysm.eri, n)
    # opposite-spin rows: (i, j) -> weights over (a, b) = |(ia|jb)|
    w_os = np.abs(eri4.transpose(0, 2, 1, 3)).reshape(n * n, n * n)
    # same-spin rows: |(ia|jb) - (ib|ja)| restricted to a < b
    anti = eri4.transpose(0, 2, 1, 3) - eri4.transpose(0, 2, 3, 1)
    w_ss = np.abs(anti) * np.triu(np.ones((n, n)), 1)[None, None]
    w_ss = w_ss.reshape(n * n, n * n)

    def sampler(w):
        cs = np.cumsum(w, axis=1)
        tot = cs[:, -1].copy()
        flat = (cs + np.concatenate([[0.0], np.cumsum(tot)[:-1]])[:, None]).ravel()
        base = np.concatenate([[0.0], np.cumsum(tot)[:-1]])
        return flat, base, tot

    os_flat, os_base, os_tot = sampler(w_os)
    ss_flat, ss_base, ss_tot = sampler(w_ss)
    del eri4, anti, w_os, w_ss
    nn = n * n
    one = np.uint64(1)
    hf = hf_determinant(na, nb)[0]
    hfa, hfb = hf[0], hf[1]
    out = np.zeros((n_dets, 2), dtype=np.uint64)
    out[0] = hf
    count = 1
    seen = {(int(hf[0]), int(hf[1]))}
    stalled = 0
    while count < n_dets and stalled < 8:
        before = count
        m = batch
        par = out[rng.integers(0, count, size=m)]
        occ_a = _occ_table(par[:, 0], n, na)
        occ_b = _occ_table(par[:, 1], n, nb)
        kind = rng.integers(0, 16, size=m)
        spin = rng.integers(0, 2, size=m)
        r = np.arange(m)
        # opposite-spin double
        i = occ_a[r, rng.integers(0, na, size=m)].astype(np.int64)
        j = occ_b[r, rng.integers(0, nb, size=m)].astype(np.int64)
        row = i * n + j
        t = os_base[row] + rng.random(m) * os_tot[row]
        k = np.minimum(np.searchsorted(os_flat, t, side="right") - row * nn, nn - 1)
        a, b = k // n, k % n
        ca_os = par[:, 0] ^ (one << i.astype(np.uint64)) ^ (one << a.astype(np.uint64))
        cb_os = par[:, 1] ^ (one << j.astype(np.uint64)) ^ (one << b.astype(np.uint64))
        ok_os = (((par[:, 0] >> a.astype(np.uint64)) & one) == 0) & \
                (((par[:, 1] >> b.astype(np.uint64)) & one) == 0) & (os_tot[row] > 0)
        # same-spin double
        ne_s = np.where(spin == 0, na, nb)
        occ_s = np.where(spin[:, None] == 0, occ_a[:, :min(na, nb)] if na <= nb else occ_a[:, :nb],
                         occ_b[:, :min(na, nb)] if nb <= na else occ_b[:, :na])
        ns = occ_s.shape[1]
        p1 = rng.integers(0, max(ns, 1), size=m)
        p2 = (p1 + rng.integers(1, max(ns, 2), size=m)) % max(ns, 1)
        si = occ_s[r, p1].astype(np.int64)
        sj = occ_s[r, p2].astype(np.int64)
        srow = np.minimum(si, sj) * n + np.maximum(si, sj)
        t = ss_base[srow] + rng.random(m) * ss_tot[srow]
        k = np.minimum(np.searchsorted(ss_flat, t, side="right") - srow * nn, nn - 1)
        sa, sb = k // n, k % n
        sm = np.where(spin == 0, par[:, 0], par[:, 1])
        ok_ss = (((sm >> sa.astype(np.uint64)) & one) == 0) & \
                (((sm >> sb.astype(np.uint64)) & one) == 0) & (ss_tot[srow] > 0) & \
                (si != sj) & (sa != sb) & (ns >= 2)
        sm2 = sm ^ (one << si.astype(np.uint64)) ^ (one << sj.astype(np.uint64)) \
            ^ (one << sa.astype(np.uint64)) ^ (one << sb.astype(np.uint64))
        ca_ss = np.where(spin == 0, sm2, par[:, 0])
        cb_ss = np.where(spin == 0, par[:, 1], sm2)
        # single
        hsel = np.where(spin == 0, occ_a[r, rng.integers(0, na, size=m)],
                        occ_b[r, rng.integers(0, nb, size=m)]).astype(np.uint64)
        pv = rng.integers(0, n, size=m).astype(np.uint64)
        ok_s = ((sm >> pv) & one) == 0
        sg = sm ^ (one << hsel) ^ (one << pv)
        ca_s = np.where(spin == 0, sg, par[:, 0])
        cb_s = np.where(spin == 0, par[:, 1], sg)
        del ne_s
        ca = np.where(kind == 0, ca_s, np.where(kind <= 5, ca_ss, ca_os))
        cb = np.where(kind == 0, cb_s, np.where(kind <= 5, cb_ss, cb_os))
        good = np.where(kind == 0, ok_s, np.where(kind <= 5, ok_ss, ok_os))
        ca, cb = ca[good], cb[good]
        lev = (_popcount64(ca ^ hfa) + _popcount64(cb ^ hfb)) // 2
        keep = lev <= max_level
        ca, cb = ca[keep], cb[keep]
        for x, y in zip(ca.tolist(), cb.tolist()):
            if (x, y) not in seen:
                seen.add((x, y))
                out[count, 0] = x
                out[count, 1] = y
                count += 1
                if count >= n_dets:
                    break
        stalled = stalled + 1 if count == before else 0
    # a space smaller than n_dets (few orbitals / low level) ends the draw
    return np.ascontiguousarray(out[:count])


def hf_determinant_wide(n_alpha: int, n_beta: int) -> np.ndarray:
    """HF determinant as uint64[1, 4] = (alpha lo, alpha hi, beta lo, beta hi)."""
    return pack_wide(np.arange(n_alpha)[None, :], np.arange(n_beta)[None, :])


def pack_wide(occ_a: np.ndarray, occ_b: np.ndarray) -> np.ndarray:
    """uint64[N, 4] two-word masks (bit i of a spin = orbital i; word 0 holds
    orbitals 0..63, word 1 orbitals 64..127) from occupied-index tables."""
    out = np.zeros((occ_a.shape[0], 4), dtype=np.uint64)
    for col, occ in ((0, occ_a), (2, occ_b)):
        occ = np.asarray(occ, dtype=np.int64)
        for w in (0, 1):
            sel = (occ >> 6) == w
            bits = np.where(sel, np.uint64(1) << (occ & 63).astype(np.uint64), np.uint64(0))
            out[:, col + w] = np.bitwise_or.reduce(bits, axis=1) if occ.shape[1] else 0
    return out


def unpack_wide(dets: np.ndarray, n_orb: int) -> tuple[np.ndarray, np.ndarray]:
    """Boolean occupations (N, n_orb) of the alpha and beta strings of
    uint64[N, 4] determinants."""
    d = np.ascontiguousarray(dets, dtype=np.uint64)
    bits = np.unpackbits(d.view(np.uint8).reshape(-1, 4, 8), axis=2, bitorder="little")
    a = bits[:, 0:2].reshape(-1, 128)[:, :n_orb].astype(bool)
    b = bits[:, 2:4].reshape(-1, 128)[:, :n_orb].astype(bool)
    return a, b


def heat_bath_sample_wide(sysm: SyntheticSystem, n_dets: int, seed: int,
                          max_level: int = 4, batch: int = 1 << 17) -> np.ndarray:
    """Iterated heat-bath sampling for up to 128 orbitals, two words per
    spin (uint64[N, 4] = alpha lo, alpha hi, beta lo, beta hi).

    The proposals are those of :func:`heat_bath_sample` (1 in 16 a uniform
    single; otherwise a double with a uniform occupied pair, same-spin with
    probability 5/15, and the virtual pair drawn with probability
    proportional to its heat-bath weight), kept when new and at most
    ``max_level`` excitations from HF.  Occupations are held as index
    tables, so any orbital count up to 128 works.  Deterministic for a
    given ``seed``."""
    n = sysm.n_orb
    if n > 128:
        raise ValueError("two-word determinants hold at most 128 orbitals")
    na, nb = sysm.n_alpha, sysm.n_beta
    rng = np.random.default_rng(seed)
    eri4 = unpack_eri(sysm.eri, n)
    w_os = np.abs(eri4.transpose(0, 2, 1, 3)).reshape(n * n, n * n)
    anti = eri4.transpose(0, 2, 1, 3) - eri4.transpose(0, 2, 3, 1)
    del eri4
    w_ss = (np.abs(anti) * np.triu(np.ones((n, n)), 1)[None, None]).reshape(n * n, n * n)
    del anti

    def sampler(w):
        cs = np.cumsum(w, axis=1)
        tot = cs[:, -1].copy()
        base = np.concatenate([[0.0], np.cumsum(tot)[:-1]])
        cs += base[:, None]
        return cs.ravel(), base, tot

    os_flat, os_base, os_tot = sampler(w_os)
    del w_os
    ss_flat, ss_base, ss_tot = sampler(w_ss)
    del w_ss
    nn = n * n
    A = np.zeros((n_dets, na), dtype=np.int16)
    B = np.zeros((n_dets, nb), dtype=np.int16)
    A[0] = np.arange(na)
    B[0] = np.arange(nb)
    out = np.zeros((n_dets, 4), dtype=np.uint64)
    out[0] = hf_determinant_wide(na, nb)[0]
    seen = {tuple(int(x) for x in out[0])}
    count, stalled = 1, 0
    while count < n_dets and stalled < 8:
        before = count
        m = batch
        par = rng.integers(0, count, size=m)
        pa, pb = A[par].astype(np.int64), B[par].astype(np.int64)
        r = np.arange(m)
        oa = np.zeros((m, n), dtype=bool)
        ob = np.zeros((m, n), dtype=bool)
        oa[r[:, None], pa] = True
        ob[r[:, None], pb] = True
        kind = rng.integers(0, 16, size=m)
        spin = rng.integers(0, 2, size=m)
        # opposite-spin double
        i = pa[r, rng.integers(0, na, size=m)]
        j = pb[r, rng.integers(0, nb, size=m)]
        row = i * n + j
        t = os_base[row] + rng.random(m) * os_tot[row]
        k = np.minimum(np.searchsorted(os_flat, t, side="right") - row * nn, nn - 1)
        a, b = k // n, k % n
        ok_os = ~oa[r, a] & ~ob[r, b] & (os_tot[row] > 0)
        # same-spin double
        ns = min(na, nb)
        ps = np.where(spin[:, None] == 0, pa[:, :ns], pb[:, :ns])
        p1 = rng.integers(0, max(ns, 1), size=m)
        p2 = (p1 + rng.integers(1, max(ns, 2), size=m)) % max(ns, 1)
        si, sj = ps[r, p1], ps[r, p2]
        srow = np.minimum(si, sj) * n + np.maximum(si, sj)
        t = ss_base[srow] + rng.random(m) * ss_tot[srow]
        k = np.minimum(np.searchsorted(ss_flat, t, side="right") - srow * nn, nn - 1)
        sa, sb = k // n, k % n
        os_ = np.where(spin[:, None] == 0, oa, ob)
        ok_ss = ~os_[r, sa] & ~os_[r, sb] & (ss_tot[srow] > 0) & (si != sj) & (sa != sb) & \
            (ns >= 2)
        # single
        hsel = np.where(spin == 0, pa[r, rng.integers(0, na, size=m)],
                        pb[r, rng.integers(0, nb, size=m)])
        pv = rng.integers(0, n, size=m)
        ok_s = ~os_[r, pv]
        good = np.where(kind == 0, ok_s, np.where(kind <= 5, ok_ss, ok_os))
        ca, cb = oa.copy(), ob.copy()
        # apply each kind on its rows
        sel = good & (kind >= 6)
        ca[r[sel], i[sel]] = False; ca[r[sel], a[sel]] = True
        cb[r[sel], j[sel]] = False; cb[r[sel], b[sel]] = True
        for sp, C in ((0, ca), (1, cb)):
            sel = good & (kind >= 1) & (kind <= 5) & (spin == sp)
            C[r[sel], si[sel]] = False; C[r[sel], sj[sel]] = False
            C[r[sel], sa[sel]] = True; C[r[sel], sb[sel]] = True
            sel = good & (kind == 0) & (spin == sp)
            C[r[sel], hsel[sel]] = False; C[r[sel], pv[sel]] = True
        lev = (~ca[:, :na]).sum(1) + (~cb[:, :nb]).sum(1)
        keep = good & (lev <= max_level)
        ca, cb = ca[keep], cb[keep]
        occa = np.nonzero(ca)[1].reshape(-1, na)
        occb = np.nonzero(cb)[1].reshape(-1, nb)
        keys = pack_wide(occa, occb)
        for q, kk in enumerate(map(tuple, keys.tolist())):
            if kk not in seen:
                seen.add(kk)
                out[count] = keys[q]
                A[count] = occa[q]
                B[count] = occb[q]
                count += 1
                if count >= n_dets:
                    break
        stalled = stalled + 1 if count == before else 0
    return np.ascontiguousarray(out[:count])


def unpack_eri(eri: np.ndarray, n: int) -> np.ndarray:
    """Dense (pq|rs) tensor from the packed 8-fold array."""
    key = pair_index(n)
    K1 = key[:, :, None, None]
    K2 = key[None, None, :, :]
    hi = np.maximum(K1, K2)
    lo = np.minimum(K1, K2)
    return eri[hi * (hi + 1) // 2 + lo]


def unpack_h1e(h1e: np.ndarray, n: int) -> np.ndarray:
    return h1e[pair_index(n)]


def normalized_psi(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.normal(size=n)
    return v / np.linalg.norm(v)


__all__ = [
    "SyntheticSystem", "make_integrals", "make_system", "write_fcidump",
    "read_fcidump", "hf_determinant", "singles_doubles", "hf_sd_space",
    "heat_bath_sample", "unpack_eri", "unpack_h1e", "normalized_psi", "scan_family",
    "heat_bath_sample_wide", "hf_determinant_wide", "pack_wide", "unpack_wide",
    "pair_index", "E_CORE",
]
