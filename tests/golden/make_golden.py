"""Generate the golden fixtures of tests/golden/ from the reference core.

Run in a container that has the reference tree (the recipe compiles it from
its own sources into oracle/_ref/):

    make -C oracle ref && python tests/golden/make_golden.py

Writes
  golden_small.npz   -- a small synthetic system (integrals included) with
                        the reference's outputs of every builder on it;
  c0_checksums.json  -- SHA-256 checksums of the reference's full outputs on
                        the 13-orbital / 10-electron workload (HF + all
                        singles and doubles = 2241 determinants, K = 26,
                        eps1 = 1e-8), so the full-size result can be checked
                        bit for bit without committing ~100 MB of arrays.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from detnqs_b200 import synthetic as S  # noqa: E402
from oracle import Checker  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

C0_SEED = 20251
SMALL_SEED = 7


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def coo_sha(d: dict) -> dict:
    return {"nnz": int(len(d["val"])), "shape": list(d["shape"]),
            "sha256": sha(d["row"].astype(np.uint32), d["col"].astype(np.uint32),
                          d["val"].astype(np.float64))}


def small_system():
    sysm = S.make_system(8, 3, 3, 16, SMALL_SEED)
    V = S.hf_sd_space(8, 3, 3)[:120]
    rng = np.random.default_rng(11)
    psi = rng.normal(size=len(V))
    psi /= np.linalg.norm(psi)
    return sysm, V, psi


def main() -> None:
    ref = Checker.reference()
    tmp = tempfile.mkdtemp()

    # ---------------- small system: full outputs ----------------
    sysm, V, psi = small_system()
    fd = os.path.join(tmp, "small.fcidump")
    S.write_fcidump(fd, sysm)
    ctx = ref.ctx_from_fcidump(fd, sysm.n_orb)
    ctx.hb_prepare(1e-15)
    out = {"h1e": sysm.h1e, "eri": sysm.eri, "e_core": np.float64(sysm.e_core),
           "n_orb": np.int64(sysm.n_orb), "V": V, "psi": psi}
    out["diag"] = ctx.get_ham_diag(V)
    def put(prefix, d):
        out[prefix + "_row"] = d["row"]
        out[prefix + "_col"] = d["col"]
        out[prefix + "_val"] = d["val"]
        out[prefix + "_shape"] = np.array(d["shape"], np.int64)
    put("vv", ctx.get_ham_vv(V))
    conn = ctx.get_ham_conn(V, True, 1e-3)
    put("conn_vv", conn["H_VV"]); put("conn_vp", conn["H_VP"]); out["conn_P"] = conn["det_P"]
    connf = ctx.get_ham_conn(V, False, 1e-3)
    put("connf_vv", connf["H_VV"]); put("connf_vp", connf["H_VP"]); out["connf_P"] = connf["det_P"]
    amp = ctx.get_ham_conn_amp(V, psi, 1e-4)
    put("amp_vv", amp["H_VV"]); put("amp_vp", amp["H_VP"]); out["amp_P"] = amp["det_P"]
    ext = S.singles_doubles(V[5], sysm.n_orb)[:200]
    blk = ctx.get_ham_block(V[:60], ext)
    put("blk_vv", blk["H_VV"]); put("blk_vp", blk["H_VP"]); out["blk_ext"] = ext
    out["evar_hb"] = np.float64(ctx.compute_variational_energy(V, psi, True, 1e-3))
    out["evar_full"] = np.float64(ctx.compute_variational_energy(V, psi, False, 1e-6))
    hpp = ctx.get_ham_diag(conn["det_P"])
    eref = float(out["diag"][0])
    heff = ref.get_ham_eff(conn["H_VV"], conn["H_VP"], hpp, eref, "sigma", 1e-12)
    put("heff", heff)
    heffl = ref.get_ham_eff(conn["H_VV"], conn["H_VP"], hpp, eref, "linear_shift", 1e-8)
    put("heffl", heffl)
    out["heff_hpp"] = hpp
    out["heff_eref"] = np.float64(eref)
    # random (bra, ket) pairs of degree 0..4 for elements and phases
    rng = np.random.default_rng(3)
    fci_a = [m for m in range(1 << 8) if bin(m).count("1") == 3]
    bra = np.array([[fci_a[rng.integers(len(fci_a))], fci_a[rng.integers(len(fci_a))]]
                    for _ in range(400)], np.uint64)
    ket = np.array([[fci_a[rng.integers(len(fci_a))], fci_a[rng.integers(len(fci_a))]]
                    for _ in range(400)], np.uint64)
    ket[:150] = V[rng.integers(0, len(V), 150)]
    bra[:150] = V[rng.integers(0, len(V), 150)]
    out["pair_bra"], out["pair_ket"] = bra, ket
    out["pair_elem"] = np.array([ctx.compute_elem(b, k) for b, k in zip(bra, ket)])
    deg_ph = [ref.analyze(b, k) for b, k in zip(bra, ket)]
    out["pair_degree"] = np.array([d for d, _ in deg_ph], np.int32)
    out["pair_phase"] = np.array([p for _, p in deg_ph])
    # heat-bath rows of a few pairs
    rows = [(1, 0), (5, 2), (7, 4), (15, 14), (9, 6)]
    for (i, j) in rows:
        a, b, w = ctx.hb_row(i, j)
        out[f"hb_{i}_{j}_a"], out[f"hb_{i}_{j}_b"], out[f"hb_{i}_{j}_w"] = a, b, w
    np.savez_compressed(os.path.join(OUT, "golden_small.npz"), **out)

    # ---------------- 13-orbital workload: checksums ----------------
    c0 = S.make_system(13, 5, 5, 26, C0_SEED)
    V0 = S.hf_sd_space(13, 5, 5)
    fd0 = os.path.join(tmp, "c0.fcidump")
    S.write_fcidump(fd0, c0)
    cx = ref.ctx_from_fcidump(fd0, 13)
    cx.hb_prepare(1e-15)
    psi0 = S.normalized_psi(len(V0), 5)
    res = {"seed": C0_SEED, "n_orb": 13, "n_alpha": 5, "n_beta": 5, "n_chol": 26,
           "n_dets": int(len(V0)), "eps1": 1e-8, "psi_seed": 5}
    conn0 = cx.get_ham_conn(V0, True, 1e-8)
    res["conn_vv"] = coo_sha(conn0["H_VV"])
    res["conn_vp"] = coo_sha(conn0["H_VP"])
    res["conn_P"] = {"n": int(conn0["size_P"]), "sha256": sha(conn0["det_P"])}
    res["diag_sha256"] = sha(cx.get_ham_diag(V0))
    amp0 = cx.get_ham_conn_amp(V0, psi0, 1e-6)
    res["amp_vv"] = coo_sha(amp0["H_VV"])
    res["amp_vp"] = coo_sha(amp0["H_VP"])
    res["amp_P"] = {"n": int(amp0["size_P"]), "sha256": sha(amp0["det_P"])}
    res["evar_hb_1e-6"] = cx.compute_variational_energy(V0, psi0, True, 1e-6)
    hpp0 = cx.get_ham_diag(conn0["det_P"])
    e0 = float(cx.get_ham_diag(V0[:1])[0])
    heff0 = ref.get_ham_eff(conn0["H_VV"], conn0["H_VP"], hpp0, e0)
    res["heff"] = coo_sha(heff0)
    res["heff_e_ref"] = e0
    with open(os.path.join(OUT, "c0_checksums.json"), "w") as f:
        json.dump(res, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
