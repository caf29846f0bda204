"""Generate the real-molecule fixtures of tests/golden/ from the reference.

Run in a container that has the reference tree (its FCIDUMP fixtures and
its C++ core, compiled from its own sources into oracle/_ref/):

    make -C oracle ref REF=<reference tree>
    python tests/golden/make_molecules.py <reference tree>

Writes
  molecules.npz          -- packed integrals (h1e, 8-fold ERI, E_nuc) of five
                            of the reference's FCIDUMP fixtures
                            (benchmark/FCIDUMP/): H2/6-31G at 2.00 bohr
                            (4 orbitals), H2O/STO-3G (7 orbitals),
                            H2O/6-31G (13 orbitals, the 13-orbital /
                            10-electron workload shape), Cr2 24e/30o (the
                            30-orbital / 24-electron shape) and N2/cc-pVDZ
                            at R = 2.118 bohr, parsed by the reference's
                            rules;
  molecule_checksums.json -- SHA-256 checksums of the reference core's
                            outputs on those integrals: the ordered heat-bath
                            rows (ties included), get_ham_conn /
                            get_ham_conn_amp / get_ham_eff, ordered
                            get_local_connections, compute_variational_energy
                            and a row sample of the screened V->V block of a
                            heat-bath-sampled Cr2 space.

Before writing anything it checks that the reference core reading each
FCIDUMP and reading the packed arrays gives bit-identical Hamiltonians, so
the arrays are exactly what the reference sees.
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import tempfile
from types import SimpleNamespace

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from detnqs_b200 import synthetic as S  # noqa: E402
from oracle import Checker  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (file under benchmark/FCIDUMP, n_orb, n_alpha, n_beta)
MOLECULES = {
    "h2_631g": ("H2_631g_2.00.FCIDUMP", 4, 1, 1),
    "h2o_sto3g": ("H2O_sto3g.FCIDUMP", 7, 5, 5),
    "h2o_631g": ("H2O_631g.FCIDUMP", 13, 5, 5),
    "cr2_24e30o": ("Cr2/Cr2_24e30o.FCIDUMP", 30, 12, 12),
    "n2_ccpvdz": ("N2_ccpvdz/N2_ccpvdz_2.118B.FCIDUMP", 28, 7, 7),
}

CONN_EPS = 1e-8          # get_ham_conn on H2O/6-31G (HF + all S + D)
AMP_EPS = 1e-6           # get_ham_conn_amp on the same space
LOCAL_EPS = 1e-6         # get_local_connections
CR2_DETS = 20000         # heat-bath-sampled Cr2 space
CR2_EPS = 1e-6
CR2_ROWS = 64


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def coo_sha(d: dict) -> dict:
    return {"nnz": int(len(d["val"])), "shape": [int(x) for x in d["shape"]],
            "sha256": sha(d["row"].astype(np.uint32), d["col"].astype(np.uint32),
                          d["val"].astype(np.float64))}


def conn_sha(c: dict) -> dict:
    return {"n": int(len(c["values"])),
            "sha256": sha(c["offsets"].astype(np.int32), c["dets"].astype(np.uint64),
                          c["values"].astype(np.float64))}


def hb_rows_sha(ctx, nso: int) -> dict:
    """Every heat-bath row (i > j) in the table's order, hashed in row order,
    and how many rows hold tied weights."""
    h = hashlib.sha256()
    ties = 0
    total = 0
    for i in range(1, nso):
        for j in range(i):
            a, b, w = ctx.hb_row(i, j)
            h.update(a.astype(np.int32).tobytes())
            h.update(b.astype(np.int32).tobytes())
            h.update(w.astype(np.float64).tobytes())
            total += len(w)
            ties += bool(len(w) > 1 and np.any(w[1:] == w[:-1]))
    return {"entries": total, "rows_with_ties": ties, "sha256": h.hexdigest()}


def ref_ctx(ref, m: dict):
    """The reference core on the packed arrays: it loads integrals from an
    FCIDUMP only, so they go through one written with %.17e (exact)."""
    sysm = SimpleNamespace(n_orb=m["n_orb"], n_alpha=m["n_alpha"], n_beta=m["n_beta"],
                           n_elec=m["n_alpha"] + m["n_beta"], h1e=m["h1e"], eri=m["eri"],
                           e_core=m["e_nuc"])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "arrays.FCIDUMP")
        S.write_fcidump(path, sysm)
        return ref.ctx_from_fcidump(path, m["n_orb"])


def sampled_space(mol, n_dets, seed):
    sysm = SimpleNamespace(n_orb=mol["n_orb"], n_alpha=mol["n_alpha"],
                           n_beta=mol["n_beta"], h1e=mol["h1e"], eri=mol["eri"])
    return S.heat_bath_sample(sysm, n_dets, seed)


def psi_for(n, seed):
    return S.normalized_psi(n, seed)


def main(tree: str) -> None:
    ref = Checker.reference()
    arrays = {}
    mols = {}
    for name, (fname, n, na, nb) in MOLECULES.items():
        path = os.path.join(tree, "benchmark", "FCIDUMP", fname)
        h1e, eri, e_nuc = S.read_fcidump(path, n)
        # the reference reading the file and reading the arrays must agree
        c_file = ref.ctx_from_fcidump(path, n)
        m = {"n_orb": n, "n_alpha": na, "n_beta": nb, "h1e": h1e, "eri": eri, "e_nuc": e_nuc}
        c_arr = ref_ctx(ref, m)
        assert c_file.get_e_nuc() == e_nuc, name
        V = S.hf_sd_space(n, na, nb)[:400]
        a, b = c_file.get_ham_vv(V), c_arr.get_ham_vv(V)
        assert coo_sha(a) == coo_sha(b), name
        np.testing.assert_array_equal(c_file.get_ham_diag(V).view(np.uint64),
                                      c_arr.get_ham_diag(V).view(np.uint64))
        mols[name] = m
        arrays[f"{name}_h1e"] = h1e
        arrays[f"{name}_eri"] = eri
        arrays[f"{name}_e_nuc"] = np.array(e_nuc)
        arrays[f"{name}_shape"] = np.array([n, na, nb])
    np.savez_compressed(os.path.join(OUT, "molecules.npz"), **arrays)

    out = {"conn_eps": CONN_EPS, "amp_eps": AMP_EPS, "local_eps": LOCAL_EPS,
           "cr2_dets": CR2_DETS, "cr2_eps": CR2_EPS, "molecules": {}}
    for name, m in mols.items():
        n, na, nb = m["n_orb"], m["n_alpha"], m["n_beta"]
        ctx = ref_ctx(ref, m)
        ctx.hb_prepare(1e-15)
        rec = {"hb_rows": hb_rows_sha(ctx, 2 * n)}
        # local connections of 48 determinants of HF + S + D, both modes
        V = S.hf_sd_space(n, na, nb)
        pick = np.random.default_rng(5).choice(len(V), size=min(48, len(V)), replace=False)
        sub = V[np.sort(pick)]
        rec["local_conn_rows"] = [int(x) for x in np.sort(pick)]
        rec["local_conn_hb"] = conn_sha(ctx.get_local_connections(sub, True, LOCAL_EPS))
        rec["local_conn_full"] = conn_sha(ctx.get_local_connections(sub, False, LOCAL_EPS))
        if name in ("h2o_sto3g", "h2o_631g"):
            psi = psi_for(len(V), 31)
            conn = ctx.get_ham_conn(V, True, CONN_EPS)
            rec["conn"] = {"H_VV": coo_sha(conn["H_VV"]), "H_VP": coo_sha(conn["H_VP"]),
                           "size_P": int(conn["size_P"]),
                           "det_P_sha256": sha(conn["det_P"].astype(np.uint64))}
            amp = ctx.get_ham_conn_amp(V, psi, AMP_EPS)
            rec["conn_amp"] = {"H_VV": coo_sha(amp["H_VV"]), "H_VP": coo_sha(amp["H_VP"]),
                               "size_P": int(amp["size_P"]),
                               "det_P_sha256": sha(amp["det_P"].astype(np.uint64))}
            hpp = ctx.get_ham_diag(amp["det_P"])
            e_var = ctx.compute_variational_energy(V, psi, True, AMP_EPS)
            e_ref = e_var                      # electronic energy of psi
            eff = ref.get_ham_eff(amp["H_VV"], amp["H_VP"], hpp, e_ref)
            rec["eff"] = {"e_ref": e_ref, **coo_sha(eff)}
            rec["e_var_hb"] = e_var
            rec["e_var_full"] = ctx.compute_variational_energy(V, psi, False, AMP_EPS)
        if name == "cr2_24e30o":
            Vs = sampled_space(m, CR2_DETS, 17)
            rows = np.random.default_rng(9).choice(len(Vs), size=CR2_ROWS, replace=False)
            rows = np.unique(np.concatenate([[0], rows]))
            blk = ctx.vv_hb_rows(Vs, rows, CR2_EPS)
            per = []
            for r in rows:
                sel = blk["row"] == r
                cols = blk["col"][sel]
                vals = blk["val"][sel]
                order = np.argsort(cols, kind="stable")
                per.append({"row": int(r), "nnz": int(sel.sum()),
                            "sha256": sha(cols[order].astype(np.uint32),
                                          vals[order].astype(np.float64))})
            rec["vv_rows"] = {"space_sha256": sha(Vs.astype(np.uint64)), "rows": per}
        out["molecules"][name] = rec
        print(name, json.dumps(rec["hb_rows"]), flush=True)
    with open(os.path.join(OUT, "molecule_checksums.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["DETNQS_REFERENCE_ROOT"])
