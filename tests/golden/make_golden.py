"""Copy the hf-rs golden vectors for the Fock-build path into small fixtures.

hf-rs keeps PySCF/mpmath-generated reference values under tests/data/ of its
own tree.  This script reads them from a local hf-rs checkout, whose root is
its one required argument (python make_golden.py <hf-rs root>), and writes the
subsets the parity tests here need, so that the tests run without the
reference tree:

  boys.json          tests/data/boys_reference.json (all 31 T values, n<=40)
  spdf_eri.npz       spherical_reference.json["spdf_integrals"]: the basis
                     text, geometry and every 7th of the 160,000 PySCF
                     Cartesian ERIs with their (i,j,k,l) indices
  scf_energies.json  scf_reference.json: RHF/UHF energies (STO-3G, 6-31G*)
  water_ccpvdz.json  spherical_reference.json["systems"]["water_ccpvdz"]
  cd_hf.json         cd_hf_reference.json: pivoted-Cholesky pivots, vector
                     counts, residuals and CD-HF energies (LiH STO-3G,
                     water and HCl 6-31G)
  df.npz             df_reference.json: metric, (P|mn) and the RI-MP2 energy
                     for water STO-3G / def2-SVP-RI, and the
                     df_hf_reference.json "water" case
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(root):
    data = os.path.join(root, "tests", "data")
    boys = json.load(open(os.path.join(data, "boys_reference.json")))
    rows = [{"t": r["t"], "f": [float(x) for x in r["f"]]} for r in boys["rows"]]
    json.dump({"source": "hf-rs tests/data/boys_reference.json (mpmath)", "rows": rows},
              open(os.path.join(HERE, "boys.json"), "w"))

    sph = json.load(open(os.path.join(data, "spherical_reference.json")))
    s = sph["spdf_integrals"]
    eri = np.array(s["eri"], dtype=np.float64)
    keep = np.arange(0, eri.size, 7)
    ijkl = np.stack([keep // 8000, keep // 400 % 20, keep // 20 % 20, keep % 20], axis=1).astype(np.int32)
    np.savez_compressed(os.path.join(HERE, "spdf_eri.npz"), basis=np.array(s["basis_gaussian94"]),
                        symbols=np.array(s["symbols"]), geometry=np.array(s["geometry_bohr"]),
                        ijkl=ijkl, eri=eri[keep])

    scf = json.load(open(os.path.join(data, "scf_reference.json")))
    out = []
    for name, sysd in scf["systems"].items():
        atoms = []
        for part in sysd["geometry_bohr"].split(";"):
            t = part.split()
            atoms.append([t[0], [float(x) for x in t[1:]]])
        for bname, res in sysd["results"].items():
            out.append({"name": name, "basis": bname, "atoms": atoms, "charge": sysd["charge"],
                        "spin_2s": sysd["spin_2s"], "reference": res["reference"], "n_ao": res["n_ao"],
                        "energy": res["energy"]})
    json.dump({"source": scf["source"], "cases": out}, open(os.path.join(HERE, "scf_energies.json"), "w"),
              indent=1)

    w = sph["systems"]["water_ccpvdz"]
    json.dump({"source": "hf-rs tests/spherical_basis_test.rs:135-166 geometry; PySCF energy",
               "atoms": [["O", [0.0, 0.0, 0.0]], ["H", [1.43, 0.2, 1.1]], ["H", [-1.2, -0.3, 1.3]]],
               "basis": "cc-pvdz", "spherical": True, "n_ao": w["n_ao"], "energy": w["energy"]},
              open(os.path.join(HERE, "water_ccpvdz.json"), "w"), indent=1)

    df = json.load(open(os.path.join(data, "df_reference.json")))
    dh = json.load(open(os.path.join(data, "df_hf_reference.json")))
    c = [x for x in dh["cases"] if x["name"] == "water"][0]
    np.savez_compressed(os.path.join(HERE, "df.npz"), metric=np.array(df["metric"]),
                        three=np.array(df["three"]), water_atoms=np.array(json.dumps(c["atoms"])),
                        e_scf=c["e_scf"], P=np.array(c["density"]), F=np.array(c["fock"]),
                        J=np.array(c["j"]), K=np.array(c["k"]), n_aux=c["n_aux"], ri_mp2=df["ri_mp2"])
    cd = json.load(open(os.path.join(data, "cd_hf_reference.json")))
    cases = []
    for c in cd["cases"]:
        cases.append({"name": c["name"], "basis": {"STO_3G_GBS": "sto-3g", "BASIS_6_31G_GBS": "6-31g"}[c["basis_constant"]],
                      "atoms": [[a["symbol"], a["position"]] for a in c["atoms"]], "e_rhf": c["e_rhf"],
                      "thresholds": [{k: t[k] for k in ("threshold", "n_vectors", "pivots", "max_residual", "e_cd_hf")}
                                     for t in c["thresholds"]]})
    json.dump({"source": "hf-rs tests/data/cd_hf_reference.json (" + cd["source"] + ")", "cases": cases},
              open(os.path.join(HERE, "cd_hf.json"), "w"), indent=1)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <hf-rs checkout root>")
    main(sys.argv[1])
