"""Extract the Gaussian-94 basis-set blocks this library ships.

The texts are Basis Set Exchange data (cc-pVDZ, STO-3G, 6-31G*, the def2
universal JK fitting set and the def2-SVP RI fitting set) as embedded in the
hf-rs sources (src/basis_data.rs: STO_3G_GBS :15, BASIS_6_31G_STAR_GBS :3344,
BASIS_CC_PVDZ_GBS :19496, AUX_DEF2_UNIVERSAL_JKFIT_GBS :42267,
AUX_DEF2_SVP_RIFIT_GBS :51585).  Only the first-row elements the water
workloads and the parity fixtures need are kept.  Run once from a checkout
that has the hf-rs sources next to it:

    python extract.py /path/to/hf-rs
"""
import os
import re
import sys

SETS = {
    "sto-3g": "STO_3G_GBS",
    "6-31g*": "BASIS_6_31G_STAR_GBS",
    "cc-pvdz": "BASIS_CC_PVDZ_GBS",
    "def2-universal-jkfit": "AUX_DEF2_UNIVERSAL_JKFIT_GBS",
    "def2-svp-ri": "AUX_DEF2_SVP_RIFIT_GBS",
}
ELEMENTS = {"H", "HE", "LI", "BE", "B", "C", "N", "O"}


def blocks(text):
    out, cur = [], []
    for line in text.strip().splitlines():
        cur.append(line)
        if line.strip() == "****":
            out.append(cur)
            cur = []
    return out


def main(root):
    src = open(os.path.join(root, "src", "basis_data.rs")).read()
    here = os.path.dirname(os.path.abspath(__file__))
    for name, const in SETS.items():
        m = re.search(r"pub const " + const + r': &str = r#"(.*?)"#;', src, re.S)
        if not m:
            raise SystemExit("missing " + const)
        keep = []
        for blk in blocks(m.group(1)):
            head = [ln for ln in blk if ln.strip() and not ln.strip().startswith("!")]
            if head and head[0].split()[0].upper() in ELEMENTS:
                keep.append("\n".join(blk))
        fn = os.path.join(here, name.replace("*", "star") + ".gbs")
        with open(fn, "w") as f:
            f.write("\n".join(keep) + "\n")
        print(fn, len(keep), "elements")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
