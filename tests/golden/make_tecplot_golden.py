"""Extracts lines written by ORION's Tecplot ASCII writer (tec_write_structured_multiblock, E23.15E3 values) from the
reference's own test inputs into tests/golden/orion_tecplot_lines.txt (run where the reference's test tree is present:
python tests/golden/make_tecplot_golden.py --reference <path of the MOSE-GPU checkout>, or with the path in the
environment variable MOSE_REFERENCE).

Sources (files of the reference's test tree, written by ORION): test/1D/Sod79/INPUT/ic.tec (a 400-cell block with
cell-centred variables and a subnormal SOLUTIONTIME) and test/2D/viscous/flat-plate-turbulent/SA/MESH/mesh.tec
(a 136 x 96 x 1 mesh). The fixture keeps each file's VARIABLES and ZONE lines and a deterministic sample of its
value lines (every value line of distinct text among the first 4000 and a stride over the rest), so that the
formatter is checked against the writer's own output without shipping the files."""
import argparse
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["test/1D/Sod79/INPUT/ic.tec", "test/2D/viscous/flat-plate-turbulent/SA/MESH/mesh.tec"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MOSE_REFERENCE"))
    args = ap.parse_args()
    if not args.reference:
        raise SystemExit("give the reference checkout with --reference or MOSE_REFERENCE")
    out = []
    for rel in SOURCES:
        with open(os.path.join(args.reference, rel)) as f:
            lines = f.read().split("\n")
        head = [ln for ln in lines[:2]]
        vals = [ln for ln in lines[2:] if ln.strip()]
        seen, sample = set(), []
        for q, ln in enumerate(vals):
            if (q < 4000 and ln not in seen) or q % 97 == 0:
                seen.add(ln)
                sample.append(ln)
        out.append(f"# {rel}: {len(vals)} value lines, {len(sample)} kept")
        out += ["H" + ln for ln in head]
        out += ["V" + ln for ln in sample[:1200]]
    with open(os.path.join(HERE, "orion_tecplot_lines.txt"), "w") as f:
        f.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
