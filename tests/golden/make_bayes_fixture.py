"""Writes bayes_a370_head.dat: the column names and the first 4 samples of the reference's
Benchmarks/ConfigFiles/hff_slmodels/A370/bayes.dat (a posterior of the A370 strong-lensing
model that the reference ships), for the bayes.dat reader and column-layout tests.

Run where the reference is present:
    python tests/golden/make_bayes_fixture.py <reference tree>
    (or with the tree in $LT_REFERENCE_TREE)"""
import os
import pathlib
import sys

OUT = pathlib.Path(__file__).resolve().parent / "bayes_a370_head.dat"


def main():
    tree = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("LT_REFERENCE_TREE")
    if not tree:
        sys.exit("give the reference tree as the argument or in LT_REFERENCE_TREE")
    SRC = pathlib.Path(tree) / "Benchmarks/ConfigFiles/hff_slmodels/A370/bayes.dat"
    names, samples = [], []
    for line in SRC.read_text().splitlines():
        if line.startswith("#"):
            names.append(line)
        elif line.strip() and len(samples) < 4:
            samples.append(line)
    OUT.write_text("\n".join(names + samples) + "\n")
    print(f"{OUT}: {len(names)} columns, {len(samples)} samples")


if __name__ == "__main__":
    main()
