"""Generate the committed golden fixtures under tests/golden/.

The reference (GPU-BLAST over NCBI BLAST+ 2.2.28) ships no tests, fixtures or
known-answer vectors.  (Its kernel source is host-compiled by `make -C oracle
ref` to pin the oracle's algorithm; see oracle/ref_driver.cpp.)  What it ships
as data is its scoring table: the int8 28x28 BLOSUM62 in NCBIstdaa order, held in
``ReadSubstitutionMatrix`` (gpu_blastp.c:44-86, values at :46-75), of which
only the first 640 bytes are sent to the GPU (SUBSTITUTION_MATRIX_LENGTH,
ncbi_blast_files/gpu_cpu_common.h:28).

This script reads that table from the reference source *as text* and writes it
to ``blosum62_ncbistdaa.txt`` (28 rows of 28 integers).  The oracle and the
CUDA path take their matrix from the package's own table; the CPU tests pin
that table against this fixture, so a transcription error in either shows up.

Run from the repository root:  python tests/golden/make_golden.py REF_ROOT
where REF_ROOT is the reference source tree.  The reference is not needed
afterwards: only the generated fixture travels with the tests.
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_reference_blosum(path):
    text = open(path, encoding="latin-1").read()
    start = text.index("Blosum62[28][28]")
    body = text[start:text.index("};", start)]
    rows = []
    for line in body.splitlines():
        if "{" not in line or "}" not in line or "Blosum62" in line:
            continue
        inner = line[line.index("{") + 1:line.index("}")]
        vals = [int(v) for v in re.findall(r"-?\d+", inner)]
        if len(vals) == 28:
            rows.append(vals)
    if len(rows) != 28:
        raise RuntimeError("expected 28 rows, parsed %d" % len(rows))
    return rows


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <reference source root (the tree holding gpu_blastp.c)>")
    ref_root = sys.argv[1]
    rows = parse_reference_blosum(os.path.join(ref_root, "gpu_blastp.c"))
    out = os.path.join(HERE, "blosum62_ncbistdaa.txt")
    with open(out, "w") as f:
        f.write("# int8 BLOSUM62, NCBIstdaa order (28x28), as held by the reference at\n")
        f.write("# gpu_blastp.c:46-75.  Generated by tests/golden/make_golden.py.\n")
        for r in rows:
            f.write(" ".join("%d" % v for v in r) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    main()
