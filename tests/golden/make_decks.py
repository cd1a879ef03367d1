"""Writes tests/golden/reference_decks.json: the keyword settings of the
reference's own test decks (test/01_npme_laplaceDM ... test/04_npme_helmholtzDM
in ElkingD/npme), so the GPU tests can run the same decks through
npme_b200/bin/npme without the reference tree.  Only keyword/value pairs are
kept (the first two words of each line, as the reference's reader does).

    python tests/golden/make_decks.py [reference root]

The reference root is the argument, else $NPME_REFERENCE.
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def keywords(path):
    kv = {}
    with open(path) as f:
        for line in f:
            w = line.split()
            if len(w) >= 2:
                kv[w[0]] = w[1]
    return kv


def main(root=None):
    root = root or os.environ.get("NPME_REFERENCE")
    if not root:
        sys.exit("give the reference root as an argument or in $NPME_REFERENCE")
    decks = {}
    for d in sorted(glob.glob(os.path.join(root, "test", "0[1-4]_*"))):
        name = os.path.basename(d)
        decks[name] = {os.path.basename(f): keywords(f)
                       for f in sorted(glob.glob(os.path.join(d, "*.txt")))}
    with open(os.path.join(HERE, "reference_decks.json"), "w") as f:
        json.dump(decks, f, indent=1, sort_keys=True)
    print(sum(len(v) for v in decks.values()), "deck files")


if __name__ == "__main__":
    main(*sys.argv[1:])
