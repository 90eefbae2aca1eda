"""Copies the reference's degenerate-hull fixture (tests/fixtures/hull-fracture-glass.json of
three-avbd: 238 points of a Voronoi glass fragment, f32) into this folder. Run once with the path
of a three-avbd checkout as its argument; the copy is committed so the tests never read the reference at
run time."""

import shutil
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(f'usage: python {Path(__file__).name} <three-avbd checkout>')
src = Path(sys.argv[1]) / 'tests' / 'fixtures' / 'hull-fracture-glass.json'
dst = Path(__file__).resolve().parent / 'hull-fracture-glass.json'
shutil.copyfile(src, dst)
print(f'copied {src} to {dst}')
