"""Copies the reference's degenerate-hull fixture (tests/fixtures/hull-fracture-glass.json of
three-avbd: 238 points of a Voronoi glass fragment, f32) into this folder. Run once in a container
that has the reference checked out; the copy is committed so the tests never read the reference at
run time."""

import shutil
import sys
from pathlib import Path

src = Path(sys.argv[1] if len(sys.argv) > 1 else '/root/reference') / 'tests' / 'fixtures' / 'hull-fracture-glass.json'
dst = Path(__file__).resolve().parent / 'hull-fracture-glass.json'
shutil.copyfile(src, dst)
print(f'copied {src} to {dst}')
