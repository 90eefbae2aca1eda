"""Copies the reference's golden trajectories (tests/fixtures/oracle3d/scene-{0..13}.json of
three-avbd, generated there by upstream avbd-demo3d compiled in double without FMA) into this
folder. Run once with the path of a three-avbd checkout as its argument; the copies are committed so
the tests never read the reference at run time."""

import shutil
import sys
from pathlib import Path

if len(sys.argv) != 2:
    sys.exit(f'usage: python {Path(__file__).name} <three-avbd checkout>')
src = Path(sys.argv[1]) / 'tests' / 'fixtures' / 'oracle3d'
dst = Path(__file__).resolve().parent
for i in range(14):
    shutil.copyfile(src / f'scene-{i}.json', dst / f'scene-{i}.json')
print(f'copied 14 fixtures from {src}')
