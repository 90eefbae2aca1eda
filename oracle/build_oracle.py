"""Build recipe for the CPU oracle (test infrastructure): one g++ call, output under oracle/_build/.

-ffp-contract=off keeps every product and sum separately rounded, as the reference's golden
trajectories were generated (upstream C++ in double without FMA contraction) and as the CUDA
collision kernels compute (--fmad=false), so the f32 predicates agree bit for bit.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, '_build', 'liboracle.so')
SRC = os.path.join(HERE, 'avbd_oracle.cpp')


def build(force: bool = False) -> str:
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= os.path.getmtime(SRC):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = ['g++', '-O2', '-std=c++17', '-ffp-contract=off', '-fno-fast-math', '-fPIC', '-shared', '-fopenmp', '-o', OUT, SRC]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv))
